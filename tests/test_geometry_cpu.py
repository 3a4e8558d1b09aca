"""Kaiser-windowed sinc taps (module_source_receiver.f90:789-828) checked against
an independent restatement built on SciPy's modified Bessel function
(scipy.special.i0) and NumPy's normalised sinc, at the fractional offsets the
headline workload's off-grid sources have (x = 100 + k 3800/31 m on a 10 m
grid, integer and half nodes), plus the on-grid delta."""
import numpy as np
import scipy.special

from owl_b200 import configs
from owl_b200.geometry import GridSpec, PreparedShots, bessel_i0, kaiser_sinc_kernel

B0 = 6.31
NKW = 4


def independent_taps(x: float) -> np.ndarray:
    i = np.arange(-NKW, NKW + 1, dtype=np.float64)
    t = i - x
    w = np.where(np.abs(t) <= NKW, scipy.special.i0(B0 * np.sqrt(np.clip(1.0 - (t / NKW) ** 2, 0.0, None))), 0.0)
    return np.sinc(t) * w / scipy.special.i0(B0)


def test_bessel_i0_matches_scipy():
    for x in np.linspace(0.0, 6.31, 64):
        assert abs(bessel_i0(x) - scipy.special.i0(x)) <= 1e-14 * scipy.special.i0(x)


def test_taps_of_headline_sources_match_independent_restatement():
    d, _, _, shots = configs.config2(32)
    ps = PreparedShots(shots, GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz), d.dt)
    offsets = 0
    for k, sh in enumerate(shots):
        src = ps.arr[k].src[0]
        xs = sh.sources[0].x
        for half, node, taps in ((False, src.gx, src.interp_ix), (True, src.hx, src.interp_hx)):
            # the offset in single precision, as the reference's real arithmetic forms it
            f32 = np.float32
            q = f32(f32(f32(xs) + f32(0.5) * f32(d.dx)) / f32(d.dx)) if half else f32(f32(xs) / f32(d.dx))
            frac = float(f32(q - f32(node - 1)))
            got = np.array(taps[:], dtype=np.float64)
            ref = independent_taps(frac)
            # single-precision taps against a double-precision restatement
            assert np.max(np.abs(got - ref)) < 1e-6, (k, frac, got, ref)
            offsets += abs(frac) > 1e-6
    assert offsets >= 30  # most headline sources are off the grid


def test_on_grid_offset_is_a_delta():
    h = kaiser_sinc_kernel(0.0)
    assert h[NKW] == 1.0 and np.count_nonzero(h) == 1
    assert np.allclose(independent_taps(0.0), np.eye(2 * NKW + 1)[NKW], atol=1e-15)


def test_taps_sweep_of_offsets():
    for x in np.linspace(-0.5, 0.5, 41):
        assert np.max(np.abs(kaiser_sinc_kernel(x) - independent_taps(float(np.float32(x))))) < 2e-6
