"""The CPU oracle against the reference's own property tests (re-expressed) and
against the committed golden fixtures.

The reference ships no golden data; its tests are properties of the modelling
and gradient (test/test_analytic.py, test_linearity_src.py, test_adjoint_src.py,
test_linearization.py, test_jacobian_linearity.py, test_jacobian_adjoint.py).
They pin the restated loops to the physics; the fixtures under tests/golden pin
the oracle against regressions.
"""
import os

import numpy as np
import pytest

import oracle
from owl_b200.geometry import Receiver, Shot, Source

from cases import desc, prepare, random_model, rel, small_shots

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("R", [4, 8])
def test_exact_adjoint_dot_product(fs, R):
    """<J dm, r> = <dm, J^T r> to 1e-10 in FP64 (J dm by complex step)."""
    nx, nz, dx, dt, nt = 40, 32, 10.0, 1e-3, 200
    d = desc(nx, nz, dx, dt, nt, R=R, fs=fs)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx, bool(fs)), nx, nz, dx, dt)
    rng = np.random.default_rng(1)
    dvp, drho = rng.standard_normal((nz, nx)), rng.standard_normal((nz, nx))
    _, jv = oracle.ac2d_jvp(d, vp, rho, dvp, drho, ps)
    r = rng.standard_normal(jv.shape)
    _, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, r, adj_kind=1, k=23)
    lhs = float(np.dot(jv, r))
    rhs = float(np.dot(dvp.T.ravel(), g[:nx * nz]) + np.dot(drho.T.ravel(), g[nx * nz:]))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_complex_step_matches_finite_difference():
    """Interior perturbations (the PML coefficients depend on the edge vp)."""
    nx, nz, dx, dt, nt = 40, 32, 10.0, 1e-3, 200
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    rng = np.random.default_rng(2)
    dvp = np.zeros((nz, nx))
    dvp[3:-3, 3:-3] = rng.standard_normal((nz - 6, nx - 6))
    drho = np.zeros((nz, nx))
    drho[3:-3, 3:-3] = rng.standard_normal((nz - 6, nx - 6))
    _, jv = oracle.ac2d_jvp(d, vp, rho, dvp, drho, ps)
    h = 1e-3
    fp = oracle.ac2d_forward(d, vp + h * dvp, rho + h * drho, ps, "f64")
    fm = oracle.ac2d_forward(d, vp - h * dvp, rho - h * drho, ps, "f64")
    assert rel((fp - fm) / (2 * h), jv) < 1e-6


def test_fp32_vs_fp64():
    nx, nz, dx, dt, nt = 40, 32, 10.0, 1e-3, 300
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    assert rel(oracle.ac2d_forward(d, vp, rho, ps, "f32"), oracle.ac2d_forward(d, vp, rho, ps, "f64")) < 1e-5


def test_golden_fixtures():
    """Regression pin: the oracle reproduces the committed FP64 vectors."""
    from golden.make_golden import golden_case
    z = np.load(os.path.join(HERE, "golden", "ac2d_golden.npz"))
    d, vp, rho, ps, obs = golden_case()
    seis = oracle.ac2d_forward(d, vp, rho, ps, "f64")
    assert rel(seis, z["seis"]) < 1e-12
    mf, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=20)
    assert rel(g, z["grad"]) < 1e-12
    assert rel(mf, z["misfit"]) < 1e-12


# ------------------------- reference Test 1: analytic ------------------------
def analytic_pressure(offset, nt, dt, f0, vp, dx, dz, shift):
    """2D whole-space pressure of an explosion injecting amp*stf*dt into one cell
    per step: p = dx dz (d/dt stf) * G2D, G2D^ = -i/(4 c^2) H0^(2)(w r / c),
    delayed by `shift` (the staggered injection / sampling order)."""
    from scipy.special import hankel2
    from owl_b200.geometry import prepare_stf
    stf, _ = prepare_stf(Source(x=0, z=0, f0=f0), dt)
    npad = 8 * nt
    s = np.zeros(npad)
    s[:len(stf)] = stf
    S = np.fft.rfft(s) * dt
    w = 2 * np.pi * np.fft.rfftfreq(npad, dt)
    with np.errstate(divide="ignore", invalid="ignore"):
        G = (-1j / (4.0 * vp ** 2)) * hankel2(0, w * offset / vp)
    G[0] = 0
    P = dx * dz * (1j * w) * S * G * np.exp(-1j * w * shift)
    return np.fft.irfft(P, n=npad)[:nt] / dt


def test_analytic_wholespace():
    """Per-trace relative L2 error < 5 % (test/test_analytic.py:135)."""
    n, dx, dt, nt, vp, f0 = 121, 10.0, 1e-3, 700, 2000.0, 15.0
    d = desc(n, n, dx, dt, nt, pml=20, f0=f0)
    m = np.full((n, n), vp, dtype=np.float32)
    r = np.ones((n, n), dtype=np.float32)
    c = (n // 2) * dx
    offs = [100.0, 200.0, 300.0, 400.0]
    sh = [Shot(1, [Source(x=c, z=c, f0=f0)], [Receiver(x=c + o, z=c) for o in offs])]
    ps = prepare(sh, n, n, dx, dt)
    seis = oracle.ac2d_forward(d, m, r, ps, "f64").reshape(len(offs), nt)
    for i, o in enumerate(offs):
        a = analytic_pressure(o, nt, dt, f0, vp, dx, dx, 1.5 * dt)
        assert rel(seis[i], a) < 0.05, (o, rel(seis[i], a))


# ------------------- reference Test 2: source linearity ----------------------
def test_source_linearity_and_superposition():
    """Amplitude scaling and two-source superposition, rel < 1e-5 (test_linearity_src.py:53)."""
    nx, nz, dx, dt, nt = 60, 40, 10.0, 1e-3, 300
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    recs = [Receiver(x=50 + 40 * i, z=50.0) for i in range(10)]
    a = Source(x=201.7, z=203.1, f0=15.0)
    b = Source(x=405.0, z=150.0, f0=12.0, amp=-0.7)
    a2 = Source(x=201.7, z=203.1, f0=15.0, amp=2.0)
    shots = [Shot(1, [a], recs), Shot(2, [b], recs), Shot(3, [a, b], recs), Shot(4, [a2], recs)]
    s = oracle.ac2d_forward(d, vp, rho, prepare(shots, nx, nz, dx, dt), "f32").reshape(4, -1)
    assert rel(s[0] + s[1], s[2]) < 1e-5
    assert rel(2 * s[0], s[3]) < 1e-5


# ---------------------- reference Test 3: reciprocity ------------------------
def test_reciprocity():
    """d(A -> B) = d(B -> A) for explosion sources and pressure receivers at the
    same bulk modulus (laterally invariant model), rel < 1e-3 (test_adjoint_src.py:46)."""
    nx, nz, dx, dt, nt = 60, 50, 10.0, 1e-3, 500
    d = desc(nx, nz, dx, dt, nt)
    z = np.arange(nz)[:, None] * dx
    vp = np.broadcast_to(2000 + 1.5 * z, (nz, nx)).astype(np.float32)
    rho = np.broadcast_to(1500 + 0.5 * z, (nz, nx)).astype(np.float32)
    pairs = [((100.0, 200.0), (450.0, 200.0)), ((150.0, 300.0), (420.0, 300.0))]
    for (ax, az), (bx, bz) in pairs:
        sh = [Shot(1, [Source(x=ax, z=az, f0=15.0)], [Receiver(x=bx, z=bz)]),
              Shot(2, [Source(x=bx, z=bz, f0=15.0)], [Receiver(x=ax, z=az)])]
        s = oracle.ac2d_forward(d, vp, rho, prepare(sh, nx, nz, dx, dt), "f64").reshape(2, nt)
        assert rel(s[0], s[1]) < 1e-3


# ----------------- reference Test 4: Taylor (linearisation) ------------------
def test_taylor_second_order():
    """||F(m + h dm) - F(m) - h J dm|| shrinks as h^2: slope >= 1.9 (test_linearization.py:122)."""
    nx, nz, dx, dt, nt = 60, 50, 10.0, 1e-3, 400
    d = desc(nx, nz, dx, dt, nt)
    z = np.arange(nz)[:, None] * dx
    vp = np.broadcast_to(2000 + 1.0 * z, (nz, nx)).astype(np.float64)
    rho = np.full((nz, nx), 1000.0)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    dvp = 0.1 * vp * np.exp(-((zz - 30) ** 2 + (xx - 30) ** 2) / (2 * 8.0 ** 2))
    sh = [Shot(1, [Source(x=300.0, z=50.0, f0=15.0)], [Receiver(x=30 + 40 * i, z=50.0) for i in range(14)])]
    ps = prepare(sh, nx, nz, dx, dt)
    f0, jv = oracle.ac2d_jvp(d, vp, rho, dvp, np.zeros_like(rho), ps)
    hs = [0.4, 0.2, 0.1, 0.05]
    e = [np.linalg.norm(oracle.ac2d_forward(d, vp + h * dvp, rho, ps, "f64") - f0 - h * jv) for h in hs]
    slopes = np.diff(np.log(e)) / np.diff(np.log(hs))
    assert np.all(slopes >= 1.9), slopes


# --------------- reference Test 5: Jacobian (FD Born) linearity --------------
def test_fd_born_linearity():
    """FD Born responses scale and superpose within 5 % (test_jacobian_linearity.py:46)."""
    nx, nz, dx, dt, nt = 60, 50, 10.0, 1e-3, 400
    d = desc(nx, nz, dx, dt, nt)
    vp = np.full((nz, nx), 2200.0)
    rho = np.full((nz, nx), 1000.0)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    g1 = 100 * np.exp(-((zz - 30) ** 2 + (xx - 20) ** 2) / 50.0)
    g2 = 100 * np.exp(-((zz - 35) ** 2 + (xx - 40) ** 2) / 50.0)
    sh = [Shot(1, [Source(x=300.0, z=50.0, f0=15.0)], [Receiver(x=30 + 40 * i, z=50.0) for i in range(14)])]
    ps = prepare(sh, nx, nz, dx, dt)
    eps = 0.02
    f = lambda m: oracle.ac2d_forward(d, m, rho, ps, "f64")
    base = f(vp)
    b1 = (f(vp + eps * g1) - base) / eps
    b2 = (f(vp + eps * g2) - base) / eps
    b12 = (f(vp + eps * (g1 + g2)) - base) / eps
    b1x2 = (f(vp + eps * 2 * g1) - base) / eps
    assert rel(b1 + b2, b12) < 0.05
    assert rel(2 * b1, b1x2) < 0.05


# --------------- reference Test 6: gradient consistency ----------------------
def test_gradient_consistency():
    """Central differences of J = 0.5 |syn - obs|^2 against <g, dm> for three probes:
    the reference asks the ratio to agree within 3 % (test_jacobian_adjoint.py:75);
    the exact adjoint in FP64 agrees to 1e-6."""
    nx, nz, dx, dt, nt = 50, 40, 10.0, 1e-3, 300
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz, seed=4)
    vp, rho = vp.astype(np.float64), rho.astype(np.float64)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp * 1.03, rho, ps, "f64")
    _, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=30)
    J = lambda m, r: 0.5 * float(np.sum((oracle.ac2d_forward(d, m, r, ps, "f64") - obs) ** 2))
    rng = np.random.default_rng(7)
    for _ in range(3):
        dv = np.zeros((nz, nx))
        dv[4:-4, 4:-4] = rng.standard_normal((nz - 8, nx - 8))
        dr = np.zeros((nz, nx))
        dr[4:-4, 4:-4] = rng.standard_normal((nz - 8, nx - 8))
        h = 1e-2
        D = (J(vp + h * dv, rho + h * dr) - J(vp - h * dv, rho - h * dr)) / (2 * h)
        G = float(np.dot(dv.T.ravel(), g[:nx * nz]) + np.dot(dr.T.ravel(), g[nx * nz:]))
        assert abs(D - G) <= 1e-6 * abs(G), (D, G)


def test_reference_gradient_loosely_agrees():
    """The reference's -dt back-propagated gradient is not the exact one (it skips
    the first half-wavelet and reconstructs the source field approximately);
    it must still point the same way: positive correlation of the vp gradients
    away from the source."""
    nx, nz, dx, dt, nt = 60, 50, 10.0, 1e-3, 500
    d = desc(nx, nz, dx, dt, nt)
    z = np.arange(nz)[:, None] * dx
    vp = np.broadcast_to(2000 + 2.0 * z, (nz, nx)).astype(np.float32)
    rho = np.full((nz, nx), 1000.0, dtype=np.float32)
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    vpt = vp + 150 * np.exp(-((zz - 30) ** 2 + (xx - 30) ** 2) / 40.0)
    sh = [Shot(1, [Source(x=300.0, z=40.0, f0=15.0)], [Receiver(x=20 + 20 * i, z=40.0) for i in range(27)])]
    ps = prepare(sh, nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vpt, rho, ps, "f32")
    syn = oracle.ac2d_forward(d, vp, rho, ps, "f32")
    _, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=50, precision="f64")
    gref = oracle.ac2d_ref_gradient(d, vp, rho, ps, syn - obs, cc=1)
    a = g[:nx * nz].reshape(nx, nz).T[8:, :].astype(np.float64)
    b = gref[:nx * nz].reshape(nx, nz).T[8:, :].astype(np.float64)
    assert np.linalg.norm(b) > 0
    corr = float(np.sum(a * b) / np.linalg.norm(a) / np.linalg.norm(b))
    assert corr > 0.8, corr
