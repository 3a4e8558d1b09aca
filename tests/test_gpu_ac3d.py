"""GPU parity tests of the 3D acoustic path through the C ABI: forward against
the FP32 oracle (1e-5 relative L2), gradient against the FP64 exact-adjoint
oracle (1e-4)."""
import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots, Receiver, Shot, Source
from owl_b200.solver import RunOpts, SSGSolver

from cases import desc, rel

pytestmark = pytest.mark.gpu


def case3(fs=0, R=4, nt=150):
    nx, ny, nz, dx, dt = 26, 22, 20, 10.0, 1e-3
    d = desc(nx, nz, dx, dt, nt, pml=6, R=R, fs=fs, ny=ny, medium=L.OWL_ACOUSTIC_ISO_3D)
    rng = np.random.default_rng(5)
    vp = (2000 + 300 * rng.random((nz, ny, nx))).astype(np.float32)
    rho = (1000 + 200 * rng.random((nz, ny, nx))).astype(np.float32)
    z0 = 0.0 if fs else 33.3
    shots = [
        Shot(1, [Source(x=123.3, y=101.7, z=91.2, f0=20.0)],
             [Receiver(x=30 + 23.3 * i, y=40.0 + 7 * i, z=z0 + 10) for i in range(7)]),
        Shot(2, [Source(x=90.0, y=80.0, z=100.0, f0=18.0, mechanism="force", polar=35.0, azimuth=20.0)],
             [Receiver(x=40 + 30 * i, y=110.0, z=150.0) for i in range(5)]),
    ]
    ps = PreparedShots(shots, GridSpec(nx=nx, nz=nz, dx=dx, dz=dx, ny=ny, dy=dx), dt)
    return d, vp, rho, ps


def solver3(d, vp, rho):
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=bool(d.free_surface), f0_max=d.f0_max, max_shots=4, ny=d.ny, dy=d.dy)
    s.set_model(vp, rho)
    return s


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("R", [4, 8])
def test_forward_parity_3d(fs, R):
    d, vp, rho, ps = case3(fs, R)
    ref = oracle.ac3d_forward(d, vp, rho, ps, "f32")
    s = solver3(d, vp, rho)
    for opts in (RunOpts(), RunOpts(shots_per_launch=1, use_graph=-1, tile_z=2)):
        got = s.forward(ps, opts)
        assert rel(got, ref) < 1e-5, (opts, rel(got, ref))


@pytest.mark.parametrize("fs", [0, 1])
def test_gradient_parity_3d(fs):
    d, vp, rho, ps = case3(fs)
    ps = PreparedShots(ps.shots[:1], GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz, ny=d.ny, dy=d.dy), d.dt)
    obs = oracle.ac3d_forward(d, vp, rho, ps, "f64").astype(np.float32)
    vp0 = vp * np.float32(1.02)
    mf_ref, g_ref = oracle.ac3d_gradient(d, vp0, rho, ps, obs, adj_kind=0, k=30)
    s = solver3(d, vp0, rho)
    # tile_z 1: the ring kernels in both passes
    for opts in (RunOpts(checkpoint_interval=30), RunOpts(checkpoint_interval=40, use_graph=-1, tile_z=8),
                 RunOpts(checkpoint_interval=30, tile_z=1)):
        mf, g = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, opts)
        assert rel(mf, mf_ref) < 1e-4
        assert rel(g, g_ref) < 1e-4, (opts, rel(g, g_ref))


@pytest.mark.parametrize("fs", [0, 1])
def test_ring_adjoint_matches_tiled(fs):
    """two shots in one CTA: the ring adjoint (one Kahan update per shot) and the
    tiled adjoint (shots summed, then one update) agree to FP32 rounding"""
    d, vp, rho, ps = case3(fs)
    ps = PreparedShots(ps.shots[:2], GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz, ny=d.ny, dy=d.dy), d.dt)
    obs = oracle.ac3d_forward(d, vp, rho, ps, "f32").astype(np.float32)
    s = solver3(d, vp * np.float32(1.02), rho)
    mf1, g1 = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, RunOpts(checkpoint_interval=30, tile_z=1, shots_per_cta=2))
    g1 = g1.copy()
    mf4, g4 = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, RunOpts(checkpoint_interval=30, tile_z=4, shots_per_cta=2))
    assert rel(g1, g4) < 1e-5, rel(g1, g4)
    assert np.allclose(mf1, mf4, rtol=1e-6)


_REF3 = {}


def _ref3_gradient():
    """FP64 oracle gradient of the 3D case (one shot, vp 2 % high), computed once."""
    if not _REF3:
        d, vp, rho, ps = case3(0, nt=200)
        ps = PreparedShots(ps.shots[:1], GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz, ny=d.ny, dy=d.dy), d.dt)
        obs = oracle.ac3d_forward(d, vp, rho, ps, "f64").astype(np.float32)
        vp0 = vp * np.float32(1.02)
        _, g_ref = oracle.ac3d_gradient(d, vp0, rho, ps, obs, adj_kind=0, k=25)
        _REF3.update(d=d, vp0=vp0, rho=rho, ps=ps, obs=obs, g=g_ref)
    return _REF3


@pytest.mark.parametrize("prec,tol", [(L.OWL_CKPT_FP32, 1e-4), (L.OWL_CKPT_FP16, 2e-3), (L.OWL_CKPT_BF16, 2e-2)])
def test_gradient_checkpoint_precision_3d(prec, tol):
    """3D forward + adjoint vp/rho gradient with FP32, FP16 and BF16 checkpoints
    (per-field, per-shot scale for the 16-bit ones), each against the FP64
    exact-adjoint oracle."""
    r = _ref3_gradient()
    s = solver3(r["d"], r["vp0"], r["rho"])
    _, g = s.gradient(r["ps"], r["obs"], L.OWL_ADJ_L2_RESIDUAL,
                      RunOpts(checkpoint_interval=25, checkpoint_precision=prec))
    e = rel(g, r["g"])
    print("3D checkpoint precision", prec, "gradient rel err vs FP64 oracle", e)
    assert e < tol, e


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("R", [4, 8])
def test_tma_forward_kernels_match_cp_async_ring(fs, R):
    """The TMA ring forward kernels (tile_z 11 / 12 / 14: 1 / 2 / 4 rows per
    thread) load the same tiles as the cp.async ring kernels (tile_z 1 / 2 / 4)
    and compute the same arithmetic: seismograms equal to the bit, and within
    1e-5 of the FP32 oracle; the gradient's forward and recomputed steps run
    on them too."""
    d, vp, rho, ps = case3(fs, R)
    ref = oracle.ac3d_forward(d, vp, rho, ps, "f32")
    s = solver3(d, vp, rho)
    for rows in (1, 2, 4):
        a = s.forward(ps, RunOpts(tile_z=rows))
        b = s.forward(ps, RunOpts(tile_z=10 + rows))
        assert np.array_equal(a, b), rows
        assert rel(b, ref) < 1e-5, (rows, rel(b, ref))
    ps1 = PreparedShots(ps.shots[:1], GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz, ny=d.ny, dy=d.dy), d.dt)
    obs = oracle.ac3d_forward(d, vp, rho, ps1, "f64").astype(np.float32)
    vp0 = vp * np.float32(1.02)
    _, g_ref = oracle.ac3d_gradient(d, vp0, rho, ps1, obs, adj_kind=0, k=30)
    s0 = solver3(d, vp0, rho)
    _, g = s0.gradient(ps1, obs, opts=RunOpts(checkpoint_interval=30, tile_z=12))
    assert rel(g, g_ref) < 1e-4, rel(g, g_ref)


_C3 = {}


@pytest.mark.parametrize("prec,tol", [(L.OWL_CKPT_FP32, 1e-4), (L.OWL_CKPT_FP16, 2e-3), (L.OWL_CKPT_BF16, 2e-2)])
def test_c3_kind_checkpoint_precision(prec, tol):
    """The 3D acoustic workload scaled down to a 48^3 model (its layered model
    generator with the 5 % lateral perturbation and Gardner rho, dx 10 m, dt
    1 ms, 20-cell PML, 8th order, the 12 Hz source at the centre, 24 x 24
    receivers every 20 m at z = 20 m), 300 steps, observed data from a 3 %
    faster model, checkpoints every 50 steps in FP32 / FP16 / BF16 (per-field,
    per-shot scale): the vp / rho gradient against the FP64 exact-adjoint
    oracle of the same stencil."""
    from owl_b200 import configs
    if not _C3:
        d, vp, rho, shots = configs.config3(48, nt=300)
        ps = PreparedShots(shots, GridSpec(nx=d.nx, nz=d.nz, dx=d.dx, dz=d.dz, ny=d.ny, dy=d.dy), d.dt)
        obs = oracle.ac3d_forward(d, (vp * np.float32(1.03)).astype(np.float32), rho, ps, "f64").astype(np.float32)
        _, g_ref = oracle.ac3d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=50)
        _C3.update(d=d, vp=vp, rho=rho, ps=ps, obs=obs, g=g_ref)
    r = _C3
    d = r["d"]
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, ny=d.ny, dy=d.dy)
    s.set_model(r["vp"], r["rho"])
    _, g = s.gradient(r["ps"], r["obs"], L.OWL_ADJ_L2_RESIDUAL, RunOpts(checkpoint_interval=50, checkpoint_precision=prec))
    e = rel(g, r["g"])
    print(f"c3-kind 48^3 gradient, checkpoint precision {prec}: rel err vs FP64 oracle {e:.3e}")
    assert e < tol, e
