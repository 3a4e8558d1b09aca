"""GPU parity tests of the 3D elastic path through the C ABI, with and without
the free surface: forward (vx, vy, vz) vs the FP32 oracle at 1e-5 relative L2;
gradient vs the FP64 exact-adjoint oracle at 1e-4; source-side gradient."""
import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.solver import RunOpts, SSGSolver

from cases import rel
from test_oracle_el3d import DX, N, el3_desc, el3_model, el3_shots

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def make(d, f):
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=bool(d.free_surface), f0_max=d.f0_max, max_shots=d.max_shots, ny=d.ny, dy=d.dy,
                  aniso=d.aniso)
    s.set_model(*f)
    return s


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("R", [4, 8])
@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_CIJ, L.OWL_ANISO_THOMSEN])
def test_el3d_forward_parity(R, aniso, fs):
    d = el3_desc(aniso, R=R, fs=fs)
    f = el3_model(aniso)
    s = make(d, f)
    ps = s.prepare(el3_shots(fs) * 2)
    ref = oracle.el3d_forward(d, f, ps, "f32")
    # tile_z=1: the z-marching ring kernels (half-width 4, no free surface; else the per-cell ones)
    for opts in (RunOpts(), RunOpts(shots_per_launch=1, use_graph=-1), RunOpts(shots_per_cta=2),
                 RunOpts(tile_z=1), RunOpts(tile_z=1, shots_per_cta=2)):
        got = s.forward(ps, opts)
        assert rel(got, ref) < FWD_TOL, (opts, rel(got, ref))
    assert abs(s.dt_stable - oracle.el3d_dt_stable(d, f)) <= 1e-6 * s.dt_stable


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_CIJ, L.OWL_ANISO_THOMSEN])
def test_el3d_gradient_parity(aniso, fs):
    d = el3_desc(aniso, fs=fs)
    f = el3_model(aniso)
    s = make(d, f)
    ps = s.prepare(el3_shots(fs) * 2)
    obs = oracle.el3d_forward(d, el3_model(aniso, seed=2), ps, "f64").astype(np.float32)
    mref, gref, _ = oracle.el3d_gradient(d, f, ps, obs, adj_kind=L.OWL_ADJ_L2_RESIDUAL, k=7)
    for opts in (RunOpts(checkpoint_interval=7), RunOpts(checkpoint_interval=7, shots_per_launch=1, use_graph=-1),
                 RunOpts(checkpoint_interval=7, tile_z=1)):
        misfit, g = s.gradient(ps, obs, opts=opts)
        assert rel(g, gref) < GRAD_TOL, (opts, rel(g, gref))
        assert np.allclose(misfit, mref, rtol=1e-4)


@pytest.mark.parametrize("fs", [0, 1])
def test_el3d_source_gradient_parity(fs):
    d = el3_desc(L.OWL_ANISO_ISO, fs=fs)
    f = el3_model(L.OWL_ANISO_ISO)
    s = make(d, f)
    ps = s.prepare(el3_shots(fs))
    adj = np.random.default_rng(5).standard_normal(s.seis_size(ps)).astype(np.float32)
    _, _, sref = oracle.el3d_gradient(d, f, ps, adj, adj_kind=L.OWL_ADJ_GIVEN, k=7, stf_grad=True)
    got = s.source_gradient(ps, adj, RunOpts(checkpoint_interval=7))
    mask = np.zeros_like(sref, dtype=bool)
    off = 0
    for sh in range(ps.nshots):
        for k in range(ps.arr[sh].nsrc):
            q = ps.arr[sh].src[k]
            for t in range(max(1, q.nbeg), min(d.nt, q.nbeg + q.nt_stf - 1) + 1):
                mask[off + t - 1] = True
            off += d.nt
    assert rel(got[mask], sref[mask]) < GRAD_TOL


def test_el3d_half_checkpoints_of_tiny_fields():
    """the orthorhombic c5 model on 96^3 (136^3 padded), 300 steps: its force
    source gives wavefields some of whose checkpointed fields have a largest
    value below the smallest normal float; FP16 / BF16 checkpoints keep the
    gradient finite and within 1e-3 of the FP32-checkpoint gradient (a
    reciprocal of such a scale overflowed and turned the field's zeros into
    NaN)."""
    from owl_b200 import configs
    d, f, shots = configs.config5(1, nt=300, n=96, nrec=32)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=1, ny=d.ny, dy=d.dy, aniso=d.aniso)
    s.set_model(*f)
    ps = s.prepare(shots)
    obs = np.zeros(s.seis_size(ps), dtype=np.float32)
    _, g32 = s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=50))
    g32 = np.array(g32, copy=True)
    assert np.all(np.isfinite(g32))
    for prec in (L.OWL_CKPT_FP16, L.OWL_CKPT_BF16):
        _, g = s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=50, checkpoint_precision=prec))
        assert np.all(np.isfinite(g)), prec
        assert rel(g, g32) < 1e-3, (prec, rel(g, g32))
