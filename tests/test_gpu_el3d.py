"""GPU parity tests of the 3D elastic path through the C ABI, with and without
the free surface: forward (vx, vy, vz) vs the FP32 oracle at 1e-5 relative L2;
gradient vs the FP64 exact-adjoint oracle at 1e-4; source-side gradient. The
anisotropic parameterisations run with their M-PML damping ratios (nonzero),
the isotropic one with zero ratios, as the reference."""
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
    """The solver of the model; the oracle runs that follow use the M-PML face
    ratios the library computed for it (all zero for iso), which
    test_mpml_faces_match_the_restated_search checks separately."""
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=bool(d.free_surface), f0_max=d.f0_max, max_shots=d.max_shots, ny=d.ny, dy=d.dy,
                  aniso=d.aniso)
    s.set_model(*f)
    faces = s.mpml_ratios()
    oracle.el3d_set_mpml(faces if np.any(faces) else None)
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


@pytest.mark.parametrize("fs", [0, 1])
@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_CIJ])
def test_mpml_faces_match_the_restated_search(aniso, fs):
    """The library's six face-ratio arrays: zero for iso; for anisotropic media
    the damping-ratio search at every 10th face cell, interpolated, exactly as
    the oracle's restatement of compute_damping_profile_ratio_face arranges it
    (fed the library's own single-cell search, which test_mpml_cpu checks
    against the literal 27 x 27 eigen-derivative form)."""
    from oracle import oracle_mpml as M
    d = el3_desc(aniso, fs=fs)
    f = el3_model(aniso)
    s = make(d, f)
    faces = s.mpml_ratios()
    if aniso == L.OWL_ANISO_ISO:
        assert not np.any(faces)
        return
    assert np.all(faces >= 0) and np.any(faces > 0)
    lib = L.load()
    P, n = d.pml, N
    npad = n + 2 * P
    # stiffness of a face cell: the model's edge cell (the padded model replicates it)
    C9 = [np.asarray(f[q], dtype=np.float32) for q in range(9)]

    def c_at(i, j, k):  # reference indices, clamped to the model
        ii, jj, kk = (min(max(v, 1), n) - 1 for v in (i, j, k))
        return np.array([c[ii, jj, kk] for c in C9], dtype=np.float32)

    def lib_ratio(c, direction):
        cc = np.ascontiguousarray(c, dtype=np.float32)
        return float(lib.owl_mpml_damp_ratio(cc.ctypes.data_as(L.C.POINTER(L.C.c_float)), "xyz".index(direction)))

    z1 = 1 if fs else -P + 1
    nzf = n + P - z1 + 1
    fx, fy, fz = npad * npad, npad * npad, npad * npad
    views = [faces[0:fx].reshape(npad, npad), faces[fx:2 * fx].reshape(npad, npad),
             faces[2 * fx:2 * fx + fy].reshape(npad, npad), faces[2 * fx + fy:2 * fx + 2 * fy].reshape(npad, npad),
             faces[2 * fx + 2 * fy:2 * fx + 2 * fy + fz].reshape(npad, npad), faces[2 * fx + 2 * fy + fz:].reshape(npad, npad)]
    zoff = z1 + P - 1
    specs = [("x", lambda a, b: c_at(1, -P + 1 + a, z1 + b), npad, nzf, zoff),
             ("x", lambda a, b: c_at(n, -P + 1 + a, z1 + b), npad, nzf, zoff),
             ("y", lambda a, b: c_at(-P + 1 + a, 1, z1 + b), npad, nzf, zoff),
             ("y", lambda a, b: c_at(-P + 1 + a, n, z1 + b), npad, nzf, zoff),
             ("z", lambda a, b: c_at(-P + 1 + a, -P + 1 + b, 1), npad, npad, 0),
             ("z", lambda a, b: c_at(-P + 1 + a, -P + 1 + b, n), npad, npad, 0)]
    for (direction, cell, n1, n2, off), got in zip(specs, views):
        cf = np.array([[cell(a, b) for b in range(n2)] for a in range(n1)])
        want = M.face_ratio(cf, direction, ratio_fn=lib_ratio)  # (n1, n2)
        assert np.allclose(got[off:off + n2, :].T, want, rtol=0, atol=1e-6), direction
        if off:
            assert not np.any(got[:off])


# ------------- depth-refined free-surface mesh (module_vars.f90:419-490) -------------
def make_refined(d, f):
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=True, f0_max=d.f0_max, max_shots=d.max_shots, ny=d.ny, dy=d.dy, aniso=d.aniso,
                  free_surface_dz_refine=d.free_surface_dz_refine, dz_max=d.dz_max,
                  refine_rows=d.free_surface_refine_rows)
    s.set_model(*f)
    faces = s.mpml_ratios()
    oracle.el3d_set_mpml(faces if np.any(faces) else None)
    return s


@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_CIJ, L.OWL_ANISO_THOMSEN])
def test_el3d_refined_forward_and_gradient_parity(aniso):
    """Refined mesh (planes dz / 2 apart near the surface, 2.5 % wider per
    plane up to 1.25 dz): forward vs the FP32 oracle, gradient (mesh-cell
    correlations, the transpose of the depth interpolation and the chain rule
    in FP64 on the regular planes) vs the FP64 exact-adjoint oracle."""
    from test_refined_mesh_cpu import refined_desc3, refined_prep3
    d = refined_desc3(aniso, nt=100)
    f = el3_model(aniso)
    s = make_refined(d, f)
    ps = s.prepare(el3_shots(1) * 2)
    ref = oracle.el3d_forward(d, f, ps, "f32")
    for opts in (RunOpts(), RunOpts(shots_per_launch=1, use_graph=-1), RunOpts(shots_per_cta=2)):
        got = s.forward(ps, opts)
        assert rel(got, ref) < FWD_TOL, (opts, rel(got, ref))
    assert abs(s.dt_stable - oracle.el3d_dt_stable(d, f)) <= 1e-6 * s.dt_stable
    obs = oracle.el3d_forward(d, el3_model(aniso, seed=2), ps, "f64").astype(np.float32)
    mref, gref, _ = oracle.el3d_gradient(d, f, ps, obs, adj_kind=L.OWL_ADJ_L2_RESIDUAL, k=7)
    for opts in (RunOpts(checkpoint_interval=7), RunOpts(checkpoint_interval=7, shots_per_launch=1, use_graph=-1)):
        misfit, g = s.gradient(ps, obs, opts=opts)
        assert rel(g, gref) < GRAD_TOL, (opts, rel(g, gref))
        assert np.allclose(misfit, mref, rtol=1e-4)


def test_el3d_refined_source_gradient_parity():
    from test_refined_mesh_cpu import refined_desc3
    d = refined_desc3(L.OWL_ANISO_ISO, nt=80)
    f = el3_model(L.OWL_ANISO_ISO)
    s = make_refined(d, f)
    ps = s.prepare(el3_shots(1))
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
