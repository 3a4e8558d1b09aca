"""CPU tests of the elastic 2D oracle (restated reference loops + exact adjoint).

The reference ships no test or golden vector for its elastic solvers, so the
oracle is pinned by properties: the exact adjoint passes the dot-product test
against complex-step Jacobian-vector products of the forward, FP32 and FP64
forwards agree, the wavefield is linear in the source, elastic reciprocity
holds between vertical forces and vertical-velocity receivers, the Cij set-up
reduces to the isotropic one when the anisotropy vanishes, and dt_stable
follows module_vars.f90:408-420.
"""
import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots, Receiver, Shot, Source
from owl_b200.solver import elastic_geometry, elastic_time_integration

from cases import rel

NX, NZ, DX, DT, NT = 40, 36, 10.0, 1e-3, 200


def el_desc(fs=0, aniso=L.OWL_ANISO_ISO, R=4, nt=NT, pml=8):
    d = L.OwlSsgDesc()
    d.medium = L.OWL_ELASTIC_VHTIORT_2D
    d.nx, d.ny, d.nz = NX, 1, NZ
    d.dx = d.dy = d.dz = DX
    d.pml, d.fdhalf, d.free_surface = pml, R, fs
    d.dt, d.nt, d.f0_max, d.max_shots = DT, nt, 15.0, 4
    d.aniso = aniso
    return d


def el_model(aniso, seed=1):
    rng = np.random.default_rng(seed)
    vp = 2000 + 300 * rng.random((NZ, NX))
    vs = vp / 1.8
    rho = 1000 + 200 * rng.random((NZ, NX))
    eps = 0.1 * rng.random((NZ, NX))
    de = 0.05 * rng.random((NZ, NX))
    th = 0.2 * rng.random((NZ, NX))
    if aniso == L.OWL_ANISO_ISO:
        return [vp, vs, rho]
    if aniso in (L.OWL_ANISO_THOMSEN, L.OWL_ANISO_AT):
        return [vp, vs, eps, de, th, rho]
    c33, c55 = rho * vp ** 2, rho * vs ** 2
    return [1.2 * c33, c33 - 2 * c55, c33, c55, rho]


def el_shots(fs):
    zr = 0.0 if fs else 42.0
    return [Shot(1, [Source(x=203.3, z=151.7, f0=15.0),
                     Source(x=120.0, z=100.0, mechanism="force", polar=30, f0=15.0),
                     Source(x=250.0, z=200.0, mechanism="mt", mt=[1, 0, 0.5, 0, 0.3, 0], f0=12.0)],
                 [Receiver(x=50 + 37.3 * i, z=zr + 10.0 * (i % 3)) for i in range(8)])]


def prep(d, shots):
    return PreparedShots(elastic_geometry(shots, d), GridSpec(nx=NX, nz=NZ, dx=DX, dz=DX), DT,
                         time_integration=elastic_time_integration)


@pytest.mark.parametrize("fs,aniso", [(0, L.OWL_ANISO_ISO), (1, L.OWL_ANISO_ISO), (0, L.OWL_ANISO_THOMSEN),
                                      (1, L.OWL_ANISO_THOMSEN), (1, L.OWL_ANISO_AT), (0, L.OWL_ANISO_CIJ)])
def test_el2d_adjoint_dot_product(fs, aniso):
    """<J dm, r> = <dm, J^T r>: the gradient of <F(m), r> from the exact adjoint
    against the complex-step directional derivative of the forward."""
    d = el_desc(fs, aniso)
    f = el_model(aniso)
    ps = prep(d, el_shots(fs))
    rng = np.random.default_rng(7)
    dm = [rng.standard_normal((NZ, NX)) * np.std(x) * 1e-3 for x in f]
    seis, jvp = oracle.el2d_jvp(d, f, dm, ps)
    r = rng.standard_normal(seis.shape)
    _, g, _ = oracle.el2d_gradient(d, f, ps, r, adj_kind=L.OWL_ADJ_GIVEN, k=7)
    nm = NX * NZ
    lhs = float(np.dot(jvp, r))
    rhs = sum(float(np.dot(g[q * nm:(q + 1) * nm], np.asfortranarray(dm[q]).ravel(order="F"))) for q in range(len(f)))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def test_el2d_misfit_gradient_matches_complex_step():
    """d/dh J(m + h dm) (complex step through the forward) = <grad J, dm>, J = 0.5 |syn - obs|^2."""
    d = el_desc(1, L.OWL_ANISO_THOMSEN)
    f = el_model(L.OWL_ANISO_THOMSEN)
    ps = prep(d, el_shots(1))
    obs = oracle.el2d_forward(d, el_model(L.OWL_ANISO_THOMSEN, seed=2), ps, "f64")
    rng = np.random.default_rng(3)
    dm = [rng.standard_normal((NZ, NX)) * np.std(x) * 1e-3 for x in f]
    syn, jvp = oracle.el2d_jvp(d, f, dm, ps)
    dj = float(np.dot(syn - obs, jvp))
    misfit, g, _ = oracle.el2d_gradient(d, f, ps, obs, adj_kind=L.OWL_ADJ_L2_RESIDUAL, k=50)
    nm = NX * NZ
    gd = sum(float(np.dot(g[q * nm:(q + 1) * nm], np.asfortranarray(dm[q]).ravel(order="F"))) for q in range(len(f)))
    assert abs(dj - gd) <= 1e-9 * abs(dj), (dj, gd)
    assert misfit[0] == pytest.approx(float(np.sum((obs - syn) ** 2)), rel=1e-12)


@pytest.mark.parametrize("fs", [0, 1])
def test_el2d_f32_matches_f64(fs):
    d = el_desc(fs, L.OWL_ANISO_THOMSEN, R=8)
    f = el_model(L.OWL_ANISO_THOMSEN)
    ps = prep(d, el_shots(fs))
    s32 = oracle.el2d_forward(d, f, ps, "f32")
    s64 = oracle.el2d_forward(d, f, ps, "f64")
    assert np.linalg.norm(s64) > 0
    assert rel(s32, s64) < 1e-5


def test_el2d_linear_in_source_amplitude():
    d = el_desc(0, L.OWL_ANISO_ISO)
    f = el_model(L.OWL_ANISO_ISO)
    a = oracle.el2d_forward(d, f, prep(d, [Shot(1, [Source(x=200.0, z=150.0, f0=15.0)],
                                                  [Receiver(x=100.0 + 20 * i, z=50.0) for i in range(5)])]), "f64")
    b = oracle.el2d_forward(d, f, prep(d, [Shot(1, [Source(x=200.0, z=150.0, f0=15.0, amp=-2.5)],
                                                  [Receiver(x=100.0 + 20 * i, z=50.0) for i in range(5)])]), "f64")
    assert rel(b, -2.5 * a) < 1e-12


def test_el2d_reciprocity_vertical_force():
    """vz at B from a vertical force at A equals vz at A from the same force at B
    (constant density, so the 1/rho force scaling is the same at both ends; the
    injection and sampling taps are the same interpolation vectors)."""
    d = el_desc(0, L.OWL_ANISO_ISO, nt=300)
    vp, vs, _ = el_model(L.OWL_ANISO_ISO)
    f = [vp, vs, np.full_like(vp, 1500.0)]
    A, B = (120.0, 100.0), (260.0, 210.0)

    def vz_trace(s, r):
        sh = [Shot(1, [Source(x=s[0], z=s[1], mechanism="force", polar=0.0, f0=15.0)], [Receiver(x=r[0], z=r[1])])]
        return oracle.el2d_forward(d, f, prep(d, sh), "f64")[300:]  # (vx, vz) traces of nt = 300

    ab, ba = vz_trace(A, B), vz_trace(B, A)
    assert np.linalg.norm(ab) > 0
    assert rel(ab, ba) < 1e-3


def test_el2d_thomsen_without_anisotropy_is_isotropic():
    d_iso = el_desc(0, L.OWL_ANISO_ISO)
    d_th = el_desc(0, L.OWL_ANISO_THOMSEN)
    vp, vs, rho = el_model(L.OWL_ANISO_ISO)
    z = np.zeros_like(vp)
    ps = prep(d_iso, el_shots(0))
    a = oracle.el2d_forward(d_iso, [vp, vs, rho], ps, "f64")
    b = oracle.el2d_forward(d_th, [vp, vs, z, z, z, rho], ps, "f64")
    # same Cij; only the M-PML ratio (non-zero for non-iso parameterisations) differs
    assert rel(b, a) < 1e-3


def test_el2d_dt_stable_formula():
    d = el_desc(0, L.OWL_ANISO_THOMSEN)
    vp, vs, eps, de, th, rho = el_model(L.OWL_ANISO_THOMSEN)
    z = np.zeros_like(vp)
    f = [vp, vs, eps, de, z, rho]
    c = np.array([0.1217990e+1, -0.9382142e-1, 0.1507536e-1, -0.1700324e-2])
    vmax = np.max(np.sqrt(1 + 2 * eps) * vp)  # c11 / rho = vp^2 (1 + 2 eps) >= c33 / rho
    want = 1.0 / (np.sum(np.abs(c)) * vmax * np.sqrt(2.0 / DX ** 2))
    assert oracle.el2d_dt_stable(d, f) == pytest.approx(want, rel=1e-5)


def test_el2d_mpml_ratio_range():
    rho, vp = 2000.0, 3000.0
    vs = vp / 1.8
    c33, c55 = rho * vp * vp, rho * vs * vs
    for eps, de in [(0.0, 0.0), (0.2, 0.1), (0.3, -0.1)]:
        c11 = c33 * (1 + 2 * eps)
        c13 = abs(2 * c33 * (c33 - c55) * de + (c33 - c55) ** 2) ** 0.5 - c55
        for direction in ("x", "z"):
            r = oracle.el2d_damp_ratio(c11, c13, c33, c55, rho, direction)
            assert 0.0 < r <= 1.0
