"""CPU tests of the 3D elastic oracle (restated reference loops + exact adjoint).

Pinned by properties (the reference ships no elastic test): the exact adjoint
passes the dot-product test against complex-step directional derivatives for the
isotropic, tilted-Thomsen and orthorhombic (nine Cij) parameterisations with explosion,
force and moment-tensor sources, with and without the free surface; the misfit
gradient matches the complex-step derivative of J; FP32 and FP64 forwards agree.
"""
import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots, Receiver, Shot, Source
from owl_b200.solver import elastic_time_integration

from cases import rel

N, DX, DT, NT = 16, 10.0, 1e-3, 80


def el3_desc(aniso=L.OWL_ANISO_ISO, R=4, nt=NT, fs=0):
    d = L.OwlSsgDesc()
    d.medium = L.OWL_ELASTIC_VHTIORT_3D
    d.nx = d.ny = d.nz = N
    d.dx = d.dy = d.dz = DX
    d.pml, d.fdhalf, d.free_surface = 5, R, fs
    d.dt, d.nt, d.f0_max, d.max_shots = DT, nt, 20.0, 4
    d.aniso = aniso
    return d


def el3_model(aniso, seed=1):
    rng = np.random.default_rng(seed)
    vp = 2000 + 300 * rng.random((N, N, N))
    vs = vp / 1.7
    rho = 1000 + 200 * rng.random((N, N, N))
    if aniso == L.OWL_ANISO_ISO:
        return [vp, vs, rho]
    if aniso == L.OWL_ANISO_THOMSEN:
        # tilted orthorhombic-free TI: epsilon, delta, gamma, tilt theta and azimuth phi (radians)
        eps = 0.05 + 0.15 * rng.random((N, N, N))
        dlt = -0.05 + 0.15 * rng.random((N, N, N))
        gam = 0.1 * rng.random((N, N, N))
        the = 0.4 * rng.random((N, N, N))
        phi = rng.random((N, N, N))
        return [vp, vs, eps, dlt, gam, the, phi, rho]
    c11, c44 = rho * vp ** 2, rho * vs ** 2
    return [1.1 * c11, c11 - 2 * c44, 0.9 * (c11 - 2 * c44), c11, c11 - 2 * c44, 0.95 * c11, c44, 1.05 * c44,
            0.9 * c44, rho]


def el3_shots(fs=0):
    if not fs:
        return [Shot(1, [Source(x=73.3, y=61.7, z=81.7, f0=20.0),
                         Source(x=60.0, y=80.0, z=50.0, mechanism="force", polar=30, azimuth=40, f0=20.0),
                         Source(x=90.0, y=70.0, z=90.0, mechanism="mt", mt=[1, 0.5, 0.7, 0.3, 0.2, 0.1], f0=18.0)],
                     [Receiver(x=30 + 17.3 * i, y=40 + 5.1 * i, z=30.0 + 3 * i) for i in range(5)])]
    # free surface: shallow sources whose taps cross the surface rows, receivers
    # on and just below the surface (their taps read the velocity images)
    return [Shot(1, [Source(x=73.3, y=61.7, z=21.7, f0=20.0),
                     Source(x=60.0, y=80.0, z=15.0, mechanism="force", polar=30, azimuth=40, f0=20.0),
                     Source(x=90.0, y=70.0, z=30.0, mechanism="mt", mt=[1, 0.5, 0.7, 0.3, 0.2, 0.1], f0=18.0)],
                 [Receiver(x=30 + 17.3 * i, y=40 + 5.1 * i, z=0.0 if i % 2 == 0 else 3.7 * i) for i in range(5)])]


def el3_prep(shots):
    return PreparedShots(shots, GridSpec(nx=N, nz=N, dx=DX, dz=DX, ny=N, dy=DX), DT,
                         time_integration=elastic_time_integration)


def _dot(g, dm):
    nm = N ** 3
    return sum(float(np.dot(g[q * nm:(q + 1) * nm], np.asfortranarray(dm[q]).ravel(order="F"))) for q in range(len(dm)))


@pytest.mark.parametrize("aniso,fs", [(L.OWL_ANISO_ISO, 0), (L.OWL_ANISO_CIJ, 0), (L.OWL_ANISO_ISO, 1),
                                      (L.OWL_ANISO_CIJ, 1), (L.OWL_ANISO_THOMSEN, 0), (L.OWL_ANISO_THOMSEN, 1)])
def test_el3d_adjoint_dot_product(aniso, fs):
    d = el3_desc(aniso, fs=fs)
    f = el3_model(aniso)
    ps = el3_prep(el3_shots(fs))
    rng = np.random.default_rng(7)
    dm = [rng.standard_normal(x.shape) * np.std(x) * 1e-3 for x in f]
    seis, jvp = oracle.el3d_jvp(d, f, dm, ps)
    r = rng.standard_normal(seis.shape)
    _, g, _ = oracle.el3d_gradient(d, f, ps, r, adj_kind=L.OWL_ADJ_GIVEN, k=7)
    lhs, rhs = float(np.dot(jvp, r)), _dot(g, dm)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("fs", [0, 1])
def test_el3d_misfit_gradient_matches_complex_step(fs):
    d = el3_desc(L.OWL_ANISO_ISO, fs=fs)
    f = el3_model(L.OWL_ANISO_ISO)
    ps = el3_prep(el3_shots(fs))
    obs = oracle.el3d_forward(d, el3_model(L.OWL_ANISO_ISO, seed=2), ps, "f64")
    rng = np.random.default_rng(3)
    dm = [rng.standard_normal(x.shape) * np.std(x) * 1e-3 for x in f]
    syn, jvp = oracle.el3d_jvp(d, f, dm, ps)
    dj = float(np.dot(syn - obs, jvp))
    misfit, g, _ = oracle.el3d_gradient(d, f, ps, obs, adj_kind=L.OWL_ADJ_L2_RESIDUAL, k=30)
    assert abs(dj - _dot(g, dm)) <= 1e-9 * abs(dj)
    assert misfit[0] == pytest.approx(float(np.sum((obs - syn) ** 2)), rel=1e-12)


@pytest.mark.parametrize("fs", [0, 1])
def test_el3d_f32_matches_f64(fs):
    d = el3_desc(L.OWL_ANISO_CIJ, R=8, fs=fs)
    f = el3_model(L.OWL_ANISO_CIJ)
    ps = el3_prep(el3_shots(fs))
    s32 = oracle.el3d_forward(d, f, ps, "f32")
    s64 = oracle.el3d_forward(d, f, ps, "f64")
    assert np.linalg.norm(s64) > 0
    assert rel(s32, s64) < 1e-5


def test_el3d_free_surface_reflects():
    """with the free surface, the surface receivers see the surface reflection:
    the traces differ from those of the absorbing top (same model and shots)"""
    f = el3_model(L.OWL_ANISO_ISO)
    ps = el3_prep(el3_shots(1))
    a = oracle.el3d_forward(el3_desc(fs=0), f, ps, "f64")
    b = oracle.el3d_forward(el3_desc(fs=1), f, ps, "f64")
    assert np.all(np.isfinite(b)) and rel(b, a) > 0.1
