"""CPU tests of the depth-refined free-surface mesh of the elastic 2D solver
(src/solver/elastic_vhtiort_2d/module_vars.f90:313-376).

The product's mesh (owl_vertical_mesh, host code of the C ABI) equals the
oracle's restatement bit for bit; the mesh has the reference's shape (rows
dz / refine apart down to (refine_rows - 1) dz, then 2.5 % wider per row up
to dz_max, down to the model's depth); refine_rows follows
ceil(0.5 lambda_R / dz); the geometry lands sources and receivers on the
mesh's rows with the reference's nearest-row rule; and the oracle's exact
adjoint on the refined mesh passes the dot-product test against complex-step
Jacobian-vector products, so the transpose of the regular-to-mesh row
interpolation is exact.
"""
import math

import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots, Receiver, Shot, Source
from owl_b200.solver import elastic_geometry, elastic_time_integration, free_surface_refine_rows, vertical_mesh

from test_oracle_el2d import DT, DX, NX, NZ, el_model


def refined_desc(rr=4.0, dz_max=15.0, rows=3, aniso=L.OWL_ANISO_ISO, nz=NZ, pml=8, nt=160):
    d = L.OwlSsgDesc()
    d.medium = L.OWL_ELASTIC_VHTIORT_2D
    d.nx, d.ny, d.nz = NX, 1, nz
    d.dx = d.dy = d.dz = DX
    d.pml, d.fdhalf, d.free_surface = pml, 4, 1
    d.dt, d.nt, d.f0_max, d.max_shots = DT / 4, nt, 15.0, 4
    d.aniso = aniso
    d.free_surface_dz_refine, d.dz_max, d.free_surface_refine_rows = rr, dz_max, rows
    return d


@pytest.mark.parametrize("rr,dz_max,rows", [(4.0, 15.0, 3), (4.0, 10.0, 5), (2.0, 12.5, 1), (1.0, 15.0, 2),
                                            (3.0, 10.0, 4)])
def test_mesh_matches_oracle_and_shape(rr, dz_max, rows):
    d = refined_desc(rr, dz_max, rows)
    m = vertical_mesh(d)
    n, zi, zh, dzi, dzh = oracle.el2d_mesh(d)
    assert m is not None and len(m.z_i) == n + 2 * d.pml + 2
    for a, b in zip((m.z_i, m.z_h, m.dz_i, m.dz_h), (zi, zh, dzi, dzh)):
        assert np.array_equal(a, b)
    P = d.pml
    z = m.z_i[P + 1:P + 1 + n]  # rows 1 .. n
    h = np.diff(z)
    fine = np.float32(DX) / np.float32(rr)
    nfine = int(round((rows - 1) * DX / fine))
    assert z[0] == 0.0
    assert np.allclose(h[:nfine], fine, rtol=1e-6)
    # below the fine rows each spacing grows by 2.5 % until it reaches dz_max
    g = h[nfine:]
    # (spacings as differences of float32 depths of a few hundred metres: 1e-4 m)
    assert np.all(g <= dz_max + 1e-4)
    assert np.all(np.diff(g) >= -1e-4)
    grow = g[1:] / g[:-1]
    assert np.all((np.abs(grow - 1.025) < 1e-4) | (np.abs(g[1:] - dz_max) < 1e-4))
    # the last row reaches the model's depth, the one before does not
    assert z[-1] >= (NZ - 1) * DX and z[-2] < (NZ - 1) * DX
    # half rows between the integer rows, one half spacing above the surface
    assert m.z_h[P + 1] == -0.5 * fine
    assert np.allclose(m.z_h[P + 2:P + 1 + n], 0.5 * (z[:-1] + z[1:]))
    # spacings: centred differences, edge values in the padding
    assert np.allclose(m.dz_i[P + 2:P + n], 0.5 * (z[2:] - z[:-2]))
    assert np.all(m.dz_i[:P + 1] == m.dz_i[P + 1]) and np.all(m.dz_i[P + n:] == m.dz_i[P + n])


def test_uniform_mesh_rows():
    d = refined_desc(1.0, DX, 0)
    nz = C_int_mesh(d)
    assert nz == NZ
    assert vertical_mesh(d) is None
    d2 = refined_desc(0.0, 0.0, 0)
    assert C_int_mesh(d2) == NZ and vertical_mesh(d2) is None


def C_int_mesh(d):
    import ctypes as C
    n = C.c_int()
    L.check(L.load().owl_vertical_mesh(C.byref(d), C.byref(n), None, None, None, None))
    return n.value


def test_mesh_rejects_bad_descriptors():
    with pytest.raises(L.OwlError):
        vertical_mesh(refined_desc(4.0, 15.0, 0))      # refine rows unset
    with pytest.raises(L.OwlError):
        vertical_mesh(refined_desc(4.0, 1.0, 3))       # dz_max below dz / refine
    with pytest.raises(L.OwlError):
        vertical_mesh(refined_desc(0.5, 15.0, 3))      # coarsening factor


def test_refine_rows_formula():
    """refine_nz = ceiling(0.5 sqrt(mean(c55 / rho)) / f0_min / dz) over the
    padded surface row (module_vars.f90:315-317)."""
    d = refined_desc()
    f = el_model(L.OWL_ANISO_ISO)
    vs, rho = f[1].astype(np.float32), f[2].astype(np.float32)
    row = np.concatenate([[vs[0, 0]] * (d.pml + 1), vs[0, :], [vs[0, -1]] * (d.pml + 1)]).astype(np.float32)
    rrow = np.concatenate([[rho[0, 0]] * (d.pml + 1), rho[0, :], [rho[0, -1]] * (d.pml + 1)]).astype(np.float32)
    c55 = (rrow * (row * row)).astype(np.float32)
    lam = math.sqrt(float(np.mean((c55 / rrow).astype(np.float64)))) / 12.0
    want = math.ceil(0.5 * lam / DX)
    got = free_surface_refine_rows(d, f, 12.0)
    assert abs(got - want) <= 0 or abs(0.5 * lam / DX - round(0.5 * lam / DX)) < 1e-5, (got, want)


def refined_shots():
    return [Shot(1, [Source(x=203.3, z=31.7, f0=15.0),
                     Source(x=120.0, z=0.0, mechanism="force", polar=20, f0=15.0),
                     Source(x=250.0, z=120.0, mechanism="mt", mt=[1, 0, 0.5, 0, 0.3, 0], f0=12.0)],
                 [Receiver(x=50 + 37.3 * i, z=[0.0, 3.1, 17.0][i % 3]) for i in range(8)])]


def refined_prep(d, shots):
    m = vertical_mesh(d)
    return PreparedShots(elastic_geometry(shots, d, m), GridSpec(nx=NX, nz=NZ, dx=DX, dz=DX, zmesh=m), d.dt,
                         time_integration=elastic_time_integration)


def test_geometry_on_mesh():
    """Nearest mesh row (first on a tie; z = 0 on the half row below the
    surface), taps from the offset over the row's spacing; a surface source
    moves to dz_i(1) with 1.2 x amplitude."""
    d = refined_desc()
    m = vertical_mesh(d)
    ps = refined_prep(d, refined_shots())
    src = ps.arr[0].src
    # the force source at z = 0 moved to dz_i(1) = dz / 4: on integer row 2
    assert src[1].gz == 2 and abs(src[1].amp - 1.2) < 1e-6
    assert np.allclose(src[1].interp_iz[:], np.eye(9)[4], atol=1e-7)
    # explosion at 31.7 m: its nearest integer row and the offset taps
    zi = m.z_i
    g = int(np.argmin(np.abs(np.float32(31.7) - zi))) - d.pml
    assert src[0].gz == g
    rec = ps.arr[0].rec
    assert rec[0].gz == 1 and rec[0].hz == 2  # z = 0: surface row, half row below it


@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_THOMSEN])
def test_refined_adjoint_dot_product(aniso):
    """<J dm, r> = <dm, J^T r> on the refined mesh: the model perturbation on
    the regular rows, its image on the mesh through the linear row
    interpolation, the gradient back through its transpose."""
    d = refined_desc(aniso=aniso, nt=120)
    f = el_model(aniso)
    ps = refined_prep(d, refined_shots())
    rng = np.random.default_rng(11)
    dm = [rng.standard_normal((NZ, NX)) * np.std(x) * 1e-3 for x in f]
    seis, jvp = oracle.el2d_jvp(d, f, dm, ps)
    r = rng.standard_normal(seis.shape)
    _, g, _ = oracle.el2d_gradient(d, f, ps, r, adj_kind=L.OWL_ADJ_GIVEN, k=7)
    nm = NX * NZ
    lhs = float(np.dot(jvp, r))
    rhs = sum(float(np.dot(g[q * nm:(q + 1) * nm], np.asfortranarray(dm[q]).ravel(order="F"))) for q in range(len(f)))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def test_refined_forward_differs_from_uniform_and_is_stable():
    """The refined mesh changes the answer (the scalings act), stays finite,
    and its dt_stable is set by the finest rows."""
    d = refined_desc(nt=200)
    f = el_model(L.OWL_ANISO_ISO)
    ps = refined_prep(d, refined_shots())
    a = oracle.el2d_forward(d, f, ps, "f64")
    assert np.all(np.isfinite(a)) and np.max(np.abs(a)) > 0
    dt_ref = oracle.el2d_dt_stable(d, f)
    du = refined_desc(1.0, DX, 0, nt=200)
    assert dt_ref < oracle.el2d_dt_stable(du, f)
    pu = PreparedShots(elastic_geometry(refined_shots(), du), GridSpec(nx=NX, nz=NZ, dx=DX, dz=DX), du.dt,
                       time_integration=elastic_time_integration)
    b = oracle.el2d_forward(du, f, pu, "f64")
    assert np.linalg.norm(a - b) > 1e-3 * np.linalg.norm(b)


# ------------------------------ elastic 3D ----------------------------------
def refined_desc3(aniso=L.OWL_ANISO_ISO, rr=2.0, dz_max=12.5, rows=2, nt=100):
    from test_oracle_el3d import N
    d = L.OwlSsgDesc()
    d.medium = L.OWL_ELASTIC_VHTIORT_3D
    d.nx = d.ny = d.nz = N
    d.dx = d.dy = d.dz = DX
    d.pml, d.fdhalf, d.free_surface = 5, 4, 1
    d.dt, d.nt, d.f0_max, d.max_shots = 5e-4, nt, 20.0, 4
    d.aniso = aniso
    d.free_surface_dz_refine, d.dz_max, d.free_surface_refine_rows = rr, dz_max, rows
    return d


def refined_prep3(d, shots):
    from test_oracle_el3d import N
    m = vertical_mesh(d)
    return PreparedShots(elastic_geometry(shots, d, m), GridSpec(nx=N, nz=N, dx=DX, dz=DX, ny=N, dy=DX, zmesh=m),
                         d.dt, time_integration=elastic_time_integration)


@pytest.mark.parametrize("aniso", [L.OWL_ANISO_ISO, L.OWL_ANISO_CIJ])
def test_refined_adjoint_dot_product_3d(aniso):
    """The elastic 3D oracle on the refined mesh: exact adjoint against
    complex-step Jacobian-vector products of the forward."""
    from test_oracle_el3d import el3_model, el3_shots, _dot
    d = refined_desc3(aniso, nt=60)
    f = el3_model(aniso)
    ps = refined_prep3(d, el3_shots(1))
    rng = np.random.default_rng(7)
    dm = [rng.standard_normal(x.shape) * np.std(x) * 1e-3 for x in f]
    seis, jvp = oracle.el3d_jvp(d, f, dm, ps)
    r = rng.standard_normal(seis.shape)
    _, g, _ = oracle.el3d_gradient(d, f, ps, r, adj_kind=L.OWL_ADJ_GIVEN, k=7)
    lhs, rhs = float(np.dot(jvp, r)), _dot(g, dm)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def test_refine_rows_3d_formula():
    """3D refine_nz: the largest of the means of c44 / rho, c55 / rho, c66 / rho
    over the padded surface plane (module_vars.f90:424-428 of the 3D solver)."""
    from test_oracle_el3d import N, el3_model
    d = refined_desc3(L.OWL_ANISO_CIJ)
    f = el3_model(L.OWL_ANISO_CIJ)
    P = d.pml
    idx = np.clip(np.arange(-P, N + P + 2), 1, N) - 1
    rho = f[9][0][np.ix_(idx, idx)].astype(np.float32)  # (y, x) at the surface (z index 0)
    means = [float(np.mean((f[q][0][np.ix_(idx, idx)].astype(np.float32) / rho).astype(np.float64)))
             for q in (6, 7, 8)]
    lam = math.sqrt(max(means)) / 17.0
    want = math.ceil(0.5 * lam / DX)
    assert free_surface_refine_rows(d, f, 17.0) == want
