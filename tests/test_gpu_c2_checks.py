"""Gradient checks of the batched 2D acoustic GPU gradient on the grid and shot
set of the headline workload (201 x 401, dx 10 m, 20-cell CFS-PML, 8th order,
dt 1 ms, 32 shots x 100..3900 m with +-1500 m receiver spreads, starting model
= true model smoothed by a 150 m Gaussian, every-50-step checkpoints):

1. central differences of the FP64 oracle's misfit 0.5 sum (syn - obs)^2 with
   h = 1e-3 Vp at 8 interior cells drawn with numpy.random.default_rng(2026),
   against the 32-shot batched GPU gradient. The time axis is cut to its first
   500 of the 2000 steps (the 16 FP64 forwards of 32 shots over all 2000 steps
   would take the oracle about 20 minutes); the cells are drawn from the part
   of the model those steps illuminate, depths 120-300 m (at least 10 cells
   below the source / receiver row at 20 m and 10 cells inside the model edges
   that the PML surrounds). Bar: 1e-4 relative L2 over the 8 cells.
2. the model-gradient dot product <J dm, r> = <dm, J^T r> with J dm from the
   FP64 oracle's complex-step linearised forward and J^T r from the GPU adjoint
   (the adjoint source r given), random dm on (Vp, rho) and random r, 4 of the
   shots over 500 steps. Bar: 1e-6 relative.
"""
import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200 import configs
from owl_b200.solver import RunOpts, SSGSolver

pytestmark = pytest.mark.gpu

NT = 500
FD_TOL = 1e-4
DOT_TOL = 1e-6


def _setup(nshots):
    d, (vp, rho), (vp0, rho0), shots = configs.config2(32)
    d.nt = NT
    shots = shots[:nshots]
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, d.nx, d.nz, d.dx, d.dz, d.dt, NT, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=nshots)
    ps = s.prepare(shots)
    return d, vp, rho, vp0, rho0, s, ps


def _cells(nx, nz):
    rng = np.random.default_rng(2026)
    cells = []
    while len(cells) < 8:
        iz = int(rng.integers(12, 31))        # 120..300 m: >= 10 cells below the 20 m source / receiver row
        ix = int(rng.integers(10, nx - 10))   # >= 10 cells inside the model edges (the PML lies outside)
        if (iz, ix) not in cells and iz <= nz - 11:
            cells.append((iz, ix))
    return cells


def test_c2_gradient_vs_central_differences():
    d, vp, rho, vp0, rho0, s, ps = _setup(32)
    s.set_model(vp, rho)
    obs = s.forward(ps)
    s.set_model(vp0, rho0)
    _, g = s.gradient(ps, obs, opts=RunOpts(checkpoint_interval=50))
    g = np.asarray(g, dtype=np.float64).reshape(2, d.nx, d.nz)  # (param, x, z): z fastest
    obs64 = obs.astype(np.float64)

    def misfit(v):
        syn = oracle.ac2d_forward(d, v, rho0, ps, "f64")
        return 0.5 * float(np.sum((syn - obs64) ** 2))

    fd, gg = [], []
    for iz, ix in _cells(d.nx, d.nz):
        h = 1e-3 * float(vp0[iz, ix])
        vp_p = vp0.astype(np.float64).copy()
        vp_m = vp_p.copy()
        vp_p[iz, ix] += h
        vp_m[iz, ix] -= h
        fd.append((misfit(vp_p) - misfit(vp_m)) / (2 * h))
        gg.append(g[0, ix, iz])
    fd, gg = np.array(fd), np.array(gg)
    e = float(np.linalg.norm(gg - fd) / np.linalg.norm(fd))
    print("cells", _cells(d.nx, d.nz))
    print("FD", fd)
    print("GPU", gg)
    print(f"c2 batched gradient vs central differences of the FP64 misfit (8 cells): rel {e:.3e}")
    assert e < FD_TOL, e


def test_c2_model_gradient_dot_product():
    d, vp, rho, vp0, rho0, s, ps = _setup(4)
    s.set_model(vp0, rho0)
    rng = np.random.default_rng(7)
    dvp = rng.standard_normal(vp0.shape)
    drho = rng.standard_normal(rho0.shape)
    _, jvp = oracle.ac2d_jvp(d, vp0, rho0, dvp, drho, ps)
    r = rng.standard_normal(jvp.shape).astype(np.float32)
    _, g = s.gradient(ps, r, adj_kind=L.OWL_ADJ_GIVEN, opts=RunOpts(checkpoint_interval=50))
    g = np.asarray(g, dtype=np.float64).reshape(2, d.nx, d.nz)
    lhs = float(np.dot(jvp, r.astype(np.float64)))
    rhs = float(np.sum(g[0] * dvp.T) + np.sum(g[1] * drho.T))
    e = abs(lhs - rhs) / abs(lhs)
    print(f"<J dm, r> = {lhs:.12e}, <dm, J^T r> = {rhs:.12e}, rel {e:.3e}")
    assert e < DOT_TOL, e
