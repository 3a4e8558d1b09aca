"""The forward of a gradient stores the stencil terms of its last segment, so
the reverse sweep recomputes every segment but that one. With the last segment
shorter than the checkpoint interval (nt % k != 0) and the time loop with and
without CUDA graphs, the gradient equals, to the bit, the one whose last
segment is checkpointed and recomputed like the others (OWL_NO_STORE_LAST=1,
a switch kept for this test): 2D acoustic, 3D acoustic and 3D elastic."""
import os

import numpy as np
import pytest

import oracle
from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots
from owl_b200.solver import RunOpts, SSGSolver

from cases import desc, prepare, random_model, small_shots

pytestmark = pytest.mark.gpu


def _both(s, ps, obs, k, graph):
    out = []
    for recompute_last in (False, True):
        if recompute_last:
            os.environ["OWL_NO_STORE_LAST"] = "1"
        try:
            mf, g = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, RunOpts(checkpoint_interval=k, use_graph=graph))
            out.append((np.array(mf, copy=True), np.array(g, copy=True)))
        finally:
            os.environ.pop("OWL_NO_STORE_LAST", None)
    return out


@pytest.mark.parametrize("graph", [0, -1])
def test_store_last_ac2d(graph):
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 300
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp, rho, ps, "f32").astype(np.float32)
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, nx, nz, dx, dx, dt, nt, pml=d.pml, fdhalf=4, f0_max=d.f0_max, max_shots=8)
    s.set_model(vp * np.float32(1.02), rho)
    (m0, g0), (m1, g1) = _both(s, ps, obs, 37, graph)  # 300 = 8 x 37 + 4
    assert np.array_equal(g0, g1) and np.array_equal(m0, m1)


@pytest.mark.parametrize("graph", [0, -1])
def test_store_last_ac3d(graph):
    from test_gpu_ac3d import case3, solver3
    d, vp, rho, ps = case3(0, nt=150)
    obs = oracle.ac3d_forward(d, vp, rho, ps, "f32").astype(np.float32)
    s = solver3(d, vp * np.float32(1.02), rho)
    (m0, g0), (m1, g1) = _both(s, ps, obs, 40, graph)  # 150 = 3 x 40 + 30
    assert np.array_equal(g0, g1) and np.array_equal(m0, m1)


@pytest.mark.parametrize("graph", [0, -1])
def test_store_last_el3d(graph):
    from test_oracle_el3d import el3_desc, el3_model, el3_shots
    d = el3_desc(L.OWL_ANISO_ISO)
    f = el3_model(L.OWL_ANISO_ISO)
    s = SSGSolver(L.OWL_ELASTIC_VHTIORT_3D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  f0_max=d.f0_max, max_shots=d.max_shots, ny=d.ny, dy=d.dy, aniso=d.aniso)
    s.set_model(*f)
    ps = s.prepare(el3_shots(0))
    obs = np.zeros(s.seis_size(ps), dtype=np.float32)
    (m0, g0), (m1, g1) = _both(s, ps, obs, 7, graph)  # 80 = 11 x 7 + 3
    assert np.array_equal(g0, g1) and np.array_equal(m0, m1)
