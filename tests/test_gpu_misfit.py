"""GPU test of the misfit-only batched forward (step-length trial forwards)
through the C ABI: per-shot and per-trace FP64 waveform misfits against the
synthetics of owl_ssg_forward, and against the misfit of owl_ssg_gradient."""
import numpy as np
import pytest

from owl_b200 import _lib as L
from owl_b200.solver import RunOpts, SSGSolver

from cases import desc, prepare, random_model, small_shots

pytestmark = pytest.mark.gpu


def test_misfit_matches_forward_and_gradient():
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 300
    d = desc(nx, nz, dx, dt, nt, R=4)
    vp, rho = random_model(nx, nz)
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, nx, nz, dx, dx, dt, nt, pml=d.pml, fdhalf=4, f0_max=d.f0_max, max_shots=8)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    s.set_model(vp * 1.03, rho)
    obs = s.forward(ps)
    s.set_model(vp, rho)
    # one tile shape for every call: the one-cell and four-cell kernels agree
    # to rounding only (the compiler contracts their sums differently), and the
    # autotuner's pick may differ between batch sizes
    syn = s.forward(ps, RunOpts(tile_z=8))
    seis = np.zeros_like(syn)
    for opts in (RunOpts(tile_z=8), RunOpts(tile_z=8, shots_per_launch=1, use_graph=-1)):
        m, tm = s.misfit(ps, obs, opts, traces=True, seis_out=seis)
        assert np.array_equal(seis, syn)
        off, t0 = 0, 0
        for sh, gather in enumerate(s.split(ps, syn)):
            n = gather.size
            o = obs[off:off + n].reshape(gather.shape).astype(np.float64)
            want_traces = np.sum((o - gather) ** 2, axis=-1).ravel()
            want_traces[[r for r in range(ps.nrec(sh)) if ps.arr[sh].rec[r].weight == 0]] = 0
            got = tm[t0:t0 + want_traces.size]
            assert np.allclose(got, want_traces, rtol=1e-12, atol=0)
            assert m[sh] == pytest.approx(float(np.sum(want_traces)), rel=1e-12)
            off += n
            t0 += want_traces.size
    mg, _ = s.gradient(ps, obs, opts=RunOpts(tile_z=8))
    assert np.allclose(mg, m, rtol=1e-9)
    # the autotuned forward and gradient of one batch size share the forward kernels
    ma = s.misfit(ps, obs)
    mga, _ = s.gradient(ps, obs)
    assert np.allclose(mga, ma, rtol=1e-9)
