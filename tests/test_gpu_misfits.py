"""GPU data-domain misfits (owl_adjoint_source, owl_ssg_gradient_misfit)
against the FP64 misfit oracle.

* adjoint sources and trace misfits of every misfit type, host and device
  buffers, gathers with a weight-0 trace, a trace below the discard threshold
  and a zero trace; FP32 transforms on the GPU, so 1e-4 relative L2 (waveform
  and correlation 1e-6);
* the gradient of each misfit through the solver equals the FP64 exact-adjoint
  oracle gradient driven by the oracle's adjoint source (1e-4; 2e-4 where the
  adjoint source depends nonlinearly on the FP32 synthetics).
"""
import numpy as np
import pytest

import oracle
import oracle.oracle_misfit as M
from owl_b200 import _lib as L
from owl_b200.solver import MisfitOpts, RunOpts, adjoint_source

from cases import desc, prepare, random_model, rel, small_shots
from test_gpu_ac2d import make_solver

pytestmark = pytest.mark.gpu

KINDS = [L.OWL_MISFIT_WAVEFORM, L.OWL_MISFIT_CORR, L.OWL_MISFIT_ENVELOPE, L.OWL_MISFIT_PHASE,
         L.OWL_MISFIT_ADAPTIVE, L.OWL_MISFIT_LOCAL_ADAPTIVE, L.OWL_MISFIT_ADAPTIVE_SPACETIME]


def _gathers(nt, seed=3):
    """two gathers: 5 and 4 traces of band-limited wavelets with shifts and
    amplitude changes; trace 1 has weight 0, trace 6 is 1e-8 of its gather's
    largest, trace 8 is zero in the synthetics"""
    rng = np.random.default_rng(seed)
    t = np.arange(nt)
    rows_o, rows_s = [], []
    for i in range(9):
        c = nt * (0.3 + 0.05 * i)
        f = 0.08 + 0.01 * i
        o = np.exp(-((t - c) / (0.04 * nt)) ** 2) * np.cos(f * (t - c)) + 0.02 * rng.standard_normal(nt)
        sh = 2.0 + i
        s = 0.85 * np.exp(-((t - c - sh) / (0.04 * nt)) ** 2) * np.cos(f * (t - c - sh)) + 0.02 * rng.standard_normal(nt)
        rows_o.append(o)
        rows_s.append(s)
    obs = np.array(rows_o, dtype=np.float32)
    syn = np.array(rows_s, dtype=np.float32)
    obs[6] *= 1e-8
    syn[8] = 0.0
    w = np.ones(9, dtype=np.float32)
    w[1] = 0.0
    return [0, 5, 9], syn, obs, w


def _mopts(kind, dt):
    return MisfitOpts(misfit=kind, dt=dt, tlag_max=0.04, penalty=L.OWL_PENALTY_LINEAR)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("nt", [300, 1201])
def test_adjoint_source_matches_oracle(kind, nt):
    import torch
    gp, syn, obs, w = _gathers(nt)
    dt = 1e-3
    ref_adj, ref_tm, ref_gm = M.adjoint_source(kind, gp, syn, obs, w, dt=dt, tlag_max=0.04)
    tol = 1e-6 if kind in (L.OWL_MISFIT_WAVEFORM, L.OWL_MISFIT_CORR) else 1e-4
    adj, tm, gm = adjoint_source(_mopts(kind, dt), gp, syn, obs, w)
    assert np.all(tm[[1, 6, 8]] == 0) and np.all(adj[[1, 6, 8]] == 0)
    assert rel(adj, ref_adj) < tol, rel(adj, ref_adj)
    assert rel(tm, ref_tm) < tol, (tm, ref_tm)
    assert np.allclose(gm, [tm[:5].sum(), tm[5:].sum()], rtol=1e-12)
    dadj, dtm, dgm = adjoint_source(_mopts(kind, dt), gp, torch.from_numpy(syn).cuda(), torch.from_numpy(obs).cuda(),
                                    torch.from_numpy(w).cuda())
    assert np.array_equal(dadj.cpu().numpy(), adj)
    assert np.array_equal(dtm.cpu().numpy(), tm)


def test_adjoint_source_penalties_and_threshold():
    gp, syn, obs, w = _gathers(500)
    for pen in (L.OWL_PENALTY_POWER, L.OWL_PENALTY_GAUSSIAN, L.OWL_PENALTY_EXP):
        mo = MisfitOpts(misfit=L.OWL_MISFIT_ADAPTIVE, dt=2e-3, tlag_max=0.1, penalty=pen, penalty_power=2.0,
                        deconv_eps=0.05)
        adj, tm, _ = adjoint_source(mo, gp, syn, obs, w)
        ref_adj, ref_tm, _ = M.adjoint_source(M.ADAPTIVE, gp, syn, obs, w, dt=2e-3, tlag_max=0.1, penalty_method=pen,
                                              penalty_power=2.0, deconv_eps=0.05)
        assert rel(adj, ref_adj) < 1e-4 and rel(tm, ref_tm) < 1e-4, pen
    # threshold off: the tiny trace is kept, the zero trace is not
    _, tm, _ = adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_WAVEFORM, discard_threshold=-1.0), gp, syn, obs, w)
    assert tm[6] > 0 and tm[8] == 0 and tm[1] == 0


def test_adjoint_source_rejects_long_traces():
    gp, syn, obs, w = _gathers(64)
    long = np.zeros((9, 9000), dtype=np.float32)
    with pytest.raises(L.OwlError):
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_ENVELOPE), gp, long, long, w)


@pytest.mark.parametrize("kind", KINDS)
def test_gradient_misfit_matches_oracle(kind):
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 240
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp, rho, ps, "f64").astype(np.float32)
    vp0 = (vp * np.float32(1.03)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    mo = MisfitOpts(misfit=kind, tlag_max=0.03)
    seis = np.zeros(s.seis_size(ps), dtype=np.float32)
    mf, g = s.gradient_misfit(ps, obs, mo, RunOpts(checkpoint_interval=30), seis_out=seis)
    # the oracle's adjoint source from the oracle's FP64 synthetics, then its exact-adjoint gradient
    syn64 = oracle.ac2d_forward(d, vp0, rho, ps, "f64")
    gp = s.gather_ptr(ps)
    live = np.concatenate([[r.weight != 0 for r in sh.receivers] for sh in ps.shots]).astype(np.float64)
    adj, tm, gm = M.adjoint_source(kind, gp, syn64.reshape(-1, nt), obs.reshape(-1, nt), live, dt=dt, tlag_max=0.03)
    _, g_ref, _ = oracle.ac2d_gradient(d, vp0, rho, ps, adj.ravel().astype(np.float32), adj_kind=1, k=30,
                                       precision="f64")
    tol = 1e-4 if kind in (L.OWL_MISFIT_WAVEFORM, L.OWL_MISFIT_CORR) else 2e-4
    assert rel(g, g_ref) < tol, rel(g, g_ref)
    assert rel(mf, gm) < tol
    if kind == L.OWL_MISFIT_WAVEFORM:
        mf2, g2 = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, RunOpts(checkpoint_interval=30))
        assert rel(g, g2) < 1e-6 and rel(mf, mf2) < 1e-6


@pytest.mark.parametrize("kind", [L.OWL_MISFIT_WAVEFORM, L.OWL_MISFIT_ENVELOPE, L.OWL_MISFIT_ADAPTIVE])
def test_adjoint_source_resampled_to_adj_nt(kind):
    """adj_nt: the misfit on the kept traces resampled (cubic) to adj_nt samples
    over the same span, the adjoint resampled back"""
    gp, syn, obs, w = _gathers(400)
    for nn in (300, 613):
        mo = MisfitOpts(misfit=kind, dt=1e-3, tlag_max=0.04, adj_nt=nn)
        adj, tm, gm = adjoint_source(mo, gp, syn, obs, w)
        ref_adj, ref_tm, ref_gm = M.adjoint_source(kind, gp, syn, obs, w, dt=1e-3, tlag_max=0.04, adj_nt=nn)
        assert np.all(tm[[1, 6, 8]] == 0)
        assert rel(adj, ref_adj) < 1e-4, (nn, rel(adj, ref_adj))
        assert rel(tm, ref_tm) < 1e-4, (nn, tm, ref_tm)
    with pytest.raises(L.OwlError):  # DTW's shift computation needs 3 .. 16384 samples
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_DTW, dt=1e-3, tlag_max=0.02, adj_nt=20000), gp, syn, obs, w)
