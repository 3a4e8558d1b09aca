"""GPU dynamic-time-warping misfit (OWL_MISFIT_DTW) against the oracle's
restatement (oracle/oracle_dtw.py).

* time shifts (owl_dtw_time_shifts): the GPU's dynamic program uses the
  oracle's double-precision operations rounded the same way, so the shifts
  agree to single-precision rounding (1e-6 s) on every trace;
* adjoint sources and trace misfits of the 'phase', 'amp' and 'phase+amp'
  forms, with and without neighbouring traces in the distance, host and
  device buffers, gathers with a weight-0 trace, a trace below the discard
  threshold and a zero trace: 1e-4 relative L2;
* the gradient of the DTW misfit through owl_ssg_gradient_misfit equals the
  FP64 exact-adjoint oracle gradient driven by the oracle's DTW adjoint source
  of the same synthetics (2e-4);
* dtw-vector (OWL_MISFIT_DTW_VECTOR): two shots of two components, a dropped
  component of a kept receiver and a dropped receiver: shifts to 1e-6 s, one
  per receiver on both component rows, adjoints and misfits 1e-4; gather
  layouts that are not groups of equal component gathers are errors;
* adj_nt: shifts and quality weights computed on the normalised traces
  resampled to adj_nt samples and brought back by pchip, scalar and vector:
  shifts to 1e-6 s, adjoints 1e-4; the gradient driver with data sampled off
  the time axis (adj_nt's default, the time axis' nt) against the FP64 oracle;
* the documented size limits are errors.
"""
import numpy as np
import pytest

import oracle
from oracle import oracle_dtw as D
from owl_b200 import _lib as L
from owl_b200.solver import MisfitOpts, RunOpts, adjoint_source, dtw_time_shifts

from cases import desc, prepare, random_model, rel, small_shots
from test_gpu_ac2d import make_solver
from test_gpu_misfits import _gathers

pytestmark = pytest.mark.gpu

DT, TLAG = 1e-3, 0.02


def _mo(form=L.OWL_DTW_PHASE, trc=0, **kw):
    return MisfitOpts(misfit=L.OWL_MISFIT_DTW, dt=DT, tlag_max=TLAG, dtw_form=form, dtw_trc=trc, **kw)


@pytest.mark.parametrize("form,trc", [(L.OWL_DTW_PHASE, 0), (L.OWL_DTW_AMP, 0), (L.OWL_DTW_PHASE_AMP, 0),
                                      (L.OWL_DTW_PHASE, 1)])
def test_dtw_matches_oracle(form, trc):
    import torch
    gp, syn, obs, w = _gathers(300)
    kw = dict(form=form, trc=trc, amp_weight=0.5 if form == L.OWL_DTW_PHASE_AMP else 1.0)
    ref_adj, ref_tm, ref_gm, ref_tau = D.adjoint_source(gp, syn, obs, w, dt=DT, tlag_max=TLAG, **kw)
    mo = _mo(form, trc, dtw_amp_weight=kw["amp_weight"])
    tau = dtw_time_shifts(mo, gp, syn, obs, w)
    assert np.max(np.abs(tau - ref_tau)) <= 1e-6, np.max(np.abs(tau - ref_tau))
    assert np.all(tau[[1, 6, 8]] == 0)
    adj, tm, gm = adjoint_source(mo, gp, syn, obs, w)
    assert np.all(tm[[1, 6, 8]] == 0) and np.all(adj[[1, 6, 8]] == 0)
    assert rel(adj, ref_adj) < 1e-4, rel(adj, ref_adj)
    assert rel(tm, ref_tm) < 1e-4, (tm, ref_tm)
    assert np.allclose(gm, [tm[:5].sum(), tm[5:].sum()], rtol=1e-12)
    # device buffers give the same bytes
    dadj, dtm, _ = adjoint_source(mo, gp, torch.from_numpy(syn).cuda(), torch.from_numpy(obs).cuda(),
                                  torch.from_numpy(w).cuda())
    assert np.array_equal(dadj.cpu().numpy(), adj)
    assert np.array_equal(dtm.cpu().numpy(), tm)
    dtau = dtw_time_shifts(mo, gp, torch.from_numpy(syn).cuda(), torch.from_numpy(obs).cuda(),
                           torch.from_numpy(w).cuda())
    assert np.array_equal(dtau.cpu().numpy(), tau)


def test_dtw_gradient_matches_oracle():
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 240
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp, rho, ps, "f64").astype(np.float32)
    vp0 = (vp * np.float32(1.03)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    mo = MisfitOpts(misfit=L.OWL_MISFIT_DTW, dt=dt, tlag_max=0.02)
    seis = np.zeros(s.seis_size(ps), dtype=np.float32)
    mf, g = s.gradient_misfit(ps, obs, mo, RunOpts(checkpoint_interval=30), seis_out=seis)
    # the oracle's DTW adjoint source of the GPU's own synthetics, then its exact-adjoint gradient
    gp = s.gather_ptr(ps)
    live = np.concatenate([[r.weight != 0 for r in sh.receivers] for sh in ps.shots]).astype(np.float64)
    adj, tm, gm, _ = D.adjoint_source(gp, seis.reshape(-1, nt), obs.reshape(-1, nt), live, dt=dt, tlag_max=0.02)
    _, g_ref, _ = oracle.ac2d_gradient(d, vp0, rho, ps, adj.ravel().astype(np.float32), adj_kind=1, k=30,
                                       precision="f64")
    assert rel(g, g_ref) < 2e-4, rel(g, g_ref)
    assert rel(mf, gm) < 1e-4
    assert np.all(mf > 0)


def test_dtw_limits():
    gp, syn, obs, w = _gathers(300)
    with pytest.raises(L.OwlError):  # 2 tlag_max / dt + 1 > 4095 candidates
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_DTW, dt=1e-5, tlag_max=0.03), gp, syn, obs, w)
    with pytest.raises(L.OwlError):  # no sample interval
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_DTW, tlag_max=0.02), gp, syn, obs, w)
    long = np.zeros((9, 16385), dtype=np.float32)
    with pytest.raises(L.OwlError):
        adjoint_source(_mo(), gp, long, long, w)
    with pytest.raises(L.OwlError):  # time shifts of another misfit
        dtw_time_shifts(MisfitOpts(misfit=L.OWL_MISFIT_WAVEFORM, dt=DT), gp, syn, obs, w)


def _vector_gathers(nt=300, seed=7):
    """two shots x two components, four receivers each: component c of
    receiver i shifted by (2 + i) samples; shot 0's component 1 of receiver 2
    has weight 0 (a dropped component of a kept receiver) and shot 1's
    receiver 3 has weight 0 on both components (a dropped receiver)"""
    rng = np.random.default_rng(seed)
    t = np.arange(nt)
    syn, obs = [], []
    for s in range(2):
        for c in range(2):
            for i in range(4):
                ctr = nt * (0.3 + 0.08 * i + 0.05 * s)
                f = 0.09 + 0.01 * c
                sh = 2.0 + i
                pol = 1.0 if c == 0 else -0.6
                obs.append(pol * np.exp(-((t - ctr) / (0.04 * nt)) ** 2) * np.cos(f * (t - ctr))
                           + 0.02 * rng.standard_normal(nt))
                syn.append(0.9 * pol * np.exp(-((t - ctr - sh) / (0.04 * nt)) ** 2) * np.cos(f * (t - ctr - sh))
                           + 0.02 * rng.standard_normal(nt))
    w = np.ones(16, dtype=np.float32)
    w[4 + 2] = 0.0          # shot 0, component 1, receiver 2
    w[8 + 3] = w[12 + 3] = 0.0  # shot 1, receiver 3, both components
    return [0, 4, 8, 12, 16], np.array(syn, dtype=np.float32), np.array(obs, dtype=np.float32), w


@pytest.mark.parametrize("form", [L.OWL_DTW_PHASE, L.OWL_DTW_AMP, L.OWL_DTW_PHASE_AMP])
def test_dtw_vector_matches_oracle(form):
    gp, syn, obs, w = _vector_gathers()
    kw = dict(form=form, amp_weight=0.5 if form == L.OWL_DTW_PHASE_AMP else 1.0)
    ref_adj, ref_tm, ref_gm, ref_tau = D.adjoint_source_vector(gp, syn, obs, 2, w, dt=DT, tlag_max=TLAG, **kw)
    mo = MisfitOpts(misfit=L.OWL_MISFIT_DTW_VECTOR, dt=DT, tlag_max=TLAG, dtw_form=form, ncomp=2,
                    dtw_amp_weight=kw["amp_weight"])
    tau = dtw_time_shifts(mo, gp, syn, obs, w)
    assert np.max(np.abs(tau - ref_tau)) <= 1e-6, np.max(np.abs(tau - ref_tau))
    # one shift per receiver, on both component rows; none for the dropped receiver
    assert np.array_equal(tau[0:4], tau[4:8]) and np.array_equal(tau[8:12], tau[12:16])
    assert np.all(tau[[11, 15]] == 0) and np.any(tau[6] != 0)
    adj, tm, gm = adjoint_source(mo, gp, syn, obs, w)
    assert np.all(adj[[6, 11, 15]] == 0)
    assert rel(adj, ref_adj) < 1e-4, rel(adj, ref_adj)
    assert rel(tm, ref_tm) < 1e-4, (tm, ref_tm)
    assert np.allclose(gm, ref_gm, rtol=1e-4)


def test_dtw_vector_layout_checks():
    gp, syn, obs, w = _vector_gathers()
    with pytest.raises(L.OwlError):  # 4 gathers are not groups of 3
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_DTW_VECTOR, dt=DT, tlag_max=TLAG, ncomp=3), gp, syn, obs, w)
    with pytest.raises(L.OwlError):  # component gathers of unequal length
        adjoint_source(MisfitOpts(misfit=L.OWL_MISFIT_DTW_VECTOR, dt=DT, tlag_max=TLAG, ncomp=2),
                       [0, 4, 7, 12, 16], syn, obs, w)


@pytest.mark.parametrize("form,nn", [(L.OWL_DTW_PHASE, 451), (L.OWL_DTW_PHASE_AMP, 200), (L.OWL_DTW_AMP, 451)])
def test_dtw_adj_nt_matches_oracle(form, nn):
    """adj_nt: the shifts and weights computed on the normalised traces
    resampled to adj_nt samples (float64 cubic, single-precision result, as the
    oracle) and interpolated back by pchip; shifts to 1e-6 s."""
    gp, syn, obs, w = _gathers(300)
    kw = dict(form=form, amp_weight=0.5 if form == L.OWL_DTW_PHASE_AMP else 1.0, adj_nt=nn)
    ref_adj, ref_tm, ref_gm, ref_tau = D.adjoint_source(gp, syn, obs, w, dt=DT, tlag_max=TLAG, **kw)
    mo = _mo(form, dtw_amp_weight=kw["amp_weight"], adj_nt=nn)
    tau = dtw_time_shifts(mo, gp, syn, obs, w)
    assert tau.shape == syn.shape
    assert np.max(np.abs(tau - ref_tau)) <= 1e-6, np.max(np.abs(tau - ref_tau))
    adj, tm, gm = adjoint_source(mo, gp, syn, obs, w)
    assert np.all(tm[[1, 6, 8]] == 0) and np.all(adj[[1, 6, 8]] == 0)
    assert rel(adj, ref_adj) < 1e-4, rel(adj, ref_adj)
    assert rel(tm, ref_tm) < 1e-4, (tm, ref_tm)
    # adj_nt equal to the trace length is no resampling
    t0 = dtw_time_shifts(_mo(form, dtw_amp_weight=kw["amp_weight"]), gp, syn, obs, w)
    t1 = dtw_time_shifts(_mo(form, dtw_amp_weight=kw["amp_weight"], adj_nt=300), gp, syn, obs, w)
    assert np.array_equal(t0, t1)


def test_dtw_vector_adj_nt_matches_oracle():
    gp, syn, obs, w = _vector_gathers()
    ref_adj, ref_tm, ref_gm, ref_tau = D.adjoint_source_vector(gp, syn, obs, 2, w, dt=DT, tlag_max=TLAG,
                                                               adj_nt=401)
    mo = MisfitOpts(misfit=L.OWL_MISFIT_DTW_VECTOR, dt=DT, tlag_max=TLAG, ncomp=2, adj_nt=401)
    tau = dtw_time_shifts(mo, gp, syn, obs, w)
    assert np.max(np.abs(tau - ref_tau)) <= 1e-6, np.max(np.abs(tau - ref_tau))
    assert np.array_equal(tau[0:4], tau[4:8]) and np.array_equal(tau[8:12], tau[12:16])
    adj, tm, gm = adjoint_source(mo, gp, syn, obs, w)
    assert rel(adj, ref_adj) < 1e-4, rel(adj, ref_adj)
    assert np.allclose(gm, ref_gm, rtol=1e-4)


def test_dtw_gradient_at_data_sampling():
    """Data sampled at 2.5 ms on a 1 ms time axis: the gradient driver's DTW
    shifts are computed at the time axis' nt samples (adj_nt's default), the
    adjoint at the data sampling, resampled back before injection."""
    import oracle.oracle_resample as R
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 241
    ddt = 2.5e-3
    dnt = int(round((nt - 1) * dt / ddt)) + 1
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = R.resample_rows(oracle.ac2d_forward(d, vp, rho, ps, "f64").reshape(-1, nt), dt, ddt, dnt)
    obs = obs.astype(np.float32)
    vp0 = (vp * np.float32(1.03)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    s.set_data_sampling(dnt, ddt)
    seis = np.zeros(s.seis_size(ps), dtype=np.float32)
    mf, g = s.gradient_misfit(ps, obs.ravel(), MisfitOpts(misfit=L.OWL_MISFIT_DTW, tlag_max=0.02),
                              RunOpts(checkpoint_interval=30), seis_out=seis)
    # the oracle's DTW adjoint source (adj_nt = nt) of the GPU's own resampled synthetics
    gp = s.gather_ptr(ps)
    live = np.concatenate([[r.weight != 0 for r in sh.receivers] for sh in ps.shots]).astype(np.float64)
    syn_d = seis.reshape(-1, dnt)
    adj_d, tm, gm, _ = D.adjoint_source(gp, syn_d, obs, live, dt=ddt, tlag_max=0.02, adj_nt=nt)
    assert rel(mf, gm) < 1e-4, (mf, gm)
    adj_t = R.resample_rows(adj_d, ddt, dt, nt).astype(np.float32)
    _, g_ref, _ = oracle.ac2d_gradient(d, vp0, rho, ps, adj_t.ravel(), adj_kind=1, k=30, precision="f64")
    assert rel(g, g_ref) < 2e-4, rel(g, g_ref)
