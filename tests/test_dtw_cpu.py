"""The DTW restatement of the oracle (oracle/oracle_dtw.py), on the CPU.

* the vectorised dynamic program equals a literal transcription of the
  reference's loops (solve_gdtw, module_inversion_adjoint_source.f90:153-194:
  rows, then candidates j, then k, strict improvement) on small random cases;
* planted shifts of band-limited wavelets are recovered (obs(t + tau) = syn(t));
* identical traces give a sub-sample shift and a negligible misfit; dropped
  traces are zero.
"""
import math

import numpy as np
import pytest

from oracle import oracle_dtw as D


def _loops_dp(tg, nu, dt, rinst):
    """solve_gdtw's dynamic program written as the reference's nested loops."""
    n, m = tg.shape
    f = np.full((n, m), D.HUGE)
    p = np.zeros((n, m), dtype=np.int64)
    jc = (m - 1) // 2
    f[0, jc] = nu[0, jc]
    for i in range(n - 1):
        for j in range(m):
            for k in range(m):
                slope = (tg[i + 1, k] - tg[i, j]) / dt
                if slope < D.S_MIN - D.DELTA or slope > D.S_MAX + D.DELTA:
                    continue
                pc = f[i, j] + dt * (rinst * (slope * slope) + nu[i + 1, k])
                if pc < f[i + 1, k]:
                    f[i + 1, k] = pc
                    p[i + 1, k] = j
    return f, p


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_vectorised_dp_matches_reference_loops(seed):
    rng = np.random.default_rng(seed)
    n, m = 14, 9
    t = np.arange(n) / (n - 1.0)
    dt = 1.0 / (n - 1.0)
    # a random band inside the first iteration's bounds
    u0 = np.minimum(np.minimum(D.S_MAX * t, 1.0 - D.S_MIN * (1.0 - t)), 1.0)
    l0 = np.maximum(np.maximum(D.S_MIN * t, 1.0 - D.S_MAX * (1.0 - t)), 0.0)
    mid = l0 + (u0 - l0) * rng.uniform(0.3, 0.7, n)
    half = (u0 - l0) * rng.uniform(0.05, 0.3, n)
    l = np.maximum(mid - half, l0)
    u = np.minimum(mid + half, u0)
    lin = np.arange(m) / (m - 1.0)
    tg = l[:, None] + (u - l)[:, None] * lin[None, :]
    nu = rng.uniform(0.0, 1.0, (n, m))
    f_ref, p_ref = _loops_dp(tg, nu, dt, 0.1)
    # the oracle's row update, applied to the same band
    f = np.full((n, m), D.HUGE)
    p = np.zeros((n, m), dtype=np.int64)
    jc = (m - 1) // 2
    f[0, jc] = nu[0, jc]
    for i in range(n - 1):
        slope = (tg[i + 1][None, :] - tg[i][:, None]) / dt
        ok = ~((slope < D.S_MIN - D.DELTA) | (slope > D.S_MAX + D.DELTA)) & (f[i] < D.HUGE)[:, None]
        pc = np.where(ok, f[i][:, None] + dt * (0.1 * (slope * slope) + nu[i + 1][None, :]), np.inf)
        jb = np.argmin(pc, axis=0)
        vb = pc[jb, np.arange(m)]
        upd = vb < D.HUGE
        f[i + 1, upd] = vb[upd]
        p[i + 1, upd] = jb[upd]
    assert np.array_equal(f, f_ref)
    assert np.array_equal(p[f < D.HUGE], p_ref[f < D.HUGE])


def _ricker(t, c, f=15.0):
    a = (math.pi * f * (t - c)) ** 2
    return (1 - 2 * a) * np.exp(-a)


def test_planted_shifts_recovered():
    n, dd = 300, 2e-3
    t = np.arange(n) * dd
    centres = [0.25, 0.30, 0.28]
    shifts = [0.012, -0.010, 0.0]
    syn = np.stack([_ricker(t, c) for c in centres]).astype(np.float32)
    obs = np.stack([_ricker(t, c + s) for c, s in zip(centres, shifts)]).astype(np.float32)
    adj, tm, tau, q = D.dtw_gather(syn, obs, np.ones(3, bool), dd, 0.04)
    for i, s in enumerate(shifts):
        j = int(np.argmax(np.abs(syn[i])))
        assert abs(tau[i, j] - s) <= 1.5 * dd, (i, tau[i, j], s)
    # identical traces: a shift of a small fraction of a sample on the event
    # (where the traces are quiet the path is held only by the shift penalty
    # and drifts by less than a sample) and a negligible misfit
    big = np.abs(syn[2]) > 0.1 * np.abs(syn[2]).max()
    assert np.all(np.abs(tau[2][big]) < 0.05 * dd) and np.all(np.abs(tau[2]) < dd)
    assert tm[2] < 1e-3 * min(tm[0], tm[1])
    assert np.all((q >= 0) & (q <= 1))


def test_forms_and_dropped_traces():
    n, dd = 200, 2e-3
    t = np.arange(n) * dd
    syn = np.stack([_ricker(t, 0.20), _ricker(t, 0.22), _ricker(t, 0.18)]).astype(np.float32)
    obs = np.stack([_ricker(t, 0.21), _ricker(t, 0.215), _ricker(t, 0.18)]).astype(np.float32)
    gp = [0, 3]
    w = np.array([1.0, 0.0, 1.0], dtype=np.float32)
    a_p, tm_p, gm_p, tau = D.adjoint_source(gp, syn, obs, w, dt=dd, tlag_max=0.03)
    a_a, tm_a, _, _ = D.adjoint_source(gp, syn, obs, w, dt=dd, tlag_max=0.03, form=D.AMP)
    a_b, tm_b, _, _ = D.adjoint_source(gp, syn, obs, w, dt=dd, tlag_max=0.03, form=D.PHASE_AMP, amp_weight=0.5)
    for a, tm in ((a_p, tm_p), (a_a, tm_a), (a_b, tm_b)):
        assert np.all(a[1] == 0) and tm[1] == 0
    assert np.all(tau[1] == 0)
    assert gm_p[0] == pytest.approx(tm_p.sum())
    # 'phase+amp' misfit is the phase misfit times (1 + amp_weight)
    assert tm_b[0] == pytest.approx(tm_p[0] * 1.5, rel=1e-12)
    # 'amp' misfit: the warped residual (here the shift is captured, so it is small)
    assert tm_a[0] < float(np.sum((syn[0].astype(np.float64) - obs[0]) ** 2))


def test_lag_count_is_odd():
    for tl, dd in ((0.04, 2e-3), (0.05, 2e-3), (0.1, 1e-3), (0.0105, 1e-3)):
        m = D.lag_count(tl, dd)
        assert m % 2 == 1 and m >= 3


def test_pchip_matches_scipy():
    """The pchip restatement is the published monotone cubic (Fritsch and
    Carlson): it agrees with SciPy's independent implementation to single
    precision, keeps monotone rows monotone and reproduces linear rows."""
    from scipy.interpolate import PchipInterpolator
    rng = np.random.default_rng(5)
    for nn, nout in ((30, 71), (57, 20), (3, 11), (2, 9)):
        x = rng.standard_normal((4, nn)).astype(np.float32)
        x[1] = np.cumsum(np.abs(x[1]))
        x[2, nn // 2:] = x[2, nn // 2]  # a flat stretch
        dout = (nn - 1) / (nout - 1)
        got = D.pchip_rows(x, 1.0, dout, nout)
        pos = np.minimum(np.arange(nout) * dout, nn - 1)
        for r in range(4):
            ref = PchipInterpolator(np.arange(nn), x[r].astype(np.float64))(pos)
            assert np.max(np.abs(got[r] - ref)) <= 1e-6 * max(1.0, np.abs(ref).max()), (nn, r)
        assert np.all(np.diff(got[1]) >= 0)
    lin = (np.arange(12) * 0.25).astype(np.float32)
    assert np.allclose(D.pchip_rows(lin, 2.0, 0.5, 45), np.arange(45) * 0.0625, atol=1e-6)


def test_adj_nt_shift_computation():
    """adj_nt: shifts computed on traces resampled to adj_nt samples and brought
    back by pchip recover the planted shifts at the trace sampling; adj_nt equal
    to the trace length is no resampling."""
    n, dd = 300, 2e-3
    t = np.arange(n) * dd
    centres, shifts = [0.25, 0.30], [0.012, -0.010]
    syn = np.stack([_ricker(t, c) for c in centres]).astype(np.float32)
    obs = np.stack([_ricker(t, c + s) for c, s in zip(centres, shifts)]).astype(np.float32)
    live = np.ones(2, bool)
    base = D.dtw_gather(syn, obs, live, dd, 0.04)
    same = D.dtw_gather(syn, obs, live, dd, 0.04, adj_nt=n)
    for a, b in zip(base, same):
        assert np.array_equal(a, b)
    for nn in (451, 200):
        adj, tm, tau, q = D.dtw_gather(syn, obs, live, dd, 0.04, adj_nt=nn)
        assert tau.shape == (2, n) and q.shape == (2, n) and adj.shape == (2, n)
        ddn = (n - 1) * dd / (nn - 1)
        for i, s in enumerate(shifts):
            j = int(np.argmax(np.abs(syn[i])))
            assert abs(tau[i, j] - s) <= 1.5 * ddn, (nn, i, tau[i, j], s)
        assert np.all((q >= -1e-6) & (q <= 1 + 1e-6))
