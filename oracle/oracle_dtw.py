"""Oracle (test infrastructure only): restatement of the reference's dynamic-time-
warping misfit and adjoint source.

Follows src/inverse/module_inversion_adjoint_source.f90:
  solve_gdtw           :73-234  generalized DTW (Deriso & Boyd) with iterative
                                refinement of the search band, double precision
  compute_adjsrc_dtw   :715-980 per-gather normalisation, GDTW time shifts,
                                windowed-correlation quality weights, adjoint
                                source of the 'phase', 'amp' and 'phase+amp' forms
  compute_adjoint_source :1224-1236 ('dtw': one call per gather and component;
                         'dtw-vector': one call on all components of a shot)
with the defaults of src/lib/module_parameters.f90:270-280, 559-569
(dtw_niter 5, dtw_rinst 0.1, dtw_rcuml 1, dtw_epsabs 1e-2, dtw_epsrel 1e-3,
dtw_loss 'l0.5', dtw_form 'phase', dtw_amp_weight 1, dtw_trc 0, no smoothing of
the shifts across traces). With adj_nt (:744-750, :765-771, :907-911) the
normalised traces are resampled to adj_nt samples over the same span (cubic,
single precision), the shifts and quality weights are computed at that
sampling and interpolated back to the trace length with 'pchip'; the adjoint
is taken on the traces as given.

The dynamic program is evaluated in the order of the reference's loops (for each
row, candidates j ascending, strict improvement), in float64 without fused
multiply-adds, so that the GPU path, which uses the same operations rounded the
same way, takes the same discrete decisions.

FLIT (github.com/lanl/flit, no version pinned by the reference) supplies
ginterp, median_filt, gauss_filt, rescale, deriv, norm2, linspace and
return_normal; none is vendored and no reference test pins them -- parity
unpinned. They are restated as:
  ginterp linear   on the sample grid, interval located by position, clamped to
                   the end values (GDTW) or zero outside the grid (warping);
  ginterp cubic    Keys cubic convolution (a = -1/2), indices clamped to the
                   trace, zero outside it, 1e-4 snap to a node (the same
                   restatement as the trace resampling);
  median_filt(q,3) median of the 7-sample window centred on each sample,
                   truncated at the ends (mean of the two middle values for an
                   even count);
  gauss_filt(q,3)  Gaussian of standard deviation 3 samples truncated at 9,
                   normalised, end samples replicated;
  deriv(x)         centred difference inside, one-sided at the ends;
  rescale(q,[0,1]) (q - min) / (max - min);  return_normal: NaN / Inf -> 0;
  interp_to cubic  the trace resampling restatement (oracle_resample), evaluated
                   in float64 and rounded to single precision;
  interp_to pchip  monotone piecewise cubic Hermite interpolation (Fritsch and
                   Carlson 1980) on the unit sample grid: interior slopes the
                   harmonic mean of the neighbouring secants (zero where they
                   differ in sign or one is zero), end slopes the three-point
                   formula (3 s0 - s1) / 2 limited to keep the secant's sign and
                   at most 3 |s0|; output sample i at x = i dout / din (1e-4
                   snap to a node), clamped to the grid; float64, rounded to
                   single precision.
"""
from __future__ import annotations

import math

import numpy as np

PHASE, AMP, PHASE_AMP = 0, 1, 2
F32_TINY = float(np.finfo(np.float32).tiny)
HUGE = float(np.finfo(np.float64).max)
S_MIN, S_MAX, S_BETA, ETA, DELTA = 1.0e-8, 1.0e2, 0.0, 0.15, 1.0e-10

f32 = np.float32


def nint(x: float) -> int:
    """Fortran nint: round half away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def lag_count(tlag_max: float, dd: float) -> int:
    """m = nint(2 tlag_max / dd) + 1, made odd (:795, :92-96); single precision."""
    m = nint(float(f32(f32(2.0) * f32(tlag_max)) / f32(dd))) + 1
    return m + 1 if m % 2 == 0 else m


def _lin_interp_clamped(t, x, tq):
    """linear interpolation of x (on the uniform grid t = i / (n-1)) at tq,
    clamped to the end values; no fused multiply-adds."""
    n = t.size
    out = np.empty(tq.shape)
    for idx, q in np.ndenumerate(tq):
        if q <= t[0]:
            out[idx] = x[0]
            continue
        if q >= t[n - 1]:
            out[idx] = x[n - 1]
            continue
        i0 = min(int(math.floor(q * (n - 1))), n - 2)
        while i0 > 0 and t[i0] > q:
            i0 -= 1
        while i0 < n - 2 and t[i0 + 1] <= q:
            i0 += 1
        w = (q - t[i0]) / (t[i0 + 1] - t[i0])
        out[idx] = x[i0] * (1.0 - w) + x[i0 + 1] * w
    return out


def _powabs(d, p):
    a = np.abs(d)
    if p == 0.5:
        return np.sqrt(a)
    if p == 1.0:
        return a
    if p == 2.0:
        return a * a
    return a ** p


def gdtw(x, y, m, niter=5, rinst=0.1, rcuml=1.0, epsabs=1.0e-2, epsrel=1.0e-3, power=0.5):
    """solve_gdtw (:73-234): x, y (n, K) float64 columns (obs, syn). Returns the
    shift in samples, tau such that x(t + tau) ~ y(t), and the final cost."""
    x = np.asarray(x, dtype=np.float64).reshape(x.shape[0], -1)
    y = np.asarray(y, dtype=np.float64).reshape(y.shape[0], -1)
    n, K = x.shape
    t = np.arange(n, dtype=np.float64) / float(n - 1)
    dt = 1.0 / (n - 1.0)
    lin = np.arange(m, dtype=np.float64) / float(m - 1)
    u0 = np.minimum(np.minimum(S_BETA + S_MAX * t, S_BETA + 1.0 - S_MIN * (1.0 - t)), 1.0)
    l0 = np.maximum(np.maximum(S_MIN * t, -S_BETA + 1.0 - S_MAX * (1.0 - t)), 0.0)
    u, l = u0.copy(), l0.copy()
    tau = np.zeros(n)
    cost_prev = F32_TINY
    jc = (m - 1) // 2
    cost = 0.0
    for it in range(niter):
        if it > 0:
            rng = ETA * (u - l) / 2.0
            u = np.minimum(tau + rng, u0)
            l = np.maximum(tau - rng, l0)
        tg = l[:, None] + (u - l)[:, None] * lin[None, :]
        dist = np.zeros((n, m))
        for k in range(K):
            v = _lin_interp_clamped(t, x[:, k], tg)
            dist = dist + _powabs(v - y[:, k][:, None], power)
        d = tg - t[:, None]
        nu = dist + rcuml * (d * d)
        f = np.full((n, m), HUGE)
        p = np.zeros((n, m), dtype=np.int64)
        f[0, jc] = nu[0, jc]
        for i in range(n - 1):
            slope = (tg[i + 1][None, :] - tg[i][:, None]) / dt
            ok = ~((slope < S_MIN - DELTA) | (slope > S_MAX + DELTA)) & (f[i] < HUGE)[:, None]
            pc = f[i][:, None] + dt * (rinst * (slope * slope) + nu[i + 1][None, :])
            pc = np.where(ok, pc, np.inf)
            jb = np.argmin(pc, axis=0)
            vb = pc[jb, np.arange(m)]
            upd = vb < HUGE
            f[i + 1, upd] = vb[upd]
            p[i + 1, upd] = jb[upd]
        cost = f[n - 1, jc]
        j = jc
        for i in range(n - 1, -1, -1):
            tau[i] = tg[i, j]
            j = p[i, j]
        if abs(cost - cost_prev) <= epsabs + epsrel * cost_prev:
            break
        cost_prev = cost
    lin32 = (np.arange(n, dtype=np.float32) / f32(n - 1)).astype(np.float64)
    return (tau - lin32) * (n - 1), cost


def _lin_interp_zero(tgrid, x, tq):
    """single-precision linear interpolation on the grid tgrid, zero outside."""
    n = tgrid.size
    out = np.zeros(tq.size, dtype=f32)
    for i, q in enumerate(tq):
        if q < tgrid[0] or q > tgrid[n - 1]:
            continue
        i0 = min(int(np.searchsorted(tgrid, q, side="right")) - 1, n - 2)
        i0 = max(i0, 0)
        w = f32((q - tgrid[i0]) / (tgrid[i0 + 1] - tgrid[i0]))
        out[i] = f32(x[i0] * (f32(1.0) - w) + x[i0 + 1] * w)
    return out


def keys_weights(u):
    u2, u3 = u * u, u * u * u
    return (0.5 * (-u3 + 2 * u2 - u), 0.5 * (3 * u3 - 5 * u2 + 2), 0.5 * (-3 * u3 + 4 * u2 + u), 0.5 * (u3 - u2))


def _cubic_warp(x, pos):
    """Keys cubic value of x at fractional sample positions pos (zero outside)."""
    n = x.size
    out = np.zeros(pos.size)
    for i, p in enumerate(pos):
        if abs(p - round(p)) <= 1e-4:
            p = float(round(p))
        if p < 0 or p > n - 1:
            continue
        j0 = int(math.floor(p))
        w = keys_weights(p - j0)
        idx = (max(j0 - 1, 0), j0, min(j0 + 1, n - 1), min(j0 + 2, n - 1))
        out[i] = sum(wk * x[jk] for wk, jk in zip(w, idx))
    return out


def median7(q):
    n = q.size
    out = np.empty_like(q)
    for i in range(n):
        w = np.sort(q[max(0, i - 3):min(n, i + 4)])
        c = w.size
        out[i] = w[c // 2] if c % 2 else f32(0.5) * (w[c // 2 - 1] + w[c // 2])
    return out


def gauss3(q):
    sg = 3.0
    rad = int(math.ceil(3.0 * sg))
    k = np.arange(-rad, rad + 1)
    w = np.exp(-0.5 * k * k / (sg * sg))
    w /= w.sum()
    n = q.size
    out = np.zeros(n)
    for kk, wk in zip(k, w):
        out += wk * q[np.clip(np.arange(n) + kk, 0, n - 1)]
    return out


def deriv(x):
    d = np.empty_like(x)
    d[1:-1] = (x[2:] - x[:-2]) * 0.5
    d[0] = x[1] - x[0]
    d[-1] = x[-1] - x[-2]
    return d


def resample_f32(rows, din, dout, nout):
    """interp_to(x, nout, method='cubic') of single-precision rows (:767-768)."""
    from .oracle_resample import resample_rows
    shp = np.shape(rows)
    out = resample_rows(np.reshape(rows, (-1, shp[-1])), din, dout, nout)
    return out.astype(f32).astype(np.float64).reshape(shp[:-1] + (nout,))


def _pchip_slope(r, k):
    nn = len(r)
    if nn == 2:
        return r[1] - r[0]
    if k == 0 or k == nn - 1:
        a, b = (r[1] - r[0], r[2] - r[1]) if k == 0 else (r[nn - 1] - r[nn - 2], r[nn - 2] - r[nn - 3])
        d = (3.0 * a - b) / 2.0
        if np.sign(d) != np.sign(a):
            return 0.0
        if np.sign(a) != np.sign(b) and abs(d) > abs(3.0 * a):
            return 3.0 * a
        return d
    a, b = r[k] - r[k - 1], r[k + 1] - r[k]
    if a == 0 or b == 0 or (a > 0) != (b > 0):
        return 0.0
    return 2.0 / (1.0 / a + 1.0 / b)


def pchip_rows(rows, din, dout, nout):
    """interp_to(x, [nout, nr], method=['pchip', 'nearest']) (:909-910) of
    single-precision rows sampled at din onto nout samples at dout."""
    shp = np.shape(rows)
    R = np.reshape(np.asarray(rows, dtype=np.float64), (-1, shp[-1]))
    nn = R.shape[1]
    out = np.zeros((R.shape[0], nout))
    for i in range(nout):
        x = (i * dout) / din
        if abs(x - np.rint(x)) <= 1e-4:
            x = float(np.rint(x))
        x = min(max(x, 0.0), float(nn - 1))
        j0 = min(int(math.floor(x)), nn - 2)
        u = x - j0
        w = 1.0 - u
        h00, h10 = (1.0 + 2.0 * u) * (w * w), u * (w * w)
        h01, h11 = (u * u) * (3.0 - 2.0 * u), (u * u) * (u - 1.0)
        for t in range(R.shape[0]):
            r = R[t]
            out[t, i] = h00 * r[j0] + h10 * _pchip_slope(r, j0) + h01 * r[j0 + 1] + h11 * _pchip_slope(r, j0 + 1)
    return out.astype(f32).reshape(shp[:-1] + (nout,))


def _adj_sampling(dsyn, dobs, dd, adj_nt):
    """(n, dd, dsyn, dobs) of the shift computation: the normalised traces
    resampled to adj_nt samples over the same span (:744-750, :765-768)."""
    n = np.shape(dsyn)[-1]
    if adj_nt <= 0 or adj_nt == n:
        return n, dd, dsyn, dobs
    ddn = float(f32(f32(n - 1) * f32(dd)) / f32(adj_nt - 1))
    return adj_nt, ddn, resample_f32(dsyn, dd, ddn, adj_nt), resample_f32(dobs, dd, ddn, adj_nt)


def _normal(a):
    a = np.asarray(a, dtype=np.float64)
    return np.where(np.isfinite(a), a, 0.0)


def dtw_gather(syn, obs, live, dd, tlag_max, form=PHASE, niter=5, rinst=0.1, rcuml=1.0, epsabs=1.0e-2,
               epsrel=1.0e-3, power=0.5, amp_weight=1.0, trc=0, adj_nt=0):
    """compute_adjsrc_dtw (:715-980) on one gather (nr, n): returns
    (adj, trace misfits, tau in seconds, quality weights)."""
    syn = np.asarray(syn, dtype=f32)
    obs = np.asarray(obs, dtype=f32)
    nr, n = syn.shape
    live = np.asarray(live, dtype=bool)
    dd = float(f32(dd))  # the reference's sample interval is single precision
    # normalised traces (:761-775), single-precision division, float64 storage
    dsyn = np.zeros((nr, n))
    dobs = np.zeros((nr, n))
    for i in range(nr):
        if live[i]:
            dsyn[i] = (syn[i] / f32(np.linalg.norm(syn[i].astype(np.float64)))).astype(np.float64)
            dobs[i] = (obs[i] / f32(np.linalg.norm(obs[i].astype(np.float64)))).astype(np.float64)
    n0, dd0 = n, dd
    n, dd, dsyn, dobs = _adj_sampling(dsyn, dobs, dd, adj_nt)
    m = lag_count(tlag_max, dd)
    tau = np.zeros((nr, n), dtype=f32)
    for i in range(nr):
        if not live[i]:
            continue
        cols = [c for c in range(i - trc, i + trc + 1)]
        X = np.stack([dobs[c] if 0 <= c < nr else np.zeros(n) for c in cols], axis=1)
        Y = np.stack([dsyn[c] if 0 <= c < nr else np.zeros(n) for c in cols], axis=1)
        ts, _ = gdtw(X, Y, m, niter, float(f32(rinst)), float(f32(rcuml)), float(f32(epsabs)), float(f32(epsrel)),
                     float(f32(power)))
        tau[i] = (ts * float(f32(dd))).astype(f32)
    # quality weights (:838-905)
    q = np.zeros((nr, n), dtype=f32)
    if form == AMP:
        q[:] = 1.0
    else:
        nw = nint(float(f32(tlag_max) / f32(dd)))
        tg = np.arange(n, dtype=f32) * f32(dd)
        for i in range(nr):
            if not live[i]:
                continue
            dw = _lin_interp_zero(tg, dobs[i].astype(f32), (tau[i] + tg).astype(f32)).astype(np.float64)
            eta = f32(max(np.linalg.norm(dsyn[i]), np.linalg.norm(dw)) * float(f32(1.0e-2)))
            if eta == 0:
                eta = f32(1.0e-9)
            qi = np.zeros(n, dtype=f32)
            for j in range(n):
                lo, hi = max(0, j - nw), min(n - 1, j + nw)
                uu = dsyn[i, lo:hi + 1].astype(f32)
                vv = dw[lo:hi + 1].astype(f32)
                num = np.dot(uu.astype(np.float64), vv.astype(np.float64))
                den = np.linalg.norm(uu.astype(np.float64)) * np.linalg.norm(vv.astype(np.float64)) + float(eta)
                qi[j] = f32(num / den)
            qi = np.abs(qi) ** f32(0.2)
            qi = median7(qi.astype(f32))
            qd = gauss3(qi.astype(np.float64))
            qd = qd / np.linalg.norm(qd)
            with np.errstate(invalid="ignore", divide="ignore"):
                qd = (qd - qd.min()) / (qd.max() - qd.min())
            q[i] = _normal(qd).astype(f32)
        for i in range(nr):
            if np.max(np.abs(q[i])) == 0:
                q[i] = 1.0
    if n != n0:  # shifts and weights back to the trace length (:907-911)
        tau, q = pchip_rows(tau, dd, dd0, n0), pchip_rows(q, dd, dd0, n0)
        n, dd = n0, dd0
    # adjoint source (:917-978)
    adj = np.zeros((nr, n))
    tm = np.zeros(nr)
    td = np.arange(n, dtype=f32) * f32(dd)
    for i in range(nr):
        if not live[i]:
            continue
        pos = ((tau[i] + td).astype(f32) / f32(dd)).astype(np.float64)
        warped = _cubic_warp(obs[i].astype(np.float64), pos)
        qi, ti = q[i].astype(np.float64), tau[i].astype(np.float64)
        mph = float(np.sum(qi * ti * ti))
        if form == PHASE:
            tm[i] = mph
            adj[i] = qi * ti * deriv(warped) / dd
        elif form == AMP:
            r = syn[i].astype(np.float64) - warped
            tm[i] = float(np.sum(r * r))
            adj[i] = r
        else:
            r = syn[i].astype(np.float64) - warped
            ma = float(np.sum(r * r))
            tm[i] = mph * (1.0 + amp_weight)
            adj[i] = qi * ti * deriv(warped) / dd + amp_weight * mph / (ma + F32_TINY) * r
    return adj, tm, tau, q


def adjoint_source(gather_ptr, syn, obs, weight=None, dt=1e-3, tlag_max=0.0, discard_threshold=0.0, **kw):
    """compute_adjoint_source (:985-1277) with misfit_type 'dtw' over gathers of
    rows: the trace discard rule (:1047-1050), then one dtw_gather per gather.
    Returns (adj, trace misfits, gather misfits, tau)."""
    syn = np.asarray(syn, dtype=f32)
    obs = np.asarray(obs, dtype=f32)
    ntr, nt = syn.shape
    tlag = tlag_max if tlag_max > 0 else float(f32(0.1) * f32(nt - 1) * f32(dt))
    thr = discard_threshold if discard_threshold != 0 else 1.0e-6
    thr = max(thr, 0.0)
    w = np.ones(ntr) if weight is None else np.asarray(weight, dtype=np.float64)
    adj = np.zeros((ntr, nt))
    tm = np.zeros(ntr)
    tau = np.zeros((ntr, nt), dtype=f32)
    gm = np.zeros(len(gather_ptr) - 1)
    for g in range(len(gather_ptr) - 1):
        r0, r1 = gather_ptr[g], gather_ptr[g + 1]
        if r1 <= r0:
            continue
        no = np.linalg.norm(obs[r0:r1].astype(np.float64), axis=1)
        ns = np.linalg.norm(syn[r0:r1].astype(np.float64), axis=1)
        mo, ms = no.max(), ns.max()
        live = np.array([not (w[r] == 0 or no[r - r0] < thr * mo or ns[r - r0] < thr * ms
                              or no[r - r0] * ns[r - r0] == 0) for r in range(r0, r1)])
        # discarded traces enter the gather as zeros (:1052-1068)
        s = np.where(live[:, None], syn[r0:r1], 0).astype(f32)
        o = np.where(live[:, None], obs[r0:r1], 0).astype(f32)
        a, t_m, ta, _ = dtw_gather(s, o, live, dt, tlag, **kw)
        adj[r0:r1] = a
        tm[r0:r1] = t_m
        tau[r0:r1] = ta
        gm[g] = tm[r0:r1].sum()
    return adj, tm, gm, tau


def dtw_vector(syn, obs, live, dd, tlag_max, form=PHASE, niter=5, rinst=0.1, rcuml=1.0, epsabs=1.0e-2,
               epsrel=1.0e-3, power=0.5, amp_weight=1.0, trc=0, adj_nt=0):
    """compute_adjsrc_dtw on the components of one shot together ('dtw-vector',
    :1232-1236): syn, obs (nc, nr, n), live (nc, nr) after the discard rule.
    A receiver is kept when any component is; traces are normalised by the
    norm over the receiver's kept components; one shift and one quality weight
    per receiver (the components' windowed correlations summed); the adjoint per
    component. Returns (adj (nc, nr, n), trace misfits (nc, nr), tau (nc, nr, n))
    with a receiver's misfit shared by its component rows: 'phase' equally,
    'amp' each row its own, 'phase+amp' each row the phase term (times
    1 + amp_weight) -- their sum is the reference's err_trc."""
    syn = np.asarray(syn, dtype=f32)
    obs = np.asarray(obs, dtype=f32)
    nc, nr, n = syn.shape
    live = np.asarray(live, dtype=bool)
    dd = float(f32(dd))
    lv = live.any(axis=0)
    dsyn = np.zeros((nc, nr, n))
    dobs = np.zeros((nc, nr, n))
    for i in range(nr):
        if not lv[i]:
            continue
        ns = f32(np.sqrt(sum(np.linalg.norm(syn[c, i].astype(np.float64)) ** 2 for c in range(nc) if live[c, i])))
        no = f32(np.sqrt(sum(np.linalg.norm(obs[c, i].astype(np.float64)) ** 2 for c in range(nc) if live[c, i])))
        for c in range(nc):
            if live[c, i]:
                dsyn[c, i] = (syn[c, i] / ns).astype(np.float64)
                dobs[c, i] = (obs[c, i] / no).astype(np.float64)
    n0, dd0 = n, dd
    n, dd, dsyn, dobs = _adj_sampling(dsyn, dobs, dd, adj_nt)
    m = lag_count(tlag_max, dd)
    tau = np.zeros((nc, nr, n), dtype=f32)
    for i in range(nr):
        if not lv[i]:
            continue
        cols = [(c, q) for c in range(nc) for q in range(i - trc, i + trc + 1)]
        X = np.stack([dobs[c, q] if 0 <= q < nr else np.zeros(n) for c, q in cols], axis=1)
        Y = np.stack([dsyn[c, q] if 0 <= q < nr else np.zeros(n) for c, q in cols], axis=1)
        ts, _ = gdtw(X, Y, m, niter, float(f32(rinst)), float(f32(rcuml)), float(f32(epsabs)), float(f32(epsrel)),
                     float(f32(power)))
        tau[:, i] = (ts * float(f32(dd))).astype(f32)
    q = np.zeros((nr, n), dtype=f32)
    if form == AMP:
        q[:] = 1.0
    else:
        nw = nint(float(f32(tlag_max) / f32(dd)))
        tg = np.arange(n, dtype=f32) * f32(dd)
        for i in range(nr):
            if not lv[i]:
                continue
            acc = np.zeros(n, dtype=f32)
            for c in range(nc):
                if not live[c, i]:
                    continue
                dw = _lin_interp_zero(tg, dobs[c, i].astype(f32), (tau[c, i] + tg).astype(f32)).astype(np.float64)
                eta = f32(max(np.linalg.norm(dsyn[c, i]), np.linalg.norm(dw)) * float(f32(1.0e-2)))
                if eta == 0:
                    eta = f32(1.0e-9)
                for j in range(n):
                    lo, hi = max(0, j - nw), min(n - 1, j + nw)
                    uu = dsyn[c, i, lo:hi + 1].astype(f32).astype(np.float64)
                    vv = dw[lo:hi + 1].astype(f32).astype(np.float64)
                    acc[j] = f32(acc[j] + f32(np.dot(uu, vv) / (np.linalg.norm(uu) * np.linalg.norm(vv) + float(eta))))
            qi = np.abs(acc) ** f32(0.2)
            qi = median7(qi.astype(f32))
            qd = gauss3(qi.astype(np.float64))
            qd = qd / np.linalg.norm(qd)
            with np.errstate(invalid="ignore", divide="ignore"):
                qd = (qd - qd.min()) / (qd.max() - qd.min())
            q[i] = _normal(qd).astype(f32)
        for i in range(nr):
            if np.max(np.abs(q[i])) == 0:
                q[i] = 1.0
    if n != n0:
        tau, q = pchip_rows(tau, dd, dd0, n0), pchip_rows(q, dd, dd0, n0)
        n, dd = n0, dd0
    adj = np.zeros((nc, nr, n))
    tm = np.zeros((nc, nr))
    td = np.arange(n, dtype=f32) * f32(dd)
    for i in range(nr):
        if not lv[i]:
            continue
        qi = q[i].astype(np.float64)
        for c in range(nc):
            ti = tau[c, i].astype(np.float64)
            mph = float(np.sum(qi * ti * ti))
            if not live[c, i]:
                tm[c, i] = mph / nc if form == PHASE else (0.0 if form == AMP else mph * (1.0 + amp_weight))
                continue
            pos = ((tau[c, i] + td).astype(f32) / f32(dd)).astype(np.float64)
            warped = _cubic_warp(obs[c, i].astype(np.float64), pos)
            r = syn[c, i].astype(np.float64) - warped
            if form == PHASE:
                tm[c, i] = mph / nc
                adj[c, i] = qi * ti * deriv(warped) / dd
            elif form == AMP:
                tm[c, i] = float(np.sum(r * r))
                adj[c, i] = r
            else:
                ma = float(np.sum(r * r))
                tm[c, i] = mph * (1.0 + amp_weight)
                adj[c, i] = qi * ti * deriv(warped) / dd + amp_weight * mph / (ma + F32_TINY) * r
    return adj, tm, tau


def adjoint_source_vector(gather_ptr, syn, obs, ncomp, weight=None, dt=1e-3, tlag_max=0.0, discard_threshold=0.0,
                          **kw):
    """'dtw-vector' over gathers of rows: consecutive groups of ncomp gathers
    (equal lengths) are one shot's components; the discard rule per gather,
    then dtw_vector per shot. Returns (adj, trace misfits, gather misfits, tau)."""
    syn = np.asarray(syn, dtype=f32)
    obs = np.asarray(obs, dtype=f32)
    ntr, nt = syn.shape
    tlag = tlag_max if tlag_max > 0 else float(f32(0.1) * f32(nt - 1) * f32(dt))
    thr = discard_threshold if discard_threshold != 0 else 1.0e-6
    thr = max(thr, 0.0)
    w = np.ones(ntr) if weight is None else np.asarray(weight, dtype=np.float64)
    ng = len(gather_ptr) - 1
    live = np.zeros(ntr, dtype=bool)
    for g in range(ng):
        r0, r1 = gather_ptr[g], gather_ptr[g + 1]
        if r1 <= r0:
            continue
        no = np.linalg.norm(obs[r0:r1].astype(np.float64), axis=1)
        ns = np.linalg.norm(syn[r0:r1].astype(np.float64), axis=1)
        mo, ms = no.max(), ns.max()
        for r in range(r0, r1):
            i = r - r0
            live[r] = not (w[r] == 0 or no[i] < thr * mo or ns[i] < thr * ms or no[i] * ns[i] == 0)
    adj = np.zeros((ntr, nt))
    tm = np.zeros(ntr)
    tau = np.zeros((ntr, nt), dtype=f32)
    for g0 in range(0, ng, ncomp):
        rows = [list(range(gather_ptr[g0 + c], gather_ptr[g0 + c + 1])) for c in range(ncomp)]
        S = np.stack([np.where(live[rs][:, None], syn[rs], 0) for rs in rows]).astype(f32)
        O = np.stack([np.where(live[rs][:, None], obs[rs], 0) for rs in rows]).astype(f32)
        Lv = np.stack([live[rs] for rs in rows])
        a, t_m, ta = dtw_vector(S, O, Lv, dt, tlag, **kw)
        for c, rs in enumerate(rows):
            adj[rs] = a[c]
            tm[rs] = t_m[c]
            tau[rs] = ta[c]
    gm = np.array([tm[gather_ptr[g]:gather_ptr[g + 1]].sum() for g in range(ng)])
    return adj, tm, gm, tau
