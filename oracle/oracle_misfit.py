"""Oracle (test infrastructure only): FP64 numpy restatement of the reference's
data-domain misfits and adjoint sources.

Follows src/inverse/module_inversion_adjoint_source.f90:
  compute_adjsrc_waveform   :371-383
  compute_adjsrc_corr       :391-412
  compute_adjsrc_envelope   :424-451
  compute_adjsrc_phase      :459-482
  compute_adjsrc_adaptive   :490-537, xcorr_penalty :321-363
  compute_adjsrc_local_adaptive     :545-625 (adaptive matching filter per
                                     Gaussian time window, lawi_sigma)
  compute_adjsrc_adaptive_spacetime :630-700 (matching filter averaged over
                                     the trace and adaptive_half_window
                                     neighbours on each side, :1168-1220)
  compute_adjoint_source    :985-1277 (trace discard rule :1038-1070, per-trace
                                       misfit sums :1150-1165)

FLIT (github.com/lanl/flit, no version pinned by the reference) supplies
`hilbert`, `envelope`, `instant_phase`, `fft` / `ifft`, `taper`, `rescale` and
`next_power_235`; none of them is vendored here and no reference test pins
them, so they are restated from their usual definitions -- parity unpinned:
  hilbert(x)       imaginary part of the analytic signal of x from a length-n
                   DFT (X[0] and, for even n, X[n/2] kept, X[1..] doubled,
                   the negative frequencies zeroed);
  envelope(x)      |analytic signal|;  instant_phase(x) its argument (atan2);
  fft / ifft       unnormalised forward, 1/n inverse;
  taper(x, [a, b]) Hann ramps 0.5 (1 - cos(pi i / a)), i = 0..a-1, over the
                   first a samples and mirrored over the last b;
  rescale(w, [0,1]) (w - min) / (max - min);
  next_power_235(n) the smallest m >= n with no prime factor above 5;
  gaussian(a, mu, sigma) exp(-(a - mu)^2 / (2 sigma^2)) (unnormalised window);
  float_small      1e-30 (only reached by all-zero traces, which the discard
                   rule drops first).
"""
from __future__ import annotations

import numpy as np

WAVEFORM, CORR, ENVELOPE, PHASE, ADAPTIVE = 0, 1, 2, 3, 4
LOCAL_ADAPTIVE, ADAPTIVE_SPACETIME = 6, 7
FLOAT_SMALL = 1.0e-30
LINEAR, POWER, GAUSSIAN, EXP = 0, 1, 2, 3


def next_power_235(n: int) -> int:
    m = max(1, int(n))
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def taper(x, a: int, b: int):
    y = np.array(x, dtype=np.float64, copy=True)
    n = y.size
    for i in range(min(a, n)):
        y[i] *= 0.5 * (1.0 - np.cos(np.pi * i / a))
    for i in range(min(b, n)):
        y[n - 1 - i] *= 0.5 * (1.0 - np.cos(np.pi * i / b))
    return y


def analytic(x):
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    X = np.fft.fft(x)
    h = np.zeros(n)
    h[0] = 1.0
    if n % 2 == 0:
        h[n // 2] = 1.0
        h[1:n // 2] = 2.0
    else:
        h[1:(n + 1) // 2] = 2.0
    return np.fft.ifft(X * h)


def hilbert(x):
    return analytic(x).imag


def envelope(x):
    return np.abs(analytic(x))


def instant_phase(x):
    z = analytic(x)
    return np.arctan2(z.imag, z.real)


def waveform(obs, syn):
    """compute_adjsrc_waveform (:371-383)"""
    r = syn - obs
    return float(np.sum(r * r)), r


def corr(obs, syn):
    """compute_adjsrc_corr (:391-412)"""
    no, ns = np.linalg.norm(obs), np.linalg.norm(syn)
    if np.max(np.abs(syn)) == 0 and np.max(np.abs(obs)) != 0:
        return float(np.sum((obs / no) ** 2)), -obs / no
    m = float(np.sum((syn / ns - obs / no) ** 2))
    adj = (np.dot(syn, obs) / ns ** 2 * syn - obs) / (no * ns)
    return m, adj


def envelope_misfit(obs, syn, stab=1.0e-2):
    """compute_adjsrc_envelope (:424-451)"""
    e1, z = envelope(obs), analytic(syn)
    e2 = np.abs(z)
    m = float(np.sum((e1 - e2) ** 2))
    mx = np.max(e2)
    coef = np.zeros_like(e2) if mx == 0 else (e2 - e1) / (e2 + stab * mx)
    adj = syn * coef - hilbert(z.imag * coef)
    return m, adj


def phase_misfit(obs, syn, stab=5.0e-2):
    """compute_adjsrc_phase (:459-482)"""
    zd, zu = analytic(obs), analytic(syn)
    phid, phiu = np.arctan2(zd.imag, zd.real), np.arctan2(zu.imag, zu.real)
    m = float(np.sum((phid - phiu) ** 2))
    env = zu.real ** 2 + zu.imag ** 2
    env = env + stab * np.max(env)
    dphi = phiu - phid
    adj = -dphi * zu.imag / env + hilbert(dphi * syn / env)
    return m, adj


def penalty(dt, maxlag, tlag_max, method=LINEAR, power=1.0):
    """xcorr_penalty (:321-363), lags -maxlag..maxlag"""
    i = np.arange(-maxlag, maxlag + 1, dtype=np.float64)
    s = 1.0 / np.sqrt(2.0 * np.log(100.0))
    if method == POWER:
        return np.abs(i * dt / tlag_max) ** abs(power)
    if method in (GAUSSIAN, EXP):
        w = np.exp(-(i * dt) ** 2 / (s * tlag_max ** 2)) if method == GAUSSIAN else np.exp(-np.abs(i * dt) / (s * tlag_max))
        w = (w - w.min()) / (w.max() - w.min())
        return 1.0 - w ** abs(power)
    return np.abs(i * dt / tlag_max)


def adaptive(obs, syn, dt, tlag_max, method=LINEAR, power=1.0, deconv_eps=0.1):
    """compute_adjsrc_adaptive (:490-537)"""
    n = obs.size
    maxlag = int(np.ceil(np.float32(tlag_max) / np.float32(dt)))
    nnt = next_power_235(2 * n)
    maxlag = min(maxlag, (nnt - 1) // 2)
    tl = int(np.floor(0.025 * n + 0.5))
    u = np.zeros(nnt)
    d = np.zeros(nnt)
    u[:n] = taper(syn, tl, tl)
    d[:n] = taper(obs, tl, tl)
    uu, dd = np.fft.fft(u), np.fft.fft(d)
    pd = (dd * np.conj(dd)).real
    eps = deconv_eps * np.max(pd)
    xc = np.fft.ifft(uu * np.conj(dd) / (pd + eps)).real
    p = penalty(dt, maxlag, tlag_max, method, power)
    w = np.zeros(nnt)
    w[:maxlag + 1] = p[maxlag:]
    if maxlag > 0:
        w[nnt - maxlag:] = p[:maxlag]
    sxx = np.sum(xc ** 2)
    m = 0.5 * float(np.sum((w * xc) ** 2)) / sxx
    g = (w ** 2 - 2.0 * m) * xc / sxx
    a = np.fft.ifft(np.fft.fft(g) * dd / (pd + eps)).real
    adj = taper(a[:n], 0, tl)
    return m, adj


def _awi_setup(n, dt, tlag_max, method, power, nnt):
    maxlag = int(np.ceil(np.float32(tlag_max) / np.float32(dt)))
    maxlag = min(maxlag, (nnt - 1) // 2)
    p = penalty(dt, maxlag, tlag_max, method, power)
    w = np.zeros(nnt)
    w[:maxlag + 1] = p[maxlag:]
    if maxlag > 0:
        w[nnt - maxlag:] = p[:maxlag]
    return w, int(np.floor(0.025 * n + 0.5))


def local_adaptive(obs, syn, dt, tlag_max, method=LINEAR, power=1.0, deconv_eps=0.1, sigma=0.25):
    """compute_adjsrc_local_adaptive (:545-625)"""
    n = obs.size
    nnt = next_power_235(2 * n)
    w, tl = _awi_setup(n, dt, tlag_max, method, power, nnt)
    u = np.zeros(nnt)
    d = np.zeros(nnt)
    u[:n] = taper(syn, tl, tl)
    d[:n] = taper(obs, tl, tl)
    u0, d0 = np.fft.fft(u), np.fft.fft(d)
    eps = deconv_eps * np.max((d0 * np.conj(d0)).real)
    eps = eps if eps != 0 else FLOAT_SMALL
    xc = np.fft.ifft(u0 * np.conj(d0) / ((d0 * np.conj(d0)).real + eps)).real
    eta = deconv_eps * np.max(xc ** 2)
    eta = eta if eta != 0 else FLOAT_SMALL
    a = np.arange(1, nnt + 1, dtype=np.float64)
    sg = sigma / dt
    adj = np.zeros(nnt)
    s = np.zeros(nnt)
    m = 0.0
    for i in range(1, n + 1):
        g = np.exp(-(a - i) ** 2 / (2.0 * sg * sg))
        uu, dd = np.fft.fft(u * g), np.fft.fft(d * g)
        pd = (dd * np.conj(dd)).real + eps
        xc = np.fft.ifft(uu * np.conj(dd) / pd).real
        sx = np.sum(xc ** 2) + eta
        vt = np.sum((w * xc) ** 2) / sx
        m += vt * vt
        af = np.fft.fft(vt * (w ** 2 - vt) * xc / sx) * dd / pd
        adj += np.fft.ifft(af).real * g
        s += g * g
    adj = taper(adj[:n] / s[:n], 0, tl)
    return float(m), adj


def adaptive_spacetime(obs_rows, syn_rows, centre, dt, tlag_max, method=LINEAR, power=1.0, deconv_eps=0.1):
    """compute_adjsrc_adaptive_spacetime (:630-700): rows (nc, n), centre the
    row of the trace whose adjoint source is formed"""
    nc, n = obs_rows.shape
    nnt = next_power_235(4 * n)
    w, tl = _awi_setup(n, dt, tlag_max, method, power, nnt)
    xcs = np.zeros(nnt, dtype=complex)
    l = 0
    dd_c = eps_c = None
    for i in range(nc):
        u = np.zeros(nnt)
        d = np.zeros(nnt)
        u[:n] = taper(syn_rows[i], tl, tl)
        d[:n] = taper(obs_rows[i], tl, tl)
        uu, dd = np.fft.fft(u), np.fft.fft(d)
        df = (dd * np.conj(dd)).real
        eps = deconv_eps * np.max(df)
        if i == centre:
            dd_c, eps_c = dd, eps
        if eps > 0:
            xcs += uu * np.conj(dd) / (df + eps)
            l += 1
    xc = np.fft.ifft(xcs).real / l if l > 0 else np.zeros(nnt)
    m = 0.5 * float(np.sum((w * xc) ** 2)) / float(np.sum(xc ** 2)) if l > 0 else 0.0
    dfc = (dd_c * np.conj(dd_c)).real
    a = np.fft.ifft(np.fft.fft((w ** 2 - 2 * m) * xc / np.sum(xc ** 2)) * dd_c / (dfc + eps_c)).real
    return m, taper(a[:n], 0, tl)


def trace_misfit(kind, obs, syn, dt=1e-3, tlag_max=0.1, penalty_method=LINEAR, penalty_power=1.0,
                 deconv_eps=0.1, lawi_sigma=0.25):
    obs = np.asarray(obs, dtype=np.float64)
    syn = np.asarray(syn, dtype=np.float64)
    if kind == WAVEFORM:
        return waveform(obs, syn)
    if kind == CORR:
        return corr(obs, syn)
    if kind == ENVELOPE:
        return envelope_misfit(obs, syn)
    if kind == PHASE:
        return phase_misfit(obs, syn)
    if kind == ADAPTIVE:
        return adaptive(obs, syn, dt, tlag_max, penalty_method, penalty_power, deconv_eps)
    if kind == LOCAL_ADAPTIVE:
        return local_adaptive(obs, syn, dt, tlag_max, penalty_method, penalty_power, deconv_eps, lawi_sigma)
    raise ValueError(kind)


def adjoint_source(kind, gather_ptr, syn, obs, weight=None, dt=1e-3, tlag_max=0.0, penalty_method=LINEAR,
                   penalty_power=0.0, deconv_eps=0.0, discard_threshold=0.0, lawi_sigma=0.0,
                   adaptive_half_window=0, adj_nt=0):
    """compute_adjoint_source (:985-1277) over gathers of rows: returns
    (adj, trace misfits, gather misfits). Zero-valued options take the
    reference's defaults (module_parameters.f90:550-570). adj_nt (:1082-1152):
    the traces kept by the discard rule are resampled to adj_nt samples over
    the same span (cubic, FLIT interp_to restated as the Keys cubic convolution
    of oracle_resample) before the misfit, the adjoint resampled back."""
    syn = np.asarray(syn, dtype=np.float64)
    obs = np.asarray(obs, dtype=np.float64)
    ntr, nt = syn.shape
    if adj_nt > 0 and adj_nt != nt:
        from oracle.oracle_resample import resample_rows
        f32 = np.float32
        dd = float(f32(f32(nt - 1) * f32(dt)) / f32(adj_nt - 1))
        thr = discard_threshold if discard_threshold != 0 else 1.0e-6
        thr = max(thr, 0.0)
        w0 = np.ones(ntr) if weight is None else np.asarray(weight, dtype=np.float64)
        keep = np.zeros(ntr)
        for g in range(len(gather_ptr) - 1):
            r0, r1 = gather_ptr[g], gather_ptr[g + 1]
            if r1 <= r0:
                continue
            no = np.linalg.norm(obs[r0:r1], axis=1)
            ns = np.linalg.norm(syn[r0:r1], axis=1)
            for r in range(r0, r1):
                i = r - r0
                keep[r] = not (w0[r] == 0 or no[i] < thr * no.max() or ns[i] < thr * ns.max() or no[i] * ns[i] == 0)
        ts = resample_rows(syn, float(f32(dt)), dd, adj_nt)
        to = resample_rows(obs, float(f32(dt)), dd, adj_nt)
        a, tm, gm = adjoint_source(kind, gather_ptr, ts, to, keep, dd, tlag_max, penalty_method, penalty_power,
                                   deconv_eps, -1.0, lawi_sigma, adaptive_half_window)
        return resample_rows(a, dd, float(f32(dt)), nt), tm, gm
    tlag = tlag_max if tlag_max > 0 else float(np.float32(0.1) * np.float32(nt - 1) * np.float32(dt))
    pp = penalty_power if penalty_power != 0 else 1.0
    eps = deconv_eps if deconv_eps > 0 else 0.1
    thr = discard_threshold if discard_threshold != 0 else 1.0e-6
    thr = max(thr, 0.0)
    sgm = lawi_sigma if lawi_sigma > 0 else 0.25
    hw = adaptive_half_window if adaptive_half_window > 0 else 3
    w = np.ones(ntr) if weight is None else np.asarray(weight, dtype=np.float64)
    adj = np.zeros_like(syn)
    tm = np.zeros(ntr)
    gm = np.zeros(len(gather_ptr) - 1)
    for g in range(len(gather_ptr) - 1):
        r0, r1 = gather_ptr[g], gather_ptr[g + 1]
        if r1 <= r0:
            continue
        no = np.linalg.norm(obs[r0:r1], axis=1)
        ns = np.linalg.norm(syn[r0:r1], axis=1)
        mo, ms = no.max(), ns.max()
        keep = [not (w[r] == 0 or no[r - r0] < thr * mo or ns[r - r0] < thr * ms or no[r - r0] * ns[r - r0] == 0)
                for r in range(r0, r1)]
        for r in range(r0, r1):
            i = r - r0
            if not keep[i]:
                continue
            if kind == ADAPTIVE_SPACETIME:
                # the gather padded with zero traces, dropped traces zero (:1168-1200)
                rows = range(r - hw, r + hw + 1)
                orows = np.array([obs[q] if r0 <= q < r1 and keep[q - r0] else np.zeros(nt) for q in rows])
                srows = np.array([syn[q] if r0 <= q < r1 and keep[q - r0] else np.zeros(nt) for q in rows])
                m, a = adaptive_spacetime(orows, srows, hw, dt, tlag, penalty_method, pp, eps)
            else:
                m, a = trace_misfit(kind, obs[r], syn[r], dt, tlag, penalty_method, pp, eps, sgm)
            tm[r] = m
            adj[r] = a
        gm[g] = tm[r0:r1].sum()
    return adj, tm, gm
