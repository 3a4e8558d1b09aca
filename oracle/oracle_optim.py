"""Oracle (test infrastructure only): FP64 restatement of the search directions
and the gradient processing the GPU path computes.

compute_search_direction (src/inverse/module_inversion_search_direction.f90):
  steepest descent -g; Polak-Ribiere CG :38-86 (beta = max(0, g.(g - gp) / gp.gp));
  L-BFGS two-loop recursion :91-246 over s_i = x_{i+1} - x_i, y_i = g_{i+1} - g_i.
process_model_single_parameter (src/inverse/2d/module_gradient.f90:733-892):
  smooth (FLIT gauss_filt), taper (FLIT taper, Blackman ramps), mask, scale,
  max_balance, rms_balance (FLIT mean(w, 2), restated as the root mean
  square), rms_balance_z / _x (:795-823, restated as written: each slice
  divided by the L2 norm of the odd window of slices around it, NaN / Inf -> 0),
  median_filt (FLIT, restated as the median of the window of the given
  half-widths, truncated at the ends, the mean of the two middle values of an
  even count). FLIT is not vendored (no version pinned) and no reference test
  pins gauss_filt or taper -- parity unpinned: restated as a Gaussian of the
  given standard deviation in cells truncated at ceil(3 sigma), normalised,
  edge samples replicated; Blackman ramps 0.42 - 0.5 cos(pi i / l) +
  0.08 cos(2 pi i / l), i = 0..l-1, from each end of an axis.
"""
from __future__ import annotations

import math

import numpy as np

SD, CG, LBFGS = 0, 1, 2
SMOOTH, TAPER, MASK, SCALE, MAX_BALANCE = 0, 1, 2, 3, 4
RMS_BALANCE, RMS_BALANCE_AXIS, MEDIAN = 5, 6, 7


def search_direction(method, models, grads, prev_srch=None):
    x = [np.asarray(m, dtype=np.float64).ravel() for m in models]
    g = [np.asarray(v, dtype=np.float64).ravel() for v in grads]
    gk = g[-1]
    if method == SD or len(g) < 2:
        return -gk
    if method == CG:
        gp = g[-2]
        s1 = float(np.dot(gp, gp))
        s2 = float(np.dot(gk, gk - gp))
        beta = 0.0 if s1 == 0 else max(0.0, s2 / s1)
        return -gk + beta * np.asarray(prev_srch, dtype=np.float64).ravel()
    npair = len(g) - 1
    q = gk.copy()
    alpha = [0.0] * npair
    ys = [0.0] * npair
    for i in range(npair - 1, -1, -1):
        s, y = x[i + 1] - x[i], g[i + 1] - g[i]
        ys[i] = float(np.dot(y, s))
        alpha[i] = 0.0 if ys[i] == 0 else float(np.dot(s, q)) / ys[i]
        q = q - alpha[i] * y
    s, y = x[npair] - x[npair - 1], g[npair] - g[npair - 1]
    yy = float(np.dot(y, y))
    r = (0.0 if yy == 0 else float(np.dot(s, y)) / yy) * q
    for i in range(npair):
        s, y = x[i + 1] - x[i], g[i + 1] - g[i]
        beta = 0.0 if ys[i] == 0 else float(np.dot(y, r)) / ys[i]
        r = r + s * (alpha[i] - beta)
    return -r


def _ramp(j, l):
    if j >= l:
        return 1.0
    t = j / l
    return 0.42 - 0.5 * math.cos(math.pi * t) + 0.08 * math.cos(2 * math.pi * t)


def process(op, field, param=None, mask=None):
    """field: array shaped (n2, n1) or (n3, n2, n1), n1 the fastest (z) axis"""
    f = np.array(field, dtype=np.float64, copy=True)
    if op == SMOOTH:
        for ax in range(3):
            sg = float(param[ax])
            axis = f.ndim - 1 - ax
            if axis < 0 or not sg > 0 or f.shape[axis] < 2:
                continue
            rad = max(1, int(math.ceil(3.0 * sg)))
            k = np.arange(-rad, rad + 1)
            w = np.exp(-0.5 * k * k / (sg * sg))
            w /= w.sum()
            n = f.shape[axis]
            out = np.zeros_like(f)
            for kk, wk in zip(k, w):
                idx = np.clip(np.arange(n) + kk, 0, n - 1)
                out += wk * np.take(f, idx, axis=axis)
            f = out
        return f
    if op == TAPER:
        ls = [int(round(v)) for v in param]
        for ax in range(3):
            axis = f.ndim - 1 - ax
            if axis < 0 or f.shape[axis] < 2:
                continue
            n = f.shape[axis]
            w = np.array([_ramp(j, ls[2 * ax]) * _ramp(n - 1 - j, ls[2 * ax + 1]) for j in range(n)])
            shape = [1] * f.ndim
            shape[axis] = n
            f = f * w.reshape(shape)
        return f
    if op == MASK:
        return f * np.asarray(mask, dtype=np.float64)
    if op == SCALE:
        return f * float(param[0])
    if op == MAX_BALANCE:
        m = f.max()
        return f / m if m != 0 else f
    if op == RMS_BALANCE:
        r = math.sqrt(float(np.mean(f * f)))
        return f / r if r != 0 else f
    if op == RMS_BALANCE_AXIS:
        axis = f.ndim - int(round(param[0]))
        wn = int(round(param[1]))
        if wn % 2 == 0:
            wn -= 1
        hw = (wn - 1) // 2
        fm = np.moveaxis(f, axis, 0)
        ss = np.array([np.sum(fm[j] ** 2) for j in range(fm.shape[0])])
        nrm = np.array([math.sqrt(ss[max(0, j - hw):j + hw + 1].sum()) for j in range(fm.shape[0])])
        with np.errstate(invalid="ignore", divide="ignore"):
            out = fm / nrm.reshape((-1,) + (1,) * (fm.ndim - 1))
        out = np.where(np.isfinite(out), out, 0.0)
        return np.moveaxis(out, 0, axis)
    if op == MEDIAN:
        h = [int(round(param[a])) for a in range(3)]
        out = np.empty_like(f)
        for idx in np.ndindex(*f.shape):
            sl = []
            for d, i in enumerate(idx):
                hh = h[f.ndim - 1 - d] if f.shape[d] > 1 else 0
                sl.append(slice(max(0, i - hh), min(f.shape[d], i + hh + 1)))
            w = np.sort(f[tuple(sl)].ravel())
            c = w.size
            out[idx] = w[c // 2] if c % 2 else 0.5 * (w[c // 2 - 1] + w[c // 2])
        return out
    raise ValueError(op)
