"""Oracle (test infrastructure only): FP64 restatement of the trace resampling
of resample_su (src/lib/module_su.f90:426-470), used after modelling when the
data sampling differs from the time axis (submodule_forward_modeling.f90:124-125)
and on the adjoint source before injection (submodule_fwi_gradient.f90:46).

The reference calls FLIT's interp(..., 'cubic'); FLIT (github.com/lanl/flit, no
version pinned) is not vendored and no reference test pins it -- parity
unpinned. Restated as cubic convolution (Keys 1981, a = -1/2): output sample i
at t = oout + i dout reads the four input samples j0-1 .. j0+2 around
x = (t - oin) / din with indices clamped to the row (x within 1e-4 of a node
snaps to it, since the sampling intervals are single precision), and is zero
outside [0, nin - 1].
"""
from __future__ import annotations

import numpy as np


def keys_weights(u):
    u2, u3 = u * u, u * u * u
    return (0.5 * (-u3 + 2 * u2 - u), 0.5 * (3 * u3 - 5 * u2 + 2), 0.5 * (-3 * u3 + 4 * u2 + u), 0.5 * (u3 - u2))


def resample_rows(rows, din, dout, nout, oin=0.0, oout=0.0):
    rows = np.atleast_2d(np.asarray(rows, dtype=np.float64))
    ntr, nin = rows.shape
    out = np.zeros((ntr, nout))
    for i in range(nout):
        x = (oout + i * dout - oin) / din
        if abs(x - np.rint(x)) <= 1e-4:
            x = float(np.rint(x))
        if x < 0 or x > nin - 1:
            continue
        j0 = int(np.floor(x))
        w = keys_weights(x - j0)
        idx = (max(j0 - 1, 0), j0, min(j0 + 1, nin - 1), min(j0 + 2, nin - 1))
        out[:, i] = sum(wk * rows[:, jk] for wk, jk in zip(w, idx))
    return out
