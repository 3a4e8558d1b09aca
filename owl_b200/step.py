"""Step-length helpers of the FWI loop around the misfit-only forward.

The reference scales its search step by a linearised estimate from three sets
of seismograms of a shot: the observed data (1), the synthetics of the current
trial model (2) and those of the previous model (3) (compute_step_coef,
src/inverse/module_inversion_step_size.f90:263-560, and
compute_step_size:627-690). Per trace, err_23 and err_13 are the waveform
misfits sum_t (a - b)^2 of (2, 3) and (1, 3); traces with weight 0, a zero
norm, or a norm below trace_discard_threshold times the median norm of their
gather are left out; the step scaling factor is sum(err_23 err_13) /
(sum(err_23^2) + tiny). The trial synthetics and err_23 come from
SSGSolver.misfit (one batched forward, no checkpoints).
"""
from __future__ import annotations

import numpy as np

FLOAT_TINY = float(np.finfo(np.float32).tiny)


def trace_weights(obs, syn, syn_prev, weight, threshold: float = 0.0):
    """0 / 1 per trace (traces x nt arrays): the discard rule of compute_step_coef (:341-357)."""
    n_obs, n_syn, n_prev = (np.linalg.norm(np.asarray(a, dtype=np.float64), axis=1) for a in (obs, syn, syn_prev))
    m_obs, m_syn, m_prev = np.median(n_obs), np.median(n_syn), np.median(n_prev)
    keep = (np.asarray(weight) != 0) & (n_obs >= threshold * m_obs) & (n_syn >= threshold * m_syn) & \
        (n_prev >= threshold * m_prev) & (n_obs * n_syn * n_prev != 0)
    return keep.astype(np.float64)


def step_sums(obs, syn, syn_prev, weight, threshold: float = 0.0):
    """(sum1, sum2) of one shot and component for the waveform misfit."""
    obs, syn, prev = (np.asarray(a, dtype=np.float64) for a in (obs, syn, syn_prev))
    w = trace_weights(obs, syn, prev, weight, threshold)
    err23 = np.sum((syn - prev) ** 2, axis=1) * w
    err13 = np.sum((obs - prev) ** 2, axis=1) * w
    return float(np.sum(err23 * err13)), float(np.sum(err23 ** 2))


def step_scaling_factor(sum1: float, sum2: float) -> float:
    """module_inversion_step_size.f90:681"""
    return sum1 / (sum2 + FLOAT_TINY)
