"""CPU tests of the step-length helpers (compute_step_coef restated)."""
import numpy as np
import pytest

from owl_b200.step import step_scaling_factor, step_sums, trace_weights


def test_step_factor_of_a_linear_update():
    # syn - prev = a (obs - prev) on every trace: err_23 = a^2 err_13, so
    # sum(err_23 err_13) / sum(err_23^2) = 1 / a^2
    rng = np.random.default_rng(0)
    prev = rng.standard_normal((5, 50))
    obs = prev + rng.standard_normal((5, 50))
    syn = prev + 0.5 * (obs - prev)
    s1, s2 = step_sums(obs, syn, prev, np.ones(5))
    assert step_scaling_factor(s1, s2) == pytest.approx(4.0, rel=1e-12)


def test_trace_discard_rule():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((6, 40))
    w = np.ones(6)
    w[2] = 0
    b = a.copy()
    b[4] *= 1e-3  # far below the median norm
    keep = trace_weights(a, b, a, w, threshold=0.1)
    assert keep.tolist() == [1, 1, 0, 1, 0, 1]
    z = a.copy()
    z[5] = 0
    assert trace_weights(a, z, a, np.ones(6))[5] == 0
