"""The search-direction and gradient-processing oracle (oracle/oracle_optim.py)
on the CPU: L-BFGS with full memory and exact line searches minimises an
n-dimensional quadratic in n steps; CG reduces to steepest descent when the
Polak-Ribiere beta is clipped at 0; the Gaussian smoothing keeps a constant
field and the mean of a periodic-free interior; the taper leaves the interior."""
import numpy as np

import oracle.oracle_optim as O


def _quadratic(n=8, seed=0):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    a = q @ np.diag(np.linspace(1.0, 30.0, n)) @ q.T
    b = rng.standard_normal(n)
    return a, b


def test_lbfgs_minimises_a_quadratic_in_n_steps():
    a, b = _quadratic()
    x = [np.zeros(8)]
    g = [a @ x[0] - b]
    for _ in range(8):
        d = O.search_direction(O.LBFGS, x, g)
        step = -float(g[-1] @ d) / float(d @ a @ d)  # exact line search
        x.append(x[-1] + step * d)
        g.append(a @ x[-1] - b)
    assert np.linalg.norm(g[-1]) < 1e-8 * np.linalg.norm(g[0])
    assert np.allclose(x[-1], np.linalg.solve(a, b), atol=1e-8)


def test_cg_and_sd():
    a, b = _quadratic(seed=1)
    g0 = a @ np.zeros(8) - b
    assert np.allclose(O.search_direction(O.SD, [np.zeros(8)], [g0]), -g0)
    g1 = 0.5 * g0
    # g1.(g1 - g0) < 0: beta clips to 0, steepest descent
    assert np.allclose(O.search_direction(O.CG, [0, 0], [g0, g1], prev_srch=-g0), -g1)


def test_processing_properties():
    f = np.ones((12, 30, 5))
    assert np.allclose(O.process(O.SMOOTH, f, [2.0, 3.0, 1.0]), 1.0)
    rng = np.random.default_rng(3)
    g = rng.standard_normal((40, 50))
    t = O.process(O.TAPER, g, [5, 5, 7, 7, 0, 0])
    assert np.array_equal(t[7:-7, 5:-5], g[7:-7, 5:-5])
    assert np.allclose(t[:, 0], 0, atol=1e-12) and np.allclose(t[0, :], 0, atol=1e-12)
    assert np.isclose(O.process(O.MAX_BALANCE, g).max(), 1.0)


def test_balance_and_median_properties():
    """rms_balance leaves unit root mean square; the windowed balance of a
    field constant along its axis is the field over sqrt(window slices);
    the median of a field with one spike removes it"""
    rng = np.random.default_rng(2)
    f = rng.standard_normal((9, 12))
    g = O.process(O.RMS_BALANCE, f)
    assert abs(np.sqrt(np.mean(g * g)) - 1.0) < 1e-12
    c = np.ones((7, 10))  # axis 1 (n1, the last numpy axis) has 10 slices of 7 ones
    b = O.process(O.RMS_BALANCE_AXIS, c, [1, 3])
    assert np.allclose(b[:, 1:-1], 1.0 / np.sqrt(21.0)) and np.allclose(b[:, 0], 1.0 / np.sqrt(14.0))
    sp = np.zeros((5, 6))
    sp[2, 3] = 100.0
    assert np.all(O.process(O.MEDIAN, sp, [1, 1, 0]) == 0.0)
