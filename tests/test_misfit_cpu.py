"""The misfit oracle (oracle/oracle_misfit.py) on the CPU.

The reference ships no fixtures for its misfits, so the restatement is pinned by
its own mathematics: for the waveform, correlation and envelope misfits the
adjoint source is the gradient of half the trace misfit (the envelope's in the
limit of its stabiliser), for the adaptive misfit the gradient of the misfit
itself away from the first taper ramp (the reference tapers the adjoint at the
end only); central differences in FP64 check each. The phase adjoint is the
reference's formula; the test records that the exact gradient of half the
phase misfit has the opposite sign on its Hilbert term.
"""
import numpy as np
import pytest

import oracle.oracle_misfit as M


def _traces(n=96, seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(n)

    def sig(shift, amp):
        return amp * np.exp(-((t - 40 - shift) / 6.0) ** 2) * np.cos(0.55 * (t - shift)) + 0.01 * rng.standard_normal(n)

    return sig(0.0, 1.0), sig(2.5, 0.8)


def _fd(f, x, h=1e-6):
    g = np.zeros_like(x)
    for i in range(x.size):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        g[i] = (f(xp) - f(xm)) / (2 * h)
    return g


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_next_power_235():
    got = [M.next_power_235(n) for n in (1, 7, 11, 13, 17, 49, 97, 4000, 4001, 8191)]
    assert got == [1, 8, 12, 15, 18, 50, 100, 4000, 4050, 8192]


@pytest.mark.parametrize("name", ["waveform", "corr", "envelope"])
def test_adjoint_is_gradient_of_half_misfit(name):
    obs, syn = _traces()
    fn = {"waveform": M.waveform, "corr": M.corr, "envelope": lambda o, s: M.envelope_misfit(o, s, stab=0.0)}[name]
    _, adj = fn(obs, syn)
    g = _fd(lambda s: 0.5 * fn(obs, s)[0], syn)
    assert _rel(adj, g) < 1e-7


def test_adaptive_adjoint_is_gradient_inside_the_ramps():
    obs, syn = _traces(200)
    n = obs.size
    tl = int(np.floor(0.025 * n + 0.5))
    for pen in (M.LINEAR, M.POWER, M.GAUSSIAN, M.EXP):
        _, adj = M.adaptive(obs, syn, 1e-3, 0.03, pen, 2.0)
        g = _fd(lambda s: M.adaptive(obs, s, 1e-3, 0.03, pen, 2.0)[0], syn)
        sl = slice(tl, n - tl)
        assert _rel(adj[sl], g[sl]) < 1e-6, pen


def test_adaptive_grows_with_the_time_shift():
    """the matching filter's energy moves to larger (penalised) lags as the shift grows"""
    n = 200
    t = np.arange(n)
    obs = np.exp(-((t - 90) / 6.0) ** 2) * np.cos(0.55 * (t - 90))
    ms = [M.adaptive(obs, np.exp(-((t - 90 - k) / 6.0) ** 2) * np.cos(0.55 * (t - 90 - k)), 1e-3, 0.05)[0]
          for k in (0, 3, 6, 12)]
    assert all(a < b for a, b in zip(ms, ms[1:])), ms


def test_phase_adjoint_sign_of_the_hilbert_term():
    obs, syn = _traces()
    _, adj = M.phase_misfit(obs, syn, stab=0.0)
    g = _fd(lambda s: 0.5 * M.phase_misfit(obs, s, stab=0.0)[0], syn)
    zu, zd = M.analytic(syn), M.analytic(obs)
    dphi = np.arctan2(zu.imag, zu.real) - np.arctan2(zd.imag, zd.real)
    env = np.abs(zu) ** 2
    exact = -dphi * zu.imag / env - M.hilbert(dphi * syn / env)
    assert _rel(exact, g) < 1e-6
    assert np.allclose(adj, -dphi * zu.imag / env + M.hilbert(dphi * syn / env))


def test_hilbert_of_cosine_is_sine():
    n = 128
    t = np.arange(n)
    x = np.cos(2 * np.pi * 5 * t / n)
    assert np.allclose(M.hilbert(x), np.sin(2 * np.pi * 5 * t / n), atol=1e-12)
    assert np.allclose(M.envelope(x), 1.0, atol=1e-12)


def test_discard_rule():
    obs, syn = _traces()
    rows_o = np.stack([obs, obs, 1e-9 * obs, obs])
    rows_s = np.stack([syn, syn, syn, 0 * syn])
    w = np.array([1.0, 0.0, 1.0, 1.0])
    adj, tm, gm = M.adjoint_source(M.WAVEFORM, [0, 4], rows_s, rows_o, w)
    assert tm[0] > 0 and np.all(tm[1:] == 0) and np.all(adj[1:] == 0)
    assert gm[0] == tm.sum()
    # a negative threshold keeps the tiny trace, not the zero one
    _, tm2, _ = M.adjoint_source(M.WAVEFORM, [0, 4], rows_s, rows_o, w, discard_threshold=-1.0)
    assert tm2[2] > 0 and tm2[3] == 0


def test_resample_oracle_properties():
    """cubic convolution: identity on the same sampling, exact for quadratics
    away from the ends, linear in the data"""
    import oracle.oracle_resample as R
    rng = np.random.default_rng(1)
    x = rng.standard_normal((3, 50))
    assert np.allclose(R.resample_rows(x, 1e-3, 1e-3, 50), x, atol=0)
    t_in = np.arange(50) * 2e-3
    q = 1.0 + 3.0 * t_in - 40.0 * t_in ** 2
    t_out = np.arange(120) * 0.7e-3
    got = R.resample_rows(q, 2e-3, 0.7e-3, 120)[0]
    inner = (t_out >= 2e-3) & (t_out <= 47 * 2e-3)
    assert np.allclose(got[inner], (1.0 + 3.0 * t_out - 40.0 * t_out ** 2)[inner], atol=1e-12)
    y = rng.standard_normal((3, 50))
    a = R.resample_rows(2 * x - y, 1e-3, 2.5e-3, 20)
    assert np.allclose(a, 2 * R.resample_rows(x, 1e-3, 2.5e-3, 20) - R.resample_rows(y, 1e-3, 2.5e-3, 20))
    assert np.all(R.resample_rows(x, 1e-3, 1e-3, 60)[:, 50:] == 0)


def test_local_and_spacetime_adaptive_properties():
    """the local adaptive misfit of a trace with itself (not zero: the water
    level spreads the matching filter) is well below that of a shifted copy;
    the space-time misfit of a trace flanked by copies of itself equals that of
    the trace alone"""
    import oracle.oracle_misfit as M
    n, dt = 256, 2e-3
    t = np.arange(n) * dt
    a = (np.pi * 12.0 * (t - 0.25)) ** 2
    syn = (1 - 2 * a) * np.exp(-a)
    a2 = (np.pi * 12.0 * (t - 0.27)) ** 2
    obs = (1 - 2 * a2) * np.exp(-a2)
    m0, _ = M.local_adaptive(syn, syn, dt, 0.08)
    m1, adj1 = M.local_adaptive(obs, syn, dt, 0.08)
    assert m0 < 0.5 * m1 and np.all(np.isfinite(adj1))
    s1, a1 = M.adaptive_spacetime(obs[None], syn[None], 0, dt, 0.08)
    s3, a3 = M.adaptive_spacetime(np.stack([obs, obs, obs]), np.stack([syn, syn, syn]), 1, dt, 0.08)
    assert s3 == pytest.approx(s1, rel=1e-10) and np.allclose(a3, a1, rtol=1e-9, atol=1e-12)
