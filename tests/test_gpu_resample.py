"""Data sampling off the time axis (owl_ssg_set_data_sampling,
owl_resample_traces) against the FP64 oracles: the synthetics resampled after
modelling, the misfit computed at the data sampling and the adjoint source
resampled back to the time axis, as the reference orders it."""
import numpy as np
import pytest

import oracle
import oracle.oracle_misfit as M
import oracle.oracle_resample as R
from owl_b200 import _lib as L
from owl_b200.solver import MisfitOpts, RunOpts, resample_traces

from cases import desc, prepare, random_model, rel, small_shots
from test_gpu_ac2d import make_solver

pytestmark = pytest.mark.gpu

NX, NZ, DX, DT, NT = 48, 40, 10.0, 1e-3, 241
DDT = 2.5e-3
DNT = int(round((NT - 1) * DT / DDT)) + 1


def test_resample_traces_matches_oracle():
    import torch
    rng = np.random.default_rng(2)
    x = rng.standard_normal((37, 301)).astype(np.float32)
    for din, dout, nout, oin, oout in ((1e-3, 2.5e-3, 121, 0.0, 0.0), (4e-3, 1e-3, 1210, 0.0, 0.0),
                                       (1e-3, 0.7e-3, 500, 0.01, -0.02)):
        got = resample_traces(x, din, dout, nout, oin, oout)
        f = lambda v: float(np.float32(v))  # noqa: E731  (the ABI takes single-precision times)
        ref = R.resample_rows(x, f(din), f(dout), nout, f(oin), f(oout))
        assert rel(got, ref) < 1e-6, (din, dout)
        dev = resample_traces(torch.from_numpy(x).cuda(), din, dout, nout, oin, oout)
        assert np.array_equal(dev.cpu().numpy(), got)


def _setup():
    d = desc(NX, NZ, DX, DT, NT)
    vp, rho = random_model(NX, NZ)
    ps = prepare(small_shots(NX, NZ, DX), NX, NZ, DX, DT)
    return d, vp, rho, ps


def test_forward_at_data_sampling():
    d, vp, rho, ps = _setup()
    s = make_solver(d, vp, rho)
    s.set_data_sampling(DNT, DDT)
    got = s.forward(ps)
    assert got.size == s.seis_size(ps) == sum(ps.nrec(i) for i in range(ps.nshots)) * DNT
    ref = R.resample_rows(oracle.ac2d_forward(d, vp, rho, ps, "f32").reshape(-1, NT), DT, DDT, DNT).ravel()
    assert rel(got, ref) < 1e-5
    s.set_data_sampling(0, 0.0)
    assert s.forward(ps).size == sum(ps.nrec(i) for i in range(ps.nshots)) * NT


@pytest.mark.parametrize("kind", ["l2", "given", L.OWL_MISFIT_ENVELOPE])
def test_gradient_at_data_sampling(kind):
    d, vp, rho, ps = _setup()
    obs = R.resample_rows(oracle.ac2d_forward(d, vp, rho, ps, "f64").reshape(-1, NT), DT, DDT, DNT)
    obs = obs.astype(np.float32)
    vp0 = (vp * np.float32(1.03)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    s.set_data_sampling(DNT, DDT)
    opts = RunOpts(checkpoint_interval=30)
    syn_d = R.resample_rows(oracle.ac2d_forward(d, vp0, rho, ps, "f64").reshape(-1, NT), DT, DDT, DNT)
    live = np.concatenate([[r.weight != 0 for r in sh.receivers] for sh in ps.shots])
    if kind == "l2":
        mf, g = s.gradient(ps, obs.ravel(), L.OWL_ADJ_L2_RESIDUAL, opts)
        adj_d = (syn_d - obs) * live[:, None]
        mref = [((obs - syn_d)[a:b] ** 2 * live[a:b, None]).sum() for a, b in
                zip(s.gather_ptr(ps)[:-1], s.gather_ptr(ps)[1:])]
        assert rel(mf, np.array(mref)) < 1e-4
    elif kind == "given":
        rng = np.random.default_rng(4)
        adj_d = (rng.standard_normal(obs.shape) * live[:, None]).astype(np.float32)
        _, g = s.gradient(ps, adj_d.ravel(), L.OWL_ADJ_GIVEN, opts)
    else:
        mf, g = s.gradient_misfit(ps, obs.ravel(), MisfitOpts(misfit=kind), opts)
        # the misfit is taken on the traces resampled to the time axis' NT samples (adj_nt's default)
        adj_d, _, gm = M.adjoint_source(kind, s.gather_ptr(ps), syn_d, obs, live.astype(np.float64), dt=DDT,
                                        adj_nt=NT)
        assert rel(mf, gm) < 2e-4
    adj_t = R.resample_rows(adj_d, DDT, DT, NT).astype(np.float32)
    _, g_ref, _ = oracle.ac2d_gradient(d, vp0, rho, ps, adj_t.ravel(), adj_kind=1, k=30, precision="f64")
    assert rel(g, g_ref) < 2e-4, rel(g, g_ref)


def test_misfit_at_data_sampling():
    d, vp, rho, ps = _setup()
    obs = R.resample_rows(oracle.ac2d_forward(d, vp, rho, ps, "f64").reshape(-1, NT), DT, DDT, DNT).astype(np.float32)
    vp0 = (vp * np.float32(1.02)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    s.set_data_sampling(DNT, DDT)
    seis = np.zeros(s.seis_size(ps), dtype=np.float32)
    mf, tm = s.misfit(ps, obs.ravel(), traces=True, seis_out=seis)
    syn_d = R.resample_rows(oracle.ac2d_forward(d, vp0, rho, ps, "f64").reshape(-1, NT), DT, DDT, DNT)
    live = np.concatenate([[r.weight != 0 for r in sh.receivers] for sh in ps.shots])
    ref_tm = ((obs - syn_d) ** 2).sum(axis=1) * live
    assert rel(tm, ref_tm) < 1e-4
    assert rel(seis, syn_d.ravel()) < 1e-5


def test_su_records_on_the_device(tmp_path):
    """owl_su_encode / owl_su_decode give the bytes and traces of the host SU writer / reader"""
    import torch

    from owl_b200 import io
    rng = np.random.default_rng(6)
    x = rng.standard_normal((23, 777)).astype(np.float32)
    io.write_su(str(tmp_path / "host.su"), x, 2.5e-3)
    io.write_su_device(str(tmp_path / "dev.su"), torch.from_numpy(x).cuda(), 2.5e-3)
    assert (tmp_path / "host.su").read_bytes() == (tmp_path / "dev.su").read_bytes()
    y, dt = io.read_su_device(str(tmp_path / "host.su"))
    assert np.array_equal(y.cpu().numpy(), x) and abs(dt - 2.5e-3) < 1e-9
