"""GPU search directions and gradient processing against the FP64 oracle, and a
three-iteration L-BFGS FWI loop that stays on the device (gradient, smoothing,
search direction, step by backtracking on misfit-only forwards)."""
import numpy as np
import pytest
import torch

import oracle
import oracle.oracle_optim as O
from owl_b200 import _lib as L
from owl_b200.optim import process, search_direction
from owl_b200.solver import RunOpts

from cases import desc, prepare, random_model, rel, small_shots
from test_gpu_ac2d import make_solver

pytestmark = pytest.mark.gpu


def _history(n, nm, seed=0):
    rng = np.random.default_rng(seed)
    x = [rng.standard_normal(n).astype(np.float32)]
    g = [rng.standard_normal(n).astype(np.float32)]
    for _ in range(nm - 1):
        x.append((x[-1] - 0.1 * g[-1] + 0.01 * rng.standard_normal(n)).astype(np.float32))
        g.append((0.8 * g[-1] + 0.2 * rng.standard_normal(n)).astype(np.float32))
    return x, g


@pytest.mark.parametrize("method", [L.OWL_SEARCH_SD, L.OWL_SEARCH_CG, L.OWL_SEARCH_LBFGS])
@pytest.mark.parametrize("nm", [1, 3, 11])
def test_search_direction_matches_oracle(method, nm):
    n = 200_003
    x, g = _history(n, nm, seed=nm)
    prev = np.random.default_rng(9).standard_normal(n).astype(np.float32)
    ref = O.search_direction(method, x, g, prev)
    got = search_direction(method, x, g, prev)
    assert rel(got, ref) < 1e-5, rel(got, ref)
    dev = search_direction(method, [torch.from_numpy(a).cuda() for a in x], [torch.from_numpy(a).cuda() for a in g],
                           torch.from_numpy(prev).cuda())
    assert np.array_equal(dev.cpu().numpy(), got)


@pytest.mark.parametrize("shape", [(40, 57), (13, 11, 17)])
def test_processing_matches_oracle(shape):
    rng = np.random.default_rng(4)
    f = rng.standard_normal(shape).astype(np.float32)
    m = (rng.random(shape) > 0.3).astype(np.float32)
    # the oracle takes the field with the fastest (z) axis last
    to_o = lambda a: np.ascontiguousarray(np.transpose(a))  # noqa: E731
    for op, par in ((L.OWL_GRAD_SMOOTH, [1.5, 2.5, 1.0]), (L.OWL_GRAD_TAPER, [3, 4, 5, 2, 2, 3]),
                    (L.OWL_GRAD_MASK, None), (L.OWL_GRAD_SCALE, [2.5]), (L.OWL_GRAD_MAX_BALANCE, None),
                    (L.OWL_GRAD_RMS_BALANCE, None), (L.OWL_GRAD_RMS_BALANCE_AXIS, [1, 5]),
                    (L.OWL_GRAD_RMS_BALANCE_AXIS, [2, 4]), (L.OWL_GRAD_RMS_BALANCE_AXIS, [len(shape), 1]),
                    (L.OWL_GRAD_MEDIAN, [1, 1, 1]), (L.OWL_GRAD_MEDIAN, [2, 1, 0])):
        got = process(f.copy(), op, par, m if op == L.OWL_GRAD_MASK else None)
        ref = np.transpose(O.process(op, to_o(f), par, to_o(m)))
        assert rel(got, ref) < 1e-6, (op, rel(got, ref))


def test_lbfgs_fwi_loop_on_the_device():
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 240
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = torch.from_numpy(oracle.ac2d_forward(d, vp, rho, ps, "f64").astype(np.float32)).cuda()
    vp0 = (vp * np.float32(1.02)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    opts = RunOpts(checkpoint_interval=30)
    nm = nx * nz
    m = torch.from_numpy(np.asfortranarray(vp0).ravel(order="F")).cuda()  # z fastest, like the gradient
    models, grads, misfits = [], [], []
    for _ in range(3):
        s.set_model(m.cpu().numpy().reshape(nx, nz).T, rho)
        mf, g = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, opts)
        gv = g[:nm].clone()
        process(gv.view(nx, nz).T, L.OWL_GRAD_SMOOTH, [1.0, 1.0, 0.0])
        models.append(m.clone())
        grads.append(gv)
        misfits.append(float(mf.sum()))
        srch = search_direction(L.OWL_SEARCH_LBFGS, models[-4:], grads[-4:])
        step = 20.0 / float(srch.abs().max())
        for _ in range(8):  # backtracking on the misfit-only forward
            trial = m + step * srch
            s.set_model(trial.cpu().numpy().reshape(nx, nz).T, rho)
            if float(s.misfit(ps, obs.cpu().numpy()).sum()) < misfits[-1]:
                break
            step *= 0.5
        m = trial
    s.set_model(m.cpu().numpy().reshape(nx, nz).T, rho)
    final = float(s.misfit(ps, obs.cpu().numpy()).sum())
    assert misfits[1] < misfits[0] and misfits[2] < misfits[1] and final < misfits[2], (misfits, final)
