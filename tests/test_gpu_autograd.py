"""The SSG solver behind torch.autograd (owl_b200.autograd.SSGForward).

* backward of the L2 waveform misfit written in torch equals the library's own
  L2-residual gradient, and both sit within 1e-4 of the FP64 exact-adjoint
  oracle;
* for a loss that is not the L2 misfit (a weighted sum of the seismograms),
  <grad, dm> matches a central finite difference of the FP64 oracle forward;
* the elastic 2D Thomsen parameterisation differentiates the same way.
"""
import numpy as np
import pytest
import torch

import oracle
from owl_b200 import _lib as L
from owl_b200.autograd import ssg_forward
from owl_b200.solver import RunOpts

from cases import desc, prepare, random_model, rel, small_shots
from test_gpu_ac2d import make_solver
from test_gpu_el2d import make as make_el
from test_oracle_el2d import el_desc, el_model, el_shots

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda", requires_grad=True)


def test_autograd_l2_matches_library_and_oracle():
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 240
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp, rho, ps, "f64").astype(np.float32)
    vp0 = (vp * np.float32(1.03)).astype(np.float32)
    s = make_solver(d, vp0, rho)
    opts = RunOpts(checkpoint_interval=30)

    tvp, trho = _t(vp0), _t(rho)
    seis = ssg_forward(s, ps, tvp, trho, opts=opts)
    loss = 0.5 * ((seis.double() - torch.from_numpy(obs).cuda().double()) ** 2).sum()
    loss.backward()

    mf, g = s.gradient(ps, obs, L.OWL_ADJ_L2_RESIDUAL, opts)
    g_vp, g_rho = s.grad_fields(g)
    assert tvp.grad.shape == (nz, nx) and trho.grad.shape == (nz, nx)
    assert rel(tvp.grad.cpu().numpy(), g_vp) < 1e-5
    assert rel(trho.grad.cpu().numpy(), g_rho) < 1e-5
    # the library's misfit is the reference's sum of squared residuals (no 1/2)
    assert abs(2 * loss.item() - mf.sum()) <= 1e-5 * mf.sum()

    _, g_ref, _ = oracle.ac2d_gradient(d, vp0, rho, ps, obs, adj_kind=0, k=30, precision="f64")
    got = np.concatenate([tvp.grad.cpu().numpy().T.ravel(), trho.grad.cpu().numpy().T.ravel()])
    assert rel(got, g_ref) < 1e-4, rel(got, g_ref)


def test_autograd_weighted_sum_vs_finite_difference():
    """loss = <w, seis(m)>, linear in the seismograms; directional derivative
    along a smooth dm against a central difference of the FP64 oracle forward."""
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 200
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    s = make_solver(d, vp, rho)
    rng = np.random.default_rng(5)
    w = rng.standard_normal(s.seis_size(ps)).astype(np.float32)
    tvp, trho = _t(vp), _t(rho)
    seis = ssg_forward(s, ps, tvp, trho, opts=RunOpts(checkpoint_interval=25))
    (seis * torch.from_numpy(w).cuda()).sum().backward()

    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    dm = np.exp(-((zz - 22.0) ** 2 + (xx - 25.0) ** 2) / 30.0)
    h = 1e-3 * float(vp.mean())
    fp = oracle.ac2d_forward(d, vp.astype(np.float64) + h * dm, rho, ps, "f64")
    fm = oracle.ac2d_forward(d, vp.astype(np.float64) - h * dm, rho, ps, "f64")
    fd = float(np.dot(w.astype(np.float64), (fp - fm) / (2 * h)))
    ad = float((tvp.grad.double().cpu().numpy() * dm).sum())
    assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)


def test_autograd_elastic_thomsen():
    d = el_desc(1, L.OWL_ANISO_THOMSEN)
    f = el_model(L.OWL_ANISO_THOMSEN)
    s = make_el(d, f)
    ps = s.prepare(el_shots(1))
    obs = oracle.el2d_forward(d, el_model(L.OWL_ANISO_THOMSEN, seed=2), ps, "f64").astype(np.float32)
    opts = RunOpts(checkpoint_interval=7)
    params = [_t(a) for a in f]
    seis = ssg_forward(s, ps, *params, opts=opts)
    (0.5 * ((seis - torch.from_numpy(obs).cuda()) ** 2).sum()).backward()
    _, g = s.gradient(ps, obs, opts=opts)
    for p, gq in zip(params, s.grad_fields(g)):
        assert rel(p.grad.cpu().numpy(), gq) < 1e-5


def test_autograd_rejects_wrong_model_shape():
    nx, nz, dx, dt, nt = 48, 40, 10.0, 1e-3, 50
    d = desc(nx, nz, dx, dt, nt)
    vp, rho = random_model(nx, nz)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    s = make_solver(d, vp, rho)
    with pytest.raises(ValueError):
        ssg_forward(s, ps, _t(vp.T), _t(rho.T))
