"""The SSG solver as a differentiable PyTorch operator.

``SSGForward`` is a ``torch.autograd.Function``: its forward runs the batched
CUDA forward (``owl_ssg_forward``) of all shots and returns the seismograms as
one flat CUDA tensor, shot after shot, each ``(ncomp, nrec, nt)``; its backward
takes the incoming seismogram gradient as the adjoint source
(``OWL_ADJ_GIVEN``) and runs the hand-written adjoint kernels
(``owl_ssg_gradient``: forward with checkpoints, segment recompute, exact
discrete adjoint, Kahan FP32 imaging sums, FP64 chain rule), which return
d<seis, adj>/d(model) for every model parameter. That is the vector-Jacobian
product autograd asks for, so any loss written in torch on the seismograms
(the reference's L2 waveform misfit, ``compute_adjsrc_waveform`` in
src/inverse/module_inversion_adjoint_source.f90:371-383, or any other)
differentiates through the solver.

The model parameters are the arrays of ``owl_ssg_set_model`` in its order
(acoustic: vp, rho; elastic: per anisotropy type), each shaped ``(nz, nx)`` or
``(nz, ny, nx)`` like OWL's model files; their gradients come back in the same
shape. The forward state is not kept between forward and backward: backward
recomputes it from checkpoints inside the gradient call (one extra forward
sweep), so the memory held between the two passes is the seismogram only.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .geometry import PreparedShots
from .solver import RunOpts, SSGSolver


def _model_shape(solver: SSGSolver):
    d = solver.desc
    return (d.nz, d.nx) if d.ny <= 1 else (d.nz, d.ny, d.nx)


def _upload(solver: SSGSolver, params: Sequence[torch.Tensor]) -> None:
    shape = _model_shape(solver)
    if len(params) != solver.nparam:
        raise ValueError(f"this medium takes {solver.nparam} model arrays, got {len(params)}")
    host = []
    for p in params:
        if tuple(p.shape) != shape:
            raise ValueError(f"model array of shape {tuple(p.shape)}, expected {shape}")
        host.append(p.detach().to("cpu", torch.float32).numpy())
    solver.set_model(*host)


def _unflatten(solver: SSGSolver, g: torch.Tensor):
    """flat (nparam * ncell) gradient, z fastest -> list of (nz, nx) / (nz, ny, nx) tensors"""
    shape = _model_shape(solver)
    nm = int(np.prod(shape))
    out = []
    for i in range(solver.nparam):
        gi = g[i * nm:(i + 1) * nm].view(tuple(reversed(shape)))
        out.append(gi.permute(*reversed(range(len(shape)))))
    return out


class SSGForward(torch.autograd.Function):
    """seis = F(model); backward = adjoint-state gradient of <seis, grad_seis>."""

    @staticmethod
    def forward(ctx, solver: SSGSolver, ps: PreparedShots, opts: Optional[RunOpts], *params: torch.Tensor):
        if not torch.cuda.is_available():
            raise RuntimeError("owl_b200: the SSG operator runs on CUDA only; no CUDA device is visible")
        device = next((p.device for p in params if p.is_cuda), torch.device("cuda"))
        _upload(solver, params)
        seis = torch.empty(solver.seis_size(ps), dtype=torch.float32, device=device)
        solver.forward(ps, opts, out=seis)
        ctx.solver, ctx.ps, ctx.opts = solver, ps, opts
        ctx.save_for_backward(*params)
        return seis

    @staticmethod
    def backward(ctx, gseis: torch.Tensor):
        solver, ps, opts = ctx.solver, ctx.ps, ctx.opts
        params = ctx.saved_tensors
        # another call on the same handle may have replaced the model in between
        _upload(solver, params)
        adj = gseis.detach().to(torch.float32).contiguous()
        if not adj.is_cuda:
            adj = adj.cuda()
        _, g = solver.gradient(ps, adj, L.OWL_ADJ_GIVEN, opts)
        grads = [gi.to(p.device, p.dtype) if ctx.needs_input_grad[3 + i] else None
                 for i, (gi, p) in enumerate(zip(_unflatten(solver, g), params))]
        return (None, None, None, *grads)


def ssg_forward(solver: SSGSolver, ps: PreparedShots, *params: torch.Tensor,
                opts: Optional[RunOpts] = None) -> torch.Tensor:
    """Differentiable seismograms of all shots of ``ps`` for the model ``params``."""
    return SSGForward.apply(solver, ps, opts, *params)


def split_seismograms(solver: SSGSolver, ps: PreparedShots, seis: torch.Tensor):
    """flat seismogram tensor -> per-shot (ncomp, nrec, nt) views"""
    return solver.split(ps, seis)
