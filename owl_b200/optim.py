"""Search directions and gradient processing on the GPU (owl_search_direction,
owl_grad_process): compute_search_direction
(src/inverse/module_inversion_search_direction.f90) and
process_model_single_parameter (src/inverse/2d/module_gradient.f90:733-892)
for fields held as numpy arrays (host) or CUDA tensors (device)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from .solver import _mem_kind, _ptr, _ready


def search_direction(method: int, models: Sequence, grads: Sequence, prev_srch=None, out=None):
    """models / grads oldest first, the last entry the current iteration"""
    lib = L.load()
    nm = len(grads)
    if len(models) != nm or nm < 1:
        raise ValueError("models and grads must have the same (non-zero) length")
    g0 = grads[-1]
    dev = _mem_kind(g0) == L.OWL_MEM_DEVICE
    if dev:
        import torch
        models = [m.contiguous() for m in models]
        grads = [g.contiguous() for g in grads]
        out = torch.empty_like(grads[-1]) if out is None else out
    else:
        models = [np.ascontiguousarray(m, dtype=np.float32) for m in models]
        grads = [np.ascontiguousarray(g, dtype=np.float32) for g in grads]
        prev_srch = None if prev_srch is None else np.ascontiguousarray(prev_srch, dtype=np.float32)
        out = np.empty_like(grads[-1]) if out is None else out
    _ready(*models, *grads, prev_srch, out)
    xs = (C.c_void_p * nm)(*[_ptr(m).value for m in models])
    gs = (C.c_void_p * nm)(*[_ptr(g).value for g in grads])
    n = int(np.prod(out.shape))
    L.check(lib.owl_search_direction(method, n, nm, xs, gs, _ptr(prev_srch) if prev_srch is not None else None,
                                     _ptr(out), L.OWL_MEM_DEVICE if dev else L.OWL_MEM_HOST))
    return out


def process(field, op: int, param: Optional[Sequence[float]] = None, mask=None):
    """In-place processing of a (nz, nx) / (nz, ny, nx) field stored z fastest
    (a numpy array in Fortran order or the flat z-fastest buffer), returned."""
    lib = L.load()
    shape = tuple(field.shape)
    if len(shape) == 1:
        raise ValueError("pass the field with its (nz, nx) or (nz, ny, nx) shape")
    n1 = shape[0]
    n2 = shape[-1] if len(shape) == 2 else shape[1]
    n3 = 1 if len(shape) == 2 else shape[2]
    p = (C.c_float * 6)(*([float(v) for v in (param or [])] + [0.0] * (6 - len(param or []))))
    if _mem_kind(field) == L.OWL_MEM_DEVICE:
        rev = tuple(reversed(range(field.dim())))
        if not field.permute(*rev).is_contiguous() or (mask is not None and not mask.permute(*rev).is_contiguous()):
            raise ValueError("device fields must be stored z fastest (a transposed view of the flat gradient)")
        _ready(field, mask)
        L.check(lib.owl_grad_process(op, n1, n2, n3, p, _ptr(mask) if mask is not None else None, _ptr(field),
                                     L.OWL_MEM_DEVICE))
        return field
    buf = np.asfortranarray(field, dtype=np.float32)
    mk = None if mask is None else np.asfortranarray(mask, dtype=np.float32)
    L.check(lib.owl_grad_process(op, n1, n2, n3, p, _ptr(mk) if mk is not None else None, _ptr(buf),
                                 L.OWL_MEM_HOST))
    return buf
