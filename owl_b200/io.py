"""File formats of OWL, restated: raw float32 models, SU seismograms, key = value
parameter files.

* models and gradients: float32, (nz, nx) or (nz, ny, nx) with z fastest
  (src/lib/module_model.f90:237-334; grad_<name>.bin in
  src/inverse/2d/module_gradient.f90:454-468);
* SU: 240-byte trace headers, native endianness, ns (int16, byte 115), dt in
  microseconds (int16, byte 117) and d1 (float32, byte 181) set as init_su does
  (src/lib/module_su.f90:1142-1193), then nt float32 samples per trace;
* parameters: one ``key = value`` per line, read by FLIT's readpar_* calls
  (src/lib/module_parameters.f90:316-703).
"""
from __future__ import annotations

import os
from typing import Dict, List, Sequence

import numpy as np

f32 = np.float32


def write_model(path: str, w: np.ndarray) -> None:
    """(nz, nx) or (nz, ny, nx) array -> float32 file, z fastest."""
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    np.asarray(w, dtype=f32).T.astype(f32).tofile(path)


def read_model(path: str, shape: Sequence[int]) -> np.ndarray:
    w = np.fromfile(path, dtype=f32)
    n = int(np.prod(shape))
    if w.size != n:
        raise ValueError(f"{path}: expected {n} floats, got {w.size}")
    return w.reshape(tuple(reversed(tuple(shape)))).T


def write_su(path: str, traces: np.ndarray, dt: float) -> None:
    """traces (ntrace, nt) float32 -> SU file with the headers init_su sets."""
    traces = np.ascontiguousarray(traces, dtype=f32)
    ntr, nt = traces.shape
    if nt > 32767:
        raise ValueError("SU header ns is int16: nt must be <= 32767")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    rec = np.zeros((ntr, 240 + 4 * nt), dtype=np.uint8)
    rec[:, :240] = su_header(nt, dt)
    rec[:, 240:] = traces.view(np.uint8).reshape(ntr, 4 * nt)
    rec.tofile(path)


def su_header(nt: int, dt: float) -> np.ndarray:
    """the 240-byte header every trace of a written SU file carries"""
    hdr = np.zeros(240, dtype=np.uint8)
    hdr[114:116] = np.frombuffer(np.int16(nt).tobytes(), dtype=np.uint8)
    hdr[116:118] = np.frombuffer(np.int16(int(f32(dt) * f32(1.0e6))).tobytes(), dtype=np.uint8)
    hdr[180:184] = np.frombuffer(f32(dt).tobytes(), dtype=np.uint8)
    return hdr


def write_su_device(path: str, traces, dt: float) -> None:
    """CUDA tensor (ntrace, nt) -> SU file: the records are assembled on the GPU
    (owl_su_encode) and leave the device in one copy."""
    import ctypes as C

    import torch

    from . import _lib as L
    ntr, nt = int(traces.shape[0]), int(traces.shape[1])
    if nt > 32767:
        raise ValueError("SU header ns is int16: nt must be <= 32767")
    traces = traces.detach().to(torch.float32).contiguous()
    out = torch.empty(ntr * (240 + 4 * nt), dtype=torch.uint8, device=traces.device)
    hdr = su_header(nt, dt)
    torch.cuda.current_stream(traces.device).synchronize()
    L.check(L.load().owl_su_encode(ntr, nt, hdr.ctypes.data_as(C.c_void_p), C.c_void_p(traces.data_ptr()),
                                   C.c_void_p(out.data_ptr()), L.OWL_MEM_DEVICE))
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    out.cpu().numpy().tofile(path)


def read_su_device(path: str, device="cuda"):
    """SU file -> (CUDA tensor (ntrace, nt), dt seconds): one copy of the file to
    the device, the samples taken out of the records there (owl_su_decode)."""
    import ctypes as C

    import torch

    from . import _lib as L
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < 240:
        raise ValueError(f"{path}: too small for an SU file")
    ns = int(np.frombuffer(raw[114:116].tobytes(), dtype=np.int16)[0])
    dt_us = int(np.frombuffer(raw[116:118].tobytes(), dtype=np.int16)[0])
    tb = 240 + 4 * ns
    if ns < 1 or raw.size % tb:
        raise ValueError(f"{path}: size {raw.size} is not a multiple of the trace size {tb}")
    ntr = raw.size // tb
    din = torch.from_numpy(raw).to(device)
    out = torch.empty((ntr, ns), dtype=torch.float32, device=din.device)
    torch.cuda.current_stream(din.device).synchronize()
    L.check(L.load().owl_su_decode(ntr, ns, C.c_void_p(din.data_ptr()), C.c_void_p(out.data_ptr()),
                                   L.OWL_MEM_DEVICE))
    return out, dt_us * 1.0e-6


def read_su(path: str):
    """SU file -> (traces (ntrace, nt) float32, dt seconds)."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < 240:
        raise ValueError(f"{path}: too small for an SU file")
    ns = int(np.frombuffer(raw[114:116].tobytes(), dtype=np.int16)[0])
    dt_us = int(np.frombuffer(raw[116:118].tobytes(), dtype=np.int16)[0])
    tb = 240 + 4 * ns
    if raw.size % tb:
        raise ValueError(f"{path}: size {raw.size} is not a multiple of the trace size {tb}")
    raw = raw.reshape(-1, tb)
    return raw[:, 240:].copy().view(f32).reshape(-1, ns), dt_us * 1.0e-6


def read_param(path: str) -> Dict[str, str]:
    """key = value lines; '#' starts a comment; values keep their text."""
    out: Dict[str, str] = {}
    with open(path) as f:
        for ln in f:
            ln = ln.split("#", 1)[0].strip()
            if "=" not in ln:
                continue
            k, v = ln.split("=", 1)
            out[k.strip()] = v.strip().strip("'\"")
    return out


def write_param(path: str, params: Dict[str, object]) -> None:
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        for k, v in params.items():
            f.write(f"{k} = {v}\n")


def param_list(v: str) -> List[str]:
    return [x.strip() for x in v.replace(",", " ").split() if x.strip()]


def param_bool(v: str) -> bool:
    return v.strip().lower() in ("y", "yes", "t", "true", ".true.", "1")
