"""ctypes wrapper of oracle/lib/liboracle.so (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "lib", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("oracle_ac2d.cpp", "oracle_ac3d.cpp", "oracle_el2d.cpp", "oracle_el3d.cpp", "oracle_common.hpp")]
    if force or not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        _lib = C.CDLL(ORACLE_LIB)
        vp = C.c_void_p
        _lib.oracle_ac2d_forward_f32.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        _lib.oracle_ac2d_forward_f64.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        _lib.oracle_ac2d_jvp_c128.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp, vp, vp]
        _lib.oracle_ac2d_gradient_f64.argtypes = [vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp, vp]
        _lib.oracle_ac2d_gradient_f32.argtypes = [vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp, vp]
        _lib.oracle_ac2d_ref_gradient_f32.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, C.c_int, vp]
        _lib.oracle_ac3d_forward_f32.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        _lib.oracle_ac3d_forward_f64.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        _lib.oracle_ac3d_jvp_c128.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp, vp]
        _lib.oracle_ac3d_gradient_f64.argtypes = [vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp]
        _lib.oracle_el2d_forward_f32.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib.oracle_el2d_forward_f64.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib.oracle_el2d_jvp_c128.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp]
        _lib.oracle_el2d_gradient_f64.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp, vp]
        _lib.oracle_el2d_setup.argtypes = [vp, vp, vp]
        _lib.oracle_el2d_damp_ratio.argtypes = [C.c_float] * 5 + [C.c_int]
        _lib.oracle_el2d_mesh.argtypes = [vp, vp, vp, vp, vp, vp]
        _lib.oracle_el2d_damp_ratio.restype = C.c_float
        _lib.oracle_el3d_forward_f32.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib.oracle_el3d_forward_f64.argtypes = [vp, vp, C.c_int, vp, vp]
        _lib.oracle_el3d_jvp_c128.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp]
        _lib.oracle_el3d_gradient_f64.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, vp, vp, vp]
        _lib.oracle_el3d_setup.argtypes = [vp, vp, vp]
        _lib.oracle_el3d_set_mpml.argtypes = [vp, C.c_longlong]
        _lib.oracle_el3d_set_mpml.restype = None
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _fort(a, dt):
    return np.asfortranarray(np.asarray(a, dtype=dt))


def _nseis(ps, nt):
    return sum(ps.arr[s].nrec for s in range(ps.nshots)) * nt


def ac2d_forward(desc, vp, rho, ps, precision="f32"):
    """Seismograms (flat, shot-major, trace-major) of the restated reference loops."""
    lib = load()
    dt = np.float32 if precision == "f32" else np.float64
    vp, rho = _fort(vp, dt), _fort(rho, dt)
    out = np.zeros(_nseis(ps, desc.nt), dtype=dt)
    fn = lib.oracle_ac2d_forward_f32 if precision == "f32" else lib.oracle_ac2d_forward_f64
    rc = fn(C.byref(desc), _p(vp), _p(rho), ps.nshots, C.cast(ps.arr, C.c_void_p), _p(out))
    if rc != 0:
        raise RuntimeError("oracle forward failed")
    return out


def ac2d_jvp(desc, vp, rho, dvp, drho, ps):
    """(seis, d seis . (dvp, drho)) by complex-step differentiation in FP64."""
    lib = load()
    a = [_fort(v, np.float64) for v in (vp, rho, dvp, drho)]
    n = _nseis(ps, desc.nt)
    seis, jvp = np.zeros(n), np.zeros(n)
    rc = lib.oracle_ac2d_jvp_c128(C.byref(desc), *[_p(v) for v in a], ps.nshots, C.cast(ps.arr, C.c_void_p),
                                  _p(seis), _p(jvp))
    if rc != 0:
        raise RuntimeError("oracle jvp failed")
    return seis, jvp


def ac2d_gradient(desc, vp, rho, ps, data, adj_kind=0, k=50, precision="f64", stf_grad=False):
    """(misfit per shot, grad (2, nz*nx) z-fastest, stf gradient or None) of the exact adjoint."""
    lib = load()
    dt = np.float64 if precision == "f64" else np.float32
    vp, rho = _fort(vp, dt), _fort(rho, dt)
    data = np.ascontiguousarray(data, dtype=dt)
    misfit = np.zeros(ps.nshots)
    grad = np.zeros(2 * desc.nx * desc.nz, dtype=dt)
    nsrc = sum(ps.arr[s].nsrc for s in range(ps.nshots))
    sg = np.zeros(nsrc * desc.nt, dtype=dt) if stf_grad else None
    fn = lib.oracle_ac2d_gradient_f64 if precision == "f64" else lib.oracle_ac2d_gradient_f32
    rc = fn(C.byref(desc), _p(vp), _p(rho), ps.nshots, C.cast(ps.arr, C.c_void_p), _p(data), adj_kind, k,
            _p(misfit), _p(grad), _p(sg))
    if rc != 0:
        raise RuntimeError("oracle gradient failed")
    return misfit, grad, sg


def ac2d_ref_gradient(desc, vp, rho, ps, adj, cc=1):
    """The reference's own (time-reversed, -dt) gradient, FP32, summed over shots:
    grad (2, nz*nx) z-fastest for (vp, rho)."""
    lib = load()
    vp, rho = _fort(vp, np.float32), _fort(rho, np.float32)
    adj = np.ascontiguousarray(adj, dtype=np.float32)
    hnt = np.array([max(1, h) for h in ps.hnt], dtype=np.int32)
    grad = np.zeros(2 * desc.nx * desc.nz, dtype=np.float32)
    rc = lib.oracle_ac2d_ref_gradient_f32(C.byref(desc), _p(vp), _p(rho), ps.nshots, C.cast(ps.arr, C.c_void_p),
                                          _p(adj), _p(hnt), cc, _p(grad))
    if rc != 0:
        raise RuntimeError("oracle ref gradient failed")
    return grad


def ac3d_forward(desc, vp, rho, ps, precision="f32"):
    """3D seismograms; vp, rho are (nz, ny, nx) arrays."""
    lib = load()
    dt = np.float32 if precision == "f32" else np.float64
    vp, rho = _fort(vp, dt), _fort(rho, dt)
    out = np.zeros(_nseis(ps, desc.nt), dtype=dt)
    fn = lib.oracle_ac3d_forward_f32 if precision == "f32" else lib.oracle_ac3d_forward_f64
    if fn(C.byref(desc), _p(vp), _p(rho), ps.nshots, C.cast(ps.arr, C.c_void_p), _p(out)) != 0:
        raise RuntimeError("oracle ac3d forward failed")
    return out


def ac3d_jvp(desc, vp, rho, dvp, drho, ps):
    lib = load()
    a = [_fort(v, np.float64) for v in (vp, rho, dvp, drho)]
    out = np.zeros(_nseis(ps, desc.nt))
    if lib.oracle_ac3d_jvp_c128(C.byref(desc), *[_p(v) for v in a], ps.nshots, C.cast(ps.arr, C.c_void_p), _p(out)):
        raise RuntimeError("oracle ac3d jvp failed")
    return out


def ac3d_gradient(desc, vp, rho, ps, data, adj_kind=0, k=50):
    """(misfit per shot, grad (2, nz*ny*nx) z-fastest) of the exact adjoint in FP64."""
    lib = load()
    vp, rho = _fort(vp, np.float64), _fort(rho, np.float64)
    data = np.ascontiguousarray(data, dtype=np.float64)
    misfit = np.zeros(ps.nshots)
    grad = np.zeros(2 * desc.nx * desc.ny * desc.nz)
    if lib.oracle_ac3d_gradient_f64(C.byref(desc), _p(vp), _p(rho), ps.nshots, C.cast(ps.arr, C.c_void_p), _p(data),
                                    adj_kind, k, _p(misfit), _p(grad)):
        raise RuntimeError("oracle ac3d gradient failed")
    return misfit, grad


# ------------------------------- elastic 2D ----------------------------------
def _fields(fields, dt):
    """list of (nz, nx) arrays -> (pointer array, kept arrays), z fastest"""
    keep = [_fort(f, dt) for f in fields]
    arr = (C.c_void_p * len(keep))(*[a.ctypes.data for a in keep])
    return arr, keep


def _nseis_el(ps, nt):
    return 2 * sum(ps.arr[s].nrec for s in range(ps.nshots)) * nt


def el2d_forward(desc, fields, ps, precision="f32"):
    """Elastic seismograms, per shot (vx traces, vz traces) x nt, shots concatenated."""
    lib = load()
    dt = np.float32 if precision == "f32" else np.float64
    arr, keep = _fields(fields, dt)
    out = np.zeros(_nseis_el(ps, desc.nt), dtype=dt)
    fn = lib.oracle_el2d_forward_f32 if precision == "f32" else lib.oracle_el2d_forward_f64
    if fn(C.byref(desc), arr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(out)) != 0:
        raise RuntimeError("oracle el2d forward failed")
    return out


def el2d_jvp(desc, fields, dfields, ps):
    """(seis, d seis . dfields) by complex-step differentiation in FP64."""
    lib = load()
    arr, k1 = _fields(fields, np.float64)
    darr, k2 = _fields(dfields, np.float64)
    n = _nseis_el(ps, desc.nt)
    seis, jvp = np.zeros(n), np.zeros(n)
    if lib.oracle_el2d_jvp_c128(C.byref(desc), arr, darr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(seis), _p(jvp)):
        raise RuntimeError("oracle el2d jvp failed")
    return seis, jvp


def el2d_gradient(desc, fields, ps, data, adj_kind=0, k=50, stf_grad=False):
    """(misfit per shot, grad (nparam, nz*nx) z-fastest, stf gradient or None), FP64 exact adjoint."""
    lib = load()
    arr, keep = _fields(fields, np.float64)
    data = np.ascontiguousarray(data, dtype=np.float64)
    misfit = np.zeros(ps.nshots)
    grad = np.zeros(len(fields) * desc.nx * desc.nz)
    nsrc = sum(ps.arr[s].nsrc for s in range(ps.nshots))
    sg = np.zeros(nsrc * desc.nt) if stf_grad else None
    if lib.oracle_el2d_gradient_f64(C.byref(desc), arr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(data), adj_kind,
                                    k, _p(misfit), _p(grad), _p(sg)):
        raise RuntimeError("oracle el2d gradient failed")
    return misfit, grad, sg


def el2d_dt_stable(desc, fields):
    lib = load()
    arr, keep = _fields(fields, np.float32)
    out = C.c_float(0)
    if lib.oracle_el2d_setup(C.byref(desc), arr, C.byref(out)):
        raise RuntimeError("oracle el2d setup failed")
    return out.value


def el2d_mesh(desc):
    """(nz_mesh, z_i, z_h, dz_i, dz_h) of the depth-refined free-surface mesh,
    rows -pml .. nz_mesh + pml + 1; the arrays are None on the uniform grid."""
    lib = load()
    n = C.c_int(0)
    if lib.oracle_el2d_mesh(C.byref(desc), C.byref(n), None, None, None, None):
        raise RuntimeError("oracle el2d mesh failed")
    arr = [np.zeros(n.value + 2 * desc.pml + 2, dtype=np.float32) for _ in range(4)]
    if lib.oracle_el2d_mesh(C.byref(desc), C.byref(n), *[_p(a) for a in arr]):
        raise RuntimeError("oracle el2d mesh failed")
    refined = bool(np.any(arr[2] != 0))
    return (n.value, *arr) if refined else (n.value, None, None, None, None)


def el2d_damp_ratio(c11, c13, c33, c55, rho, direction="x"):
    return load().oracle_el2d_damp_ratio(c11, c13, c33, c55, rho, 1 if direction == "z" else 0)


# ------------------------------- elastic 3D ----------------------------------
def _nseis_el3(ps, nt):
    return 3 * sum(ps.arr[s].nrec for s in range(ps.nshots)) * nt


def el3d_set_mpml(faces=None):
    """M-PML face ratios (the layout of owl_ssg_mpml_ratios) for the following
    elastic 3D oracle runs; None: all zero."""
    lib = load()
    if faces is None:
        lib.oracle_el3d_set_mpml(None, 0)
        return
    f = np.ascontiguousarray(faces, dtype=np.float32)
    lib.oracle_el3d_set_mpml(f.ctypes.data, f.size)


def el3d_forward(desc, fields, ps, precision="f32"):
    """3D elastic seismograms, per shot (vx, vy, vz traces) x nt; fields (nz, ny, nx)."""
    lib = load()
    dt = np.float32 if precision == "f32" else np.float64
    arr, keep = _fields(fields, dt)
    out = np.zeros(_nseis_el3(ps, desc.nt), dtype=dt)
    fn = lib.oracle_el3d_forward_f32 if precision == "f32" else lib.oracle_el3d_forward_f64
    if fn(C.byref(desc), arr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(out)) != 0:
        raise RuntimeError("oracle el3d forward failed")
    return out


def el3d_jvp(desc, fields, dfields, ps):
    lib = load()
    arr, k1 = _fields(fields, np.float64)
    darr, k2 = _fields(dfields, np.float64)
    n = _nseis_el3(ps, desc.nt)
    seis, jvp = np.zeros(n), np.zeros(n)
    if lib.oracle_el3d_jvp_c128(C.byref(desc), arr, darr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(seis), _p(jvp)):
        raise RuntimeError("oracle el3d jvp failed")
    return seis, jvp


def el3d_gradient(desc, fields, ps, data, adj_kind=0, k=50, stf_grad=False):
    lib = load()
    arr, keep = _fields(fields, np.float64)
    data = np.ascontiguousarray(data, dtype=np.float64)
    misfit = np.zeros(ps.nshots)
    grad = np.zeros(len(fields) * desc.nx * desc.ny * desc.nz)
    nsrc = sum(ps.arr[s].nsrc for s in range(ps.nshots))
    sg = np.zeros(nsrc * desc.nt) if stf_grad else None
    if lib.oracle_el3d_gradient_f64(C.byref(desc), arr, ps.nshots, C.cast(ps.arr, C.c_void_p), _p(data), adj_kind,
                                    k, _p(misfit), _p(grad), _p(sg)):
        raise RuntimeError("oracle el3d gradient failed")
    return misfit, grad, sg


def el3d_dt_stable(desc, fields):
    lib = load()
    arr, keep = _fields(fields, np.float32)
    out = C.c_float(0)
    if lib.oracle_el3d_setup(C.byref(desc), arr, C.byref(out)):
        raise RuntimeError("oracle el3d setup failed")
    return out.value
