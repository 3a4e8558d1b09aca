"""GPU test of owl_ssg_forward_noalloc, the forward entry point that allocates
no device memory (for callers that cannot call cudaMalloc because their
device memory is owned by another allocator or reserved as a fixed budget).

The file name sorts last so that pytest collects it after every other test:
the entry point shares one static device array across calls and keeps the
last call's contents, so it must give the right answer both in a fresh
process and after the other tests have used the device.

Each call goes through the C ABI and is compared with owl_ssg_forward on the
same shot, with the forward tolerance of the other GPU tests (1e-5 relative
L2). Two calls in a row on different grids check that the second call does not
see what the first left in the array.
"""
import ctypes as C

import numpy as np
import pytest

from owl_b200 import _lib as L
from owl_b200.geometry import Receiver, Shot, Source
from owl_b200.solver import SSGSolver

from cases import desc, prepare, random_model, rel

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-5


def _fields(vp, rho):
    keep = [np.asfortranarray(np.asarray(f, dtype=np.float32)) for f in (vp, rho)]
    arr = (C.POINTER(C.c_float) * 2)(*[f.ctypes.data_as(C.POINTER(C.c_float)) for f in keep])
    return arr, keep


def _noalloc(d, vp, rho, ps):
    lib = L.load()
    arr, keep = _fields(vp, rho)
    nrec = ps.nrec(0)
    out = np.full(nrec * d.nt, np.nan, dtype=np.float32)
    rc = lib.owl_ssg_forward_noalloc(C.byref(d), 2, arr, C.byref(ps.arr[0]), out.ctypes.data_as(C.c_void_p))
    L.check(rc)
    del keep
    return out


def _regular(d, vp, rho, ps):
    s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, d.nx, d.nz, d.dx, d.dz, d.dt, d.nt, pml=d.pml, fdhalf=d.fdhalf,
                  free_surface=False, f0_max=d.f0_max, max_shots=1)
    s.set_model(vp, rho)
    return s.forward(ps)


def _case(nx, nz, R, nt, seed):
    dx, dt = 10.0, 1e-3
    d = desc(nx, nz, dx, dt, nt, pml=12, R=R, f0=15.0, max_shots=1)
    vp, rho = random_model(nx, nz, seed=seed)
    xs, zs = 0.43 * (nx - 1) * dx + 0.7, 0.55 * (nz - 1) * dx + 1.3
    shot = Shot(1, [Source(x=xs, z=zs, f0=15.0, amp=2.0, t0=0.01), Source(x=xs + 40.0, z=zs - 30.0, f0=12.0, amp=-1.0)],
                [Receiver(x=30.0 + 9.7 * i, z=42.1, weight=(0.0 if i == 3 else 1.0)) for i in range((nx - 8) // 1)])
    return d, vp, rho, prepare([shot], nx, nz, dx, dt)


def test_noalloc_matches_forward_two_calls():
    first = _case(96, 72, 8, 500, seed=3)
    second = _case(64, 48, 4, 400, seed=5)
    for d, vp, rho, ps in (first, second):
        got = _noalloc(d, vp, rho, ps)
        ref = _regular(d, vp, rho, ps)
        assert np.all(np.isfinite(got))
        assert np.linalg.norm(ref) > 0
        assert rel(got, ref) < FWD_TOL, rel(got, ref)
        assert np.all(got.reshape(ps.nrec(0), d.nt)[3] == 0)  # zero-weight receiver


def test_noalloc_rejects_beyond_limit():
    n = 4200  # 4200 x 4200 needs more than OWL_NOALLOC_MAX_FLOATS floats
    d = desc(n, n, 10.0, 1e-3, 10, pml=12, R=4, f0=15.0, max_shots=1)
    vp = np.full((n, n), 2000.0, dtype=np.float32)
    rho = np.full((n, n), 1000.0, dtype=np.float32)
    ps = prepare([Shot(1, [Source(x=100.0, z=100.0, f0=15.0)], [Receiver(x=200.0, z=100.0)])], n, n, 10.0, 1e-3)
    lib = L.load()
    arr, keep = _fields(vp, rho)
    out = np.zeros(10, dtype=np.float32)
    rc = lib.owl_ssg_forward_noalloc(C.byref(d), 2, arr, C.byref(ps.arr[0]), out.ctypes.data_as(C.c_void_p))
    assert rc == L.OWL_ERR_INVALID
    assert "OWL_NOALLOC_MAX_FLOATS" in lib.owl_last_error().decode()
