"""Shared test cases (geometries and models) for the acoustic 2D path."""
from __future__ import annotations

import numpy as np

from owl_b200 import _lib as L
from owl_b200.geometry import GridSpec, PreparedShots, Receiver, Shot, Source


def desc(nx, nz, dx, dt, nt, pml=10, R=4, fs=0, f0=15.0, max_shots=8, medium=1, ny=1):
    d = L.OwlSsgDesc()
    d.medium = medium
    d.nx, d.ny, d.nz = nx, ny, nz
    d.dx = d.dy = d.dz = dx
    d.pml, d.fdhalf, d.free_surface = pml, R, fs
    d.dt, d.nt, d.f0_max, d.max_shots = dt, nt, f0, max_shots
    return d


def random_model(nx, nz, seed=0):
    rng = np.random.default_rng(seed)
    vp = (2000 + 300 * rng.random((nz, nx))).astype(np.float32)
    rho = (1000 + 200 * rng.random((nz, nx))).astype(np.float32)
    return vp, rho


def small_shots(nx, nz, dx, fs=False):
    """Mixed off-grid / on-grid explosion and force sources, uneven receiver counts,
    a zero-weight receiver, receivers sharing taps."""
    zr = 0.0 if fs else 42.1
    s = [
        Shot(1, [Source(x=203.3, z=151.7, f0=15.0)], [Receiver(x=50 + 37.3 * i, z=zr + 10.0) for i in range(8)]),
        Shot(2, [Source(x=120.0, z=100.0, mechanism="force", polar=30, f0=15.0)],
             [Receiver(x=60 + 35 * i, z=300.0, weight=(0.0 if i == 2 else 1.0)) for i in range(6)]),
        Shot(3, [Source(x=300.0, z=200.0, f0=12.0, amp=2.0, t0=0.01),
                 Source(x=304.0, z=204.0, f0=15.0, amp=-1.0)],
             [Receiver(x=100 + 3.3 * i, z=250.5) for i in range(11)]),
    ]
    return s


def prepare(shots, nx, nz, dx, dt):
    return PreparedShots(shots, GridSpec(nx=nx, nz=nz, dx=dx, dz=dx), dt)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
