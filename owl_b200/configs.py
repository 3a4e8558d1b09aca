"""Synthetic workloads with the shapes of the benchmark configurations.

No external dataset is involved: every model is generated here from closed
forms or seeded random fields.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .geometry import Receiver, Shot, Source


def _desc(medium, nx, nz, dx, dt, nt, pml, fdhalf=4, fs=0, f0=10.0, max_shots=1, ny=1):
    d = L.OwlSsgDesc()
    d.medium = medium
    d.nx, d.ny, d.nz = nx, ny, nz
    d.dx = d.dy = d.dz = dx
    d.pml, d.fdhalf, d.free_surface = pml, fdhalf, fs
    d.dt, d.nt, d.f0_max, d.max_shots = dt, nt, f0, max_shots
    return d


def acoustic_2d_true_model(nz=201, nx=401, dx=10.0):
    """Vp linear 1500 -> 4000 m/s over depth plus a +300 m/s Gaussian (sigma 300 m)
    centred at depth 1000 m, x 2000 m (the model centre); rho = 310 * Vp^0.25."""
    z = np.arange(nz, dtype=np.float64)[:, None] * dx
    x = np.arange(nx, dtype=np.float64)[None, :] * dx
    zmax = (nz - 1) * dx
    vp = 1500.0 + 2500.0 * z / zmax
    vp = vp + 300.0 * np.exp(-((z - 1000.0) ** 2 + (x - 2000.0) ** 2) / (2 * 300.0 ** 2))
    vp = np.broadcast_to(vp, (nz, nx)).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    return vp, rho


def config1():
    """Plain 2D acoustic forward: 201 x 401, dx 10 m, dt 1 ms, 2000 steps, PML 20,
    8th order, one 10 Hz Ricker explosion at (x 2000, z 20), 401 receivers at z 20."""
    nz, nx, dx, dt, nt = 201, 401, 10.0, 1e-3, 2000
    d = _desc(L.OWL_ACOUSTIC_ISO_2D, nx, nz, dx, dt, nt, pml=20, f0=10.0)
    vp, rho = acoustic_2d_true_model(nz, nx, dx)
    shots = [Shot(1, [Source(x=2000.0, z=20.0, f0=10.0)], [Receiver(x=10.0 * i, z=20.0) for i in range(nx)])]
    return d, vp, rho, shots


def config2_shots(nshots=32, nx=401, dx=10.0, offset_max=1500.0):
    """Shots evenly spaced from 100 m to 3900 m at z 20 m; receivers every grid
    column at z 20 m, kept only within +-offset_max of the source (uneven counts)."""
    shots = []
    for k in range(nshots):
        xs = 100.0 + k * (3800.0 / (nshots - 1)) if nshots > 1 else 2000.0
        recs = [Receiver(x=10.0 * i, z=20.0) for i in range(nx) if abs(10.0 * i - xs) <= offset_max]
        shots.append(Shot(k + 1, [Source(x=xs, z=20.0, f0=10.0)], recs))
    return shots


def smooth(a, sigma_cells):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(np.asarray(a, dtype=np.float64), sigma=sigma_cells, mode="nearest").astype(np.float32)


def config2(nshots=32):
    """2D acoustic FWI gradient: true model of config1, starting model = both Vp and
    rho smoothed by a Gaussian of sigma 150 m, 32 shots, checkpoints every 50 steps."""
    nz, nx, dx, dt, nt = 201, 401, 10.0, 1e-3, 2000
    d = _desc(L.OWL_ACOUSTIC_ISO_2D, nx, nz, dx, dt, nt, pml=20, f0=10.0, max_shots=nshots)
    vp, rho = acoustic_2d_true_model(nz, nx, dx)
    vp0, rho0 = smooth(vp, 15.0), smooth(rho, 15.0)
    return d, (vp, rho), (vp0, rho0), config2_shots(nshots, nx, dx)
