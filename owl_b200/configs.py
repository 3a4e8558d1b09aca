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


def value_noise_3d(shape, cells_per_node, seed):
    """Smooth seeded noise in [-1, 1]: uniform random values on a coarse lattice
    every `cells_per_node` cells, cubic-spline interpolated to the grid."""
    from scipy.ndimage import zoom
    rng = np.random.default_rng(seed)
    coarse = [max(2, int(np.ceil(n / cells_per_node)) + 1) for n in shape]
    c = rng.uniform(-1.0, 1.0, size=coarse)
    f = zoom(c, [n / m for n, m in zip(shape, coarse)], order=3, mode="nearest")[: shape[0], : shape[1], : shape[2]]
    f = f - f.mean()
    return (f / max(1e-12, np.abs(f).max())).astype(np.float32)


def acoustic_3d_model(n=400, dx=10.0, nlayers=8, vmax_layer=4000.0):
    """8 layers with Vp uniform in [1500, vmax_layer] (seed 3) at sorted uniform
    depths (seed 4), times (1 + 0.05 noise) with smooth value noise (seed 5,
    ~500 m wavelength); Gardner rho. vmax_layer = 4000 keeps Vp <= 4200 m/s, the
    CFL bound of dt = 1 ms at dx = 10 m for the 8th-order scheme (the layer
    range [1500, 4500] of the benchmark description would need dt <= 0.92 ms)."""
    v = np.random.default_rng(3).uniform(1500.0, vmax_layer, nlayers)
    tops = np.sort(np.random.default_rng(4).uniform(0.0, (n - 1) * dx, nlayers - 1))
    z = np.arange(n) * dx
    idx = np.searchsorted(tops, z, side="right")
    vz = v[idx].astype(np.float32)
    noise = value_noise_3d((n, n, n), max(2, int(round(500.0 / dx))), 5)
    vp = (vz[:, None, None] * (1.0 + 0.05 * noise)).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    return vp, rho


def config3(n=400, nt=1500):
    """3D acoustic: 400^3, dx 10 m, 8th order, PML 20, dt 1 ms, 1500 steps, one
    12 Hz Ricker at the centre x, y and z = 20 m, 200 x 200 receivers every 20 m at z = 20 m."""
    dx, dt = 10.0, 1e-3
    d = _desc(L.OWL_ACOUSTIC_ISO_3D, n, n, dx, dt, nt, pml=20, f0=12.0, ny=n)
    vp, rho = acoustic_3d_model(n, dx)
    c = (n // 2) * dx
    nr = min(200, n // 2)
    recs = [Receiver(x=20.0 * i, y=20.0 * j, z=20.0) for j in range(nr) for i in range(nr)]
    shots = [Shot(1, [Source(x=c, y=c, z=20.0, f0=12.0)], recs)]
    return d, vp, rho, shots


def _rescaled_noise(shape, sigma_cells, seed, lo, hi):
    """Gaussian-filtered seeded white noise rescaled to [lo, hi]."""
    from scipy.ndimage import gaussian_filter
    w = np.random.default_rng(seed).standard_normal(shape)
    f = gaussian_filter(w, sigma=sigma_cells, mode="nearest")
    f = (f - f.min()) / max(1e-30, f.max() - f.min())
    return (lo + (hi - lo) * f).astype(np.float32)


def elastic_2d_vti_model(nz=301, nx=601, dx=5.0, eps_max=0.2):
    """Vp 1800 -> 4500 m/s linear in depth, Vs = Vp / 1.8, Gardner rho, Thomsen
    epsilon in [0, eps_max] and delta in [-0.05, 0.1] as smooth seeded fields
    (Gaussian-filtered white noise, sigma 100 m, seeds 7 and 8), no tilt.
    Returns (vp, vs, epsilon, delta, theta, rho), each (nz, nx)."""
    z = np.arange(nz, dtype=np.float64)[:, None] * dx
    vp = np.broadcast_to(1800.0 + 2700.0 * z / ((nz - 1) * dx), (nz, nx)).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    sig = 100.0 / dx
    eps = _rescaled_noise((nz, nx), sig, 7, 0.0, eps_max)
    dl = _rescaled_noise((nz, nx), sig, 8, -0.05, 0.1)
    return vp, vs, eps, dl, np.zeros_like(vp), rho


def config4_shots(nshots=64, nx=601, dx=5.0, zsrc=10.0):
    """Shots evenly spaced from 100 m to (nx-1) dx - 100 m at z = zsrc, alternating an
    explosion and a vertical force (polar 0), 15 Hz Ricker; receivers every 10 m at
    z = 0 (two components, vx and vz)."""
    xmax = (nx - 1) * dx
    recs = [Receiver(x=10.0 * i, z=0.0) for i in range(int(xmax // 10.0) + 1)]
    shots = []
    for k in range(nshots):
        xs = 100.0 + k * ((xmax - 200.0) / max(1, nshots - 1))
        src = Source(x=xs, z=zsrc, f0=15.0) if k % 2 == 0 else Source(x=xs, z=zsrc, mechanism="force", polar=0.0, f0=15.0)
        shots.append(Shot(k + 1, [src], recs))
    return shots


def config4(nshots=64, nt=4000):
    """2D elastic VTI with a flat free surface on the uniform grid: 301 x 601,
    dx = dz = 5 m, dt = 0.5 ms, 4000 steps, PML 20, 8th order, Thomsen
    parameterisation; 64 shots (explosion / vertical force, 15 Hz); receivers every
    10 m at the surface. epsilon is capped at 0.19 so that the fastest qP speed
    (Vp sqrt(1 + 2 eps) at Vp = 4500) keeps dt = 0.5 ms inside the CFL bound."""
    nz, nx, dx, dt = 301, 601, 5.0, 5e-4
    d = _desc(L.OWL_ELASTIC_VHTIORT_2D, nx, nz, dx, dt, nt, pml=20, fs=1, f0=15.0, max_shots=nshots)
    d.aniso = L.OWL_ANISO_THOMSEN
    return d, elastic_2d_vti_model(nz, nx, dx, eps_max=0.19), config4_shots(nshots, nx, dx)


def _value_noise_linear(shape, cells_per_node, seed):
    """Seeded noise in [-1, 1]: uniform values on a coarse lattice, trilinear
    interpolation to the grid."""
    from scipy.ndimage import zoom
    rng = np.random.default_rng(seed)
    coarse = [max(2, int(np.ceil(n / cells_per_node)) + 1) for n in shape]
    c = rng.uniform(-1.0, 1.0, size=coarse).astype(np.float32)
    f = zoom(c, [n / m for n, m in zip(shape, coarse)], order=1, mode="nearest")[: shape[0], : shape[1], : shape[2]]
    f = f - f.mean()
    return (f / max(1e-12, float(np.abs(f).max()))).astype(np.float32)


def elastic_3d_ort_model(n=256, dx=10.0):
    """Vp 2000 -> 5000 m/s linear in depth, Vs = Vp / 1.73, Gardner rho, and an
    orthorhombic perturbation: c11, c22, c55, c66 scaled by (1 + a) with a in
    [0, 0.15] smooth seeded fields (value noise, seed 11, ~300 m wavelength);
    c12 = c13 = c23 = rho (vp^2 - 2 vs^2), c33 = rho vp^2, c44 = rho vs^2. The
    fastest qP speed, vp sqrt(1.15) <= 5362 m/s, keeps dt = 0.8 ms inside the CFL
    bound at dx = 10 m. Returns the ten (nz, ny, nx) fields c11 c12 c13 c22 c23
    c33 c44 c55 c66 rho."""
    z = np.arange(n, dtype=np.float64) * dx
    vp = (2000.0 + 3000.0 * z / ((n - 1) * dx))[:, None, None] * np.ones((1, n, n))
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    cells = max(2, int(round(300.0 / dx)))
    fac = [0.075 * (1.0 + _value_noise_linear((n, n, n), cells, 11 + q)) for q in range(4)]
    c33, c44 = rho * vp ** 2, rho * vs ** 2
    c12 = rho * (vp ** 2 - 2 * vs ** 2)
    f = [c33 * (1 + fac[0]), c12, c12, c33 * (1 + fac[1]), c12, c33, c44, c44 * (1 + fac[2]), c44 * (1 + fac[3]), rho]
    return [np.asarray(x, dtype=np.float32) for x in f]


def config5(nshots=16, nt=2500, n=256, nrec=128):
    """3D elastic orthorhombic: n^3 (256^3), dx 10 m, dt 0.8 ms, PML 20, 8th order,
    nine-Cij parameterisation; vertical-force 10 Hz shots on a line at 20 m depth;
    nrec x nrec three-component receivers every 2 cells at 20 m depth, centred and
    on grid nodes (their interpolation taps collapse to one node)."""
    dx, dt = 10.0, 8e-4
    d = _desc(L.OWL_ELASTIC_VHTIORT_3D, n, n, dx, dt, nt, pml=20, f0=10.0, max_shots=nshots, ny=n)
    d.aniso = L.OWL_ANISO_CIJ
    step = 2 * dx
    nr = min(nrec, n // 2)
    x0 = dx * float(int(((n - 1) * dx / 2 - step * (nr - 1) / 2) / dx))
    recs = [Receiver(x=x0 + step * i, y=x0 + step * j, z=20.0) for j in range(nr) for i in range(nr)]
    shots = []
    for k in range(nshots):
        xs = 200.0 + k * (((n - 1) * dx - 400.0) / max(1, nshots - 1))
        shots.append(Shot(k + 1, [Source(x=xs, y=(n - 1) * dx / 2, z=20.0, mechanism="force", polar=0.0, f0=10.0)], recs))
    return d, elastic_3d_ort_model(n, dx), shots
