"""Host-side source / receiver preparation, restating OWL's geometry module.

Follows src/lib/module_source_receiver.f90:
  * types source / receiver / source_receiver_geometry  (:29-142)
  * prepare_geometry: grid indices gx/hx, 9-tap Kaiser-windowed sinc (:556-830)
  * wavelets and prepare_stf (:835-997, :1002-1130)
  * load_geometry's ASCII per-shot files (:183-300)
Arithmetic is float32 like the Fortran ``real`` variables.

FLIT (github.com/lanl/flit, no version pinned by the reference) supplies
``sinc`` and ``bessel_i0``; they are restated here from their definitions
(sin(x)/x, and the power series of I0), so the off-grid taps are not pinned
bit-for-bit to the reference build.
"""
from __future__ import annotations

import ctypes as C
import functools
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L

f32 = np.float32
NKW = 4  # half length of the Kaiser sinc (module_source_receiver.f90:146)
KAISER_B0 = float(np.float32(6.31))  # double parameter initialised from a real literal (:147)
CONST_PI = math.pi


def nint(v) -> int:
    """Fortran NINT: round half away from zero."""
    v = float(v)
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))


def bessel_i0(x: float) -> float:
    """Modified Bessel function I0 by its power series sum (x/2)^(2k)/(k!)^2."""
    x = float(x)
    term, acc, k = 1.0, 1.0, 0
    q = 0.25 * x * x
    while True:
        k += 1
        term *= q / (k * k)
        acc += term
        if term < 1e-17 * acc:
            return acc


def kaiser_sinc_kernel(x) -> np.ndarray:
    """9-tap Kaiser-windowed sinc for a fractional offset x (module_source_receiver.f90:789-828)."""
    return _kaiser_cached(float(f32(x))).copy()


@functools.lru_cache(maxsize=65536)
def _kaiser_cached(xv: float) -> np.ndarray:
    x = f32(xv)
    h = np.zeros(2 * NKW + 1, dtype=f32)
    if x == 0:
        h[NKW] = 1.0
        return h
    i0b = bessel_i0(KAISER_B0)
    for i in range(-NKW, NKW + 1):
        t = f32(f32(i) - x)
        arg = CONST_PI * float(t)
        s = f32(math.sin(arg) / arg) if arg != 0.0 else f32(1.0)
        if -NKW <= t <= NKW:
            r = f32(math.sqrt(float(f32(1.0) - f32(t / f32(NKW)) ** 2)))
            r = f32(bessel_i0(KAISER_B0 * float(r)) / i0b)
        else:
            r = f32(0.0)
        h[i + NKW] = f32(s * r)
    return h


# ------------------------------- wavelets -----------------------------------
def ricker_wavelet(f0, t):
    w = f32((CONST_PI * float(f0) * float(t)) ** 2)
    return f32(f32(1.0 - f32(2.0) * w) * f32(math.exp(-float(w))))


def ricker_deriv_wavelet(f0, t):
    w = f32((CONST_PI * float(f0) * float(t)) ** 2)
    return f32(f32(f32(2.0) * w - f32(3.0)) * f32(math.exp(-float(w))) * f32(t))


def gaussian_wavelet(f0, t):
    return f32(math.exp(-(CONST_PI * float(f0) * float(t)) ** 2))


def gaussian_deriv_wavelet(f0, t):
    return f32(-float(t) * math.exp(-(CONST_PI * float(f0) * float(t)) ** 2))


WAVELETS = {
    "ricker": ricker_wavelet, "gaussian_deriv_deriv": ricker_wavelet, "gaussian_deriv2": ricker_wavelet,
    "ricker_deriv": ricker_deriv_wavelet, "ricker_deriv1": ricker_deriv_wavelet,
    "gaussian_deriv_deriv_deriv": ricker_deriv_wavelet, "gaussian_deriv3": ricker_deriv_wavelet,
    "gaussian": gaussian_wavelet, "gaussian_deriv": gaussian_deriv_wavelet, "gaussian_deriv1": gaussian_deriv_wavelet,
}


@dataclass
class Source:
    """One source line of an OWL geometry file. polar/azimuth in degrees."""
    x: float
    z: float
    y: float = 0.0
    mechanism: str = "explosion"
    polar: float = 0.0
    azimuth: float = 0.0
    mt: Sequence[float] = (0, 0, 0, 0, 0, 0)
    wavelet: str = "ricker"
    f0: float = 20.0
    amp: float = 1.0
    t0: float = 0.0
    stf: Optional[np.ndarray] = None  # custom wavelet samples at the modelling dt


@dataclass
class Receiver:
    x: float
    z: float
    y: float = 0.0
    weight: float = 1.0


@dataclass
class Shot:
    id: int
    sources: List[Source]
    receivers: List[Receiver]


def prepare_stf(src: Source, dt: float, f0factor: float = 1.0, time_integration: int = 0):
    """Prepared STF samples and hnt (prepare_stf, module_source_receiver.f90:1002-1130)."""
    dt = f32(dt)
    if src.wavelet == "custom":
        stf = np.asarray(src.stf, dtype=f32).copy()
    else:
        nt = int(math.ceil(float(f32(f32(f32(2.0) * f32(f0factor)) / f32(src.f0)) / dt)))
        fn = WAVELETS.get(src.wavelet, ricker_wavelet)
        delay = f32(f32(f0factor) / f32(src.f0))
        stf = np.array([fn(src.f0, f32(f32(t) * dt) - delay) for t in range(nt)], dtype=f32)
        stf = (stf / f32(np.max(np.abs(stf)))).astype(f32)
    hnt = nint(len(stf) / 2.0)
    if time_integration < 0:
        # finite-difference derivative of the STF: centred inside, one-sided at the ends
        for _ in range(-time_integration):
            d = np.empty_like(stf)
            d[1:-1] = (stf[2:] - stf[:-2]) * f32(0.5)
            d[0] = stf[1] - stf[0]
            d[-1] = stf[-1] - stf[-2]
            stf = (d / dt).astype(f32)
    elif time_integration > 0:
        for _ in range(time_integration):
            stf = (np.cumsum(stf, dtype=f32) * dt).astype(f32)
    return stf, hnt


def _node(x, o, d):
    """gx = nint((x-o)/d)+1 and hx = nint((x-o+d/2)/d)+1 with their sinc taps."""
    x, o, d = f32(x), f32(o), f32(d)
    q = f32(f32(x - o) / d)
    g = nint(q) + 1
    qh = f32(f32(f32(x - o) + f32(0.5) * d) / d)
    h = nint(qh) + 1
    ti = kaiser_sinc_kernel(f32(q - f32(g - 1)))
    th = kaiser_sinc_kernel(f32(qh - f32(h - 1)))
    return g, h, ti, th


@dataclass
class ZMesh:
    """Computational rows of the depth-refined free-surface mesh
    (owl_vertical_mesh): rows -pml .. n + pml + 1 of the reference's zz_i,
    zz_h, dz_i, dz_h (src/solver/elastic_vhtiort_2d/module_vars.f90:313-376)."""
    pml: int
    z_i: np.ndarray
    z_h: np.ndarray
    dz_i: np.ndarray
    dz_h: np.ndarray

    def at(self, arr: np.ndarray, j: int) -> np.float32:
        return arr[j + self.pml]


#: the small offset that places a source or receiver at z = 0 on the half row
#: below the free surface (module_source_receiver.f90:614-616); FLIT's own
#: value is not vendored, any positive offset well below the row spacing gives
#: the same row
FLOAT_SMALL = f32(1.0e-6)


def _node_mesh(z, o, m: ZMesh):
    """gz / hz as the nearest integer / half row of the mesh (the first on a
    tie), taps from the offset in units of the row's spacing
    (module_source_receiver.f90:596-616, 640-680)."""
    z, o = f32(z), f32(o)
    rel = f32(z - o)
    g = int(np.argmin(np.abs(f32(rel) - m.z_i))) - m.pml
    relh = f32(f32(z + (FLOAT_SMALL if z == 0 else f32(0))) - o)
    h = int(np.argmin(np.abs(relh - m.z_h))) - m.pml
    ti = kaiser_sinc_kernel(f32(f32(rel - m.at(m.z_i, g)) / m.at(m.dz_i, g)))
    th = kaiser_sinc_kernel(f32(f32(rel - m.at(m.z_h, h)) / m.at(m.dz_h, h)))
    return g, h, ti, th


@dataclass
class GridSpec:
    nx: int
    nz: int
    dx: float
    dz: float
    ox: float = 0.0
    oz: float = 0.0
    ny: int = 1
    dy: float = 1.0
    oy: float = 0.0
    zmesh: Optional[ZMesh] = None  # rows of the refined free-surface mesh, None on the uniform grid

    def node_z(self, z):
        return _node(z, self.oz, self.dz) if self.zmesh is None else _node_mesh(z, self.oz, self.zmesh)


class PreparedShots:
    """ctypes owl_shot array (plus the memory it points to) for a list of shots."""

    def __init__(self, shots: Sequence[Shot], grid: GridSpec, dt: float, f0factor: float = 1.0,
                 time_integration: int = 0, fill_struct=None):
        self.shots = list(shots)
        self._keep = []
        arr = (L.OwlShot * len(self.shots))()
        self.hnt = []
        dim3 = grid.ny > 1
        xmax = f32((grid.nx - 1) * grid.dx + grid.ox)
        zmax = f32((grid.nz - 1) * grid.dz + grid.oz)
        ymax = f32((grid.ny - 1) * grid.dy + grid.oy)
        for s, sh in enumerate(self.shots):
            srcs = (L.OwlSource * max(1, len(sh.sources)))()
            nvalid = 0
            hnt = 0
            for q in sh.sources:
                valid = grid.ox <= q.x <= xmax and grid.oz <= q.z <= zmax and (not dim3 or grid.oy <= q.y <= ymax)
                if not valid:
                    continue
                o = srcs[nvalid]
                self._fill_source(o, q, grid, dt, f0factor, time_integration)
                hnt = self.hnt_last
                nvalid += 1
            recs = (L.OwlReceiver * max(1, len(sh.receivers)))()
            for r, q in enumerate(sh.receivers):
                o = recs[r]
                valid = grid.ox <= q.x <= xmax and grid.oz <= q.z <= zmax and (not dim3 or grid.oy <= q.y <= ymax)
                if q.weight != 0 and valid:
                    o.gx, o.hx, ix, hx = _node(q.x, grid.ox, grid.dx)
                    o.gz, o.hz, iz, hz = grid.node_z(q.z)
                    o.interp_ix[:] = ix.tolist(); o.interp_hx[:] = hx.tolist()
                    o.interp_iz[:] = iz.tolist(); o.interp_hz[:] = hz.tolist()
                    if dim3:
                        o.gy, o.hy, iy, hy = _node(q.y, grid.oy, grid.dy)
                        o.interp_iy[:] = iy.tolist(); o.interp_hy[:] = hy.tolist()
                    o.weight = float(q.weight)
                else:
                    o.weight = 0.0
            self._keep += [srcs, recs]
            arr[s].id = int(sh.id)
            arr[s].nsrc = nvalid
            arr[s].src = srcs
            arr[s].nrec = len(sh.receivers)
            arr[s].rec = recs
            self.hnt.append(hnt)
        self.arr = arr

    def _fill_source(self, o, q: Source, grid: GridSpec, dt, f0factor, time_integration):
        o.mechanism = {"explosion": L.OWL_SRC_EXPLOSION, "force": L.OWL_SRC_FORCE, "mt": L.OWL_SRC_MT}[q.mechanism]
        o.gx, o.hx, ix, hx = _node(q.x, grid.ox, grid.dx)
        o.gz, o.hz, iz, hz = grid.node_z(q.z)
        o.interp_ix[:] = ix.tolist(); o.interp_hx[:] = hx.tolist()
        o.interp_iz[:] = iz.tolist(); o.interp_hz[:] = hz.tolist()
        if grid.ny > 1:
            o.gy, o.hy, iy, hy = _node(q.y, grid.oy, grid.dy)
            o.interp_iy[:] = iy.tolist(); o.interp_hy[:] = hy.tolist()
        o.amp = float(q.amp)
        deg2rad = f32(math.pi / 180.0)
        o.polar = float(f32(q.polar) * deg2rad)
        o.azimuth = float(f32(q.azimuth) * deg2rad)
        o.mt[:] = [float(v) for v in q.mt]
        # time_integration may depend on the mechanism (elastic media differentiate
        # the STF of explosion and moment-tensor sources, module_vars.f90:472-477)
        ti = time_integration(q.mechanism) if callable(time_integration) else time_integration
        stf, hnt = prepare_stf(q, dt, f0factor, ti)
        stf = np.ascontiguousarray(stf, dtype=f32)
        self._keep.append(stf)
        o.stf = stf.ctypes.data_as(C.POINTER(C.c_float))
        o.nt_stf = len(stf)
        o.nbeg = nint(f32(q.t0) / f32(dt)) + 1
        self.hnt_last = hnt

    @property
    def nshots(self) -> int:
        return len(self.shots)

    def nrec(self, s: int) -> int:
        return self.arr[s].nrec


# --------------------------- geometry file I/O -------------------------------
def write_geometry(geom_dir: str, shots: Sequence[Shot]) -> str:
    """Write OWL's geometry.txt plus one file per shot (load_geometry's format)."""
    os.makedirs(geom_dir, exist_ok=True)
    with open(os.path.join(geom_dir, "geometry.txt"), "w") as f:
        for sh in shots:
            f.write(f"shot_{sh.id}_geometry.txt\n")
    for sh in shots:
        with open(os.path.join(geom_dir, f"shot_{sh.id}_geometry.txt"), "w") as f:
            f.write(f"{sh.id}\n{len(sh.sources)}\n")
            for s in sh.sources:
                f.write(f"{s.x} {s.y} {s.z}\n")
                if s.mechanism == "force":
                    f.write(f"force {s.polar} {s.azimuth}\n")
                elif s.mechanism == "mt":
                    f.write("mt " + " ".join(str(v) for v in s.mt) + "\n")
                else:
                    f.write("explosion\n")
                f.write(f"{s.wavelet} {s.f0} {s.amp} {s.t0}\n")
                f.write("0 0\n")
            f.write(f"{len(sh.receivers)}\n")
            for r in sh.receivers:
                f.write(f"{r.x} {r.y} {r.z} {r.weight}\n")
    return os.path.join(geom_dir, "geometry.txt")


def load_geometry(file_geometry: str, ns: Optional[int] = None) -> List[Shot]:
    """Read OWL's geometry files (module_source_receiver.f90:183-276)."""
    d = os.path.dirname(os.path.abspath(file_geometry))
    with open(file_geometry) as f:
        names = [ln.strip() for ln in f if ln.strip()]
    if ns is not None:
        names = names[:ns]
    shots = []
    for name in names:
        with open(os.path.join(d, name)) as f:
            lines = [ln.strip() for ln in f if ln.strip()]
        it = iter(lines)
        sid = int(next(it).split()[0])
        nsrc = int(next(it).split()[0])
        srcs = []
        for _ in range(nsrc):
            x, y, z = (float(v) for v in next(it).split()[:3])
            mech = next(it).split()
            s = Source(x=x, y=y, z=z, mechanism=mech[0])
            if mech[0] == "force":
                s.polar = float(mech[1]) if len(mech) > 1 else 0.0
                s.azimuth = float(mech[2]) if len(mech) > 2 else 0.0
            elif mech[0] == "mt":
                s.mt = tuple(float(v) for v in mech[1:7])
            w = next(it).split()
            s.wavelet, s.f0, s.amp, s.t0 = w[0], float(w[1]), float(w[2]), float(w[3])
            if s.wavelet == "custom":
                next(it)
            next(it)  # filtering frequencies
            srcs.append(s)
        nrec = int(next(it).split()[0])
        recs = []
        for _ in range(nrec):
            x, y, z, wgt = (float(v) for v in next(it).split()[:4])
            recs.append(Receiver(x=x, y=y, z=z, weight=wgt))
        shots.append(Shot(id=sid, sources=srcs, receivers=recs))
    return shots


def apply_offset_window(shot: Shot, offset_max: float, offset_min: float = 0.0) -> Shot:
    """Zero receiver weights outside [offset_min, offset_max] of absolute offset
    from the shot's first source (load_geometry's offset selection, :239-258)."""
    s0 = shot.sources[0]
    recs = []
    for r in shot.receivers:
        aoff = math.sqrt((r.x - s0.x) ** 2 + (r.y - s0.y) ** 2 + (r.z - s0.z) ** 2)
        w = r.weight if offset_min <= aoff <= offset_max else 0.0
        recs.append(Receiver(x=r.x, y=r.y, z=r.z, weight=w))
    return Shot(id=shot.id, sources=shot.sources, receivers=recs)
