"""Drop-in host side for OWL's SSG solver path.

* ``WaveSolverAcousticIso2D`` mirrors ``type wave_solver_acoustic_iso_2d``
  (src/solver/acoustic_iso_2d/interface.f90:30-60): same public fields, and
  ``forward()`` / ``adjoint()`` with the reference's file contract
  (``<dir_synthetic>/shot_<id>_seismogram_p.su`` out of forward, adjoint source
  ``<dir_adjoint>/shot_<id>_seismogram_p.su`` in, per-shot gradients out).
* ``forward_modeling(param_file)`` mirrors ``owl_modeling2`` (src/forward/main_forward.f90,
  src/forward/2d/module_modeling.f90:49-242), all shots in batched launches.
* ``fwi_gradient(param_file)`` mirrors one gradient evaluation of ``owl_fwi2``
  (src/inverse/2d/module_gradient.f90:57-417): forward, L2 adjoint source,
  adjoint, stack, and writes ``iteration_1/model/grad_<name>.bin``.

Differences from the reference, by design: the adjoint is the exact discrete
transpose of the forward (every step, so cc_step_interval does not apply);
per-shot gradients are raw float32 (nz, nx) files instead of FLIT grid2 files.
"""
from __future__ import annotations

import os
from typing import List, Optional

import numpy as np

from . import _lib as L
from . import io as owlio
from .geometry import GridSpec, PreparedShots, Shot, apply_offset_window, load_geometry
from .solver import RunOpts, SSGSolver

f32 = np.float32


def _nint(v: float) -> int:
    return int(np.floor(v + 0.5)) if v >= 0 else -int(np.floor(-v + 0.5))


class WaveSolverAcousticIso2D:
    """Fields of wave_solver_acoustic_iso_2d; one shot (gmtr) per object."""

    def __init__(self):
        self.nx = 0
        self.nz = 0
        self.dx = 0.0
        self.dz = 0.0
        self.ox = 0.0
        self.oz = 0.0
        self.tmax = 1.0
        self.dt = 0.0
        self.data_tmax = 1.0
        self.data_dt = 0.0
        self.pml = 15
        self.free_surface = False
        self.vp: Optional[np.ndarray] = None
        self.rho: Optional[np.ndarray] = None
        self.dir_synthetic = "./"
        self.dir_adjoint = "./"
        self.dir_snapshot = "./"
        self.dir_working = "./"
        self.cc_step_interval = 1
        self.verbose = False
        self.snaps: List[float] = []
        self.gmtr: Optional[Shot] = None
        self.energy_precond = False
        self.reconstruct = False
        self.f0factor = 1.0
        self.seis_p: Optional[np.ndarray] = None
        self._solver: Optional[SSGSolver] = None

    @property
    def nt(self) -> int:
        return _nint(self.tmax / self.dt + 1)

    def _make(self) -> SSGSolver:
        f0 = max(s.f0 for s in self.gmtr.sources)
        s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, self.nx, self.nz, self.dx, self.dz, self.dt, self.nt, pml=self.pml,
                      free_surface=self.free_surface, f0_max=f0, max_shots=1, ox=self.ox, oz=self.oz)
        s.set_model(self.vp, self.rho)
        self._solver = s
        return s

    def forward(self) -> np.ndarray:
        s = self._make()
        ps = s.prepare([self.gmtr], f0factor=self.f0factor)
        seis = s.forward(ps).reshape(-1, self.nt)
        self.seis_p = seis
        owlio.write_su(os.path.join(self.dir_synthetic, f"shot_{self.gmtr.id}_seismogram_p.su"), seis, self.dt)
        return seis

    def adjoint(self):
        """Gradient of <syn, adj> for the adjoint source in dir_adjoint; writes
        shot_<id>_grad_{vp,rho}.bin to dir_working and returns (grad_vp, grad_rho)."""
        s = self._make()
        ps = s.prepare([self.gmtr], f0factor=self.f0factor)
        adj, _ = owlio.read_su(os.path.join(self.dir_adjoint, f"shot_{self.gmtr.id}_seismogram_p.su"))
        _, g = s.gradient(ps, np.ascontiguousarray(adj, dtype=f32).ravel(), adj_kind=L.OWL_ADJ_GIVEN,
                          opts=RunOpts(checkpoint_interval=50))
        gvp, grho = s.grad_fields(g)
        owlio.write_model(os.path.join(self.dir_working, f"shot_{self.gmtr.id}_grad_vp.bin"), gvp)
        owlio.write_model(os.path.join(self.dir_working, f"shot_{self.gmtr.id}_grad_rho.bin"), grho)
        return gvp, grho


class _Run:
    """Parameters of one run, read like read_parameters / set_regular_space."""

    def __init__(self, param_file: str):
        self.dir = os.path.dirname(os.path.abspath(param_file))
        p = owlio.read_param(param_file)
        self.p = p
        g = lambda k, d=None: p.get(k, d)
        self.nx, self.nz = int(g("nx")), int(g("nz"))
        self.dx, self.dz = float(g("dx")), float(g("dz"))
        self.ox, self.oz = float(g("ox", 0.0)), float(g("oz", 0.0))
        self.dt = float(g("dt"))
        self.tmax = float(g("tmax", 1.0))
        self.data_dt = float(g("data_dt", self.dt))
        self.ns = int(g("ns", 1))
        self.medium = g("which_medium", "acoustic-iso")
        if self.medium != "acoustic-iso":
            raise NotImplementedError(f"which_medium = {self.medium} is not built in this driver")
        self.pml = int(g("npml", 15))
        self.free_surface = owlio.param_bool(g("yn_free_surface", "n"))
        self.f0factor = float(g("f0_factor", 1.0))
        self.offset_min = float(g("offset_min", 0.0))
        self.offset_max = float(g("offset_max", 3.0e38))
        self.nt = _nint(self.tmax / self.dt + 1)
        if abs(self.data_dt - self.dt) > 1e-9 * self.dt:
            raise NotImplementedError("data_dt != dt (SU resampling) is not supported")
        names = owlio.param_list(g("model_name", "vp, rho"))
        self.model = {}
        for name in ("vp", "rho"):
            fk = g(f"file_{name}")
            if fk:
                self.model[name] = owlio.read_model(self._path(fk), (self.nz, self.nx))
            elif name in p:
                self.model[name] = np.full((self.nz, self.nx), float(p[name]), dtype=f32)
            elif name == "rho":
                self.model[name] = np.full((self.nz, self.nx), 1000.0, dtype=f32)
            else:
                raise ValueError(f"model {name} missing ({names})")
        shots = load_geometry(self._path(g("file_geometry")), self.ns)
        self.shots = [apply_offset_window(s, self.offset_max, self.offset_min) for s in shots]
        self.f0_max = max(src.f0 for s in self.shots for src in s.sources)

    def _path(self, v: str) -> str:
        return v if os.path.isabs(v) else os.path.join(self.dir, v)

    def solver(self) -> SSGSolver:
        s = SSGSolver(L.OWL_ACOUSTIC_ISO_2D, self.nx, self.nz, self.dx, self.dz, self.dt, self.nt, pml=self.pml,
                      free_surface=self.free_surface, f0_max=self.f0_max, max_shots=len(self.shots), ox=self.ox,
                      oz=self.oz)
        s.set_model(self.model["vp"], self.model["rho"])
        return s


def forward_modeling(param_file: str) -> List[np.ndarray]:
    """owl_modeling2: every shot, SU files in dir_synthetic; returns per-shot (nrec, nt) arrays."""
    r = _Run(param_file)
    s = r.solver()
    ps = s.prepare(r.shots, f0factor=r.f0factor)
    seis = s.split(ps, s.forward(ps))
    out_dir = r._path(r.p.get("dir_synthetic", "./data_synthetic"))
    for sh, d in zip(r.shots, seis):
        owlio.write_su(os.path.join(out_dir, f"shot_{sh.id}_seismogram_p.su"), d[0], r.dt)
    return [d[0] for d in seis]


def fwi_gradient(param_file: str):
    """One gradient evaluation of owl_fwi2 with the L2 waveform misfit: returns
    (misfit per shot, grad_vp, grad_rho) and writes iteration_1/model/grad_*.bin."""
    r = _Run(param_file)
    s = r.solver()
    ps = s.prepare(r.shots, f0factor=r.f0factor)
    rec_dir = r._path(r.p.get("dir_record", "./data_record"))
    obs = []
    for sh in r.shots:
        d, _ = owlio.read_su(os.path.join(rec_dir, f"shot_{sh.id}_seismogram_p.su"))
        obs.append(np.ascontiguousarray(d, dtype=f32).ravel())
    mf, g = s.gradient(ps, np.concatenate(obs), adj_kind=L.OWL_ADJ_L2_RESIDUAL, opts=RunOpts(checkpoint_interval=50))
    gvp, grho = s.grad_fields(g)
    wd = os.path.join(r._path(r.p.get("dir_working", "./test")), "iteration_1", "model")
    owlio.write_model(os.path.join(wd, "grad_vp.bin"), gvp)
    owlio.write_model(os.path.join(wd, "grad_rho.bin"), grho)
    return mf, gvp, grho
