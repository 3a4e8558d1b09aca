"""Python handle over the C ABI (include/owl_ssg.h).

``SSGSolver`` is the batched, B200-first entry: many shots per call, model
set once, seismograms and gradients as numpy arrays (host) or torch CUDA
tensors (device, no host round trip).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L
from .geometry import GridSpec, PreparedShots, ZMesh

f32 = np.float32


@dataclass
class RunOpts:
    shots_per_launch: int = 0      # 0 = all shots of the call in one launch (<= max_shots)
    checkpoint_interval: int = 50  # >= nt: one segment, stored by the forward, no recompute; -1: sized to free memory
    checkpoint_precision: int = L.OWL_CKPT_FP32
    use_graph: int = 0             # 0 / 1: CUDA graphs on; -1: plain launches
    shots_per_cta: int = 0
    tile_x: int = 0
    tile_z: int = 0
    check_every: int = 0

    def c(self) -> L.OwlRunOpts:
        o = L.OwlRunOpts()
        for k in ("shots_per_launch", "checkpoint_interval", "checkpoint_precision", "use_graph",
                  "shots_per_cta", "tile_x", "tile_z", "check_every"):
            setattr(o, k, int(getattr(self, k)))
        return o


def _ptr(a) -> C.c_void_p:
    """host numpy array or torch tensor -> void*"""
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


def _mem_kind(a) -> int:
    if hasattr(a, "is_cuda") and a.is_cuda:
        return L.OWL_MEM_DEVICE
    return L.OWL_MEM_HOST


def _ready(*bufs) -> None:
    """Device buffers must be complete when a call starts (the library works on
    its own stream): wait for torch's current stream when any buffer is a CUDA
    tensor."""
    for b in bufs:
        if b is not None and hasattr(b, "is_cuda") and b.is_cuda:
            import torch
            torch.cuda.current_stream(b.device).synchronize()
            return


@dataclass
class MisfitOpts:
    """owl_misfit_opts: the reference's misfit_type and its parameters
    (src/lib/module_parameters.f90:550-570); zeros take the reference's defaults."""
    misfit: int = L.OWL_MISFIT_WAVEFORM
    dt: float = 0.0
    tlag_max: float = 0.0
    penalty: int = L.OWL_PENALTY_LINEAR
    penalty_power: float = 0.0
    deconv_eps: float = 0.0
    discard_threshold: float = 0.0
    dtw_form: int = L.OWL_DTW_PHASE
    dtw_niter: int = 0
    dtw_trc: int = 0
    dtw_rinst: float = 0.0
    dtw_rcuml: float = 0.0
    dtw_epsabs: float = 0.0
    dtw_epsrel: float = 0.0
    dtw_loss_power: float = 0.0
    dtw_amp_weight: float = 0.0
    lawi_sigma: float = 0.0
    adaptive_half_window: int = 0
    ncomp: int = 0
    adj_nt: int = 0

    def c(self) -> L.OwlMisfitOpts:
        o = L.OwlMisfitOpts()
        for k in ("misfit", "penalty", "dtw_form", "dtw_niter", "dtw_trc", "adaptive_half_window", "ncomp", "adj_nt"):
            setattr(o, k, int(getattr(self, k)))
        for k in ("dt", "tlag_max", "penalty_power", "deconv_eps", "discard_threshold", "dtw_rinst", "dtw_rcuml",
                  "dtw_epsabs", "dtw_epsrel", "dtw_loss_power", "dtw_amp_weight", "lawi_sigma"):
            setattr(o, k, float(getattr(self, k)))
        return o


def resample_traces(rows, din: float, dout: float, nout: int, oin: float = 0.0, oout: float = 0.0):
    """Cubic-convolution resampling of trace rows (ntr, nin) on the GPU
    (owl_resample_traces); numpy in -> numpy out, CUDA tensor in -> CUDA tensor out."""
    lib = L.load()
    ntr, nin = int(rows.shape[0]), int(rows.shape[1])
    if hasattr(rows, "is_cuda") and rows.is_cuda:
        import torch
        out = torch.empty((ntr, nout), dtype=torch.float32, device=rows.device)
        _ready(rows, out)
    else:
        rows = np.ascontiguousarray(rows, dtype=f32)
        out = np.empty((ntr, nout), dtype=f32)
    L.check(lib.owl_resample_traces(ntr, nin, din, oin, _ptr(rows), nout, dout, oout, _ptr(out), _mem_kind(rows)))
    return out


def adjoint_source(mopts: MisfitOpts, gather_ptr, syn, obs, weight=None, adj=None, trace_misfit=None,
                   gather_misfit=None):
    """compute_adjoint_source on the GPU for traces given as rows (ntr, nt) of
    numpy arrays (host) or CUDA tensors (device); gathers are the row ranges
    gather_ptr[g] .. gather_ptr[g+1]-1. Returns (adj, trace misfits, gather misfits)."""
    lib = L.load()
    gp = np.ascontiguousarray(np.asarray(gather_ptr, dtype=np.int32))
    ng = gp.size - 1
    ntr, nt = int(syn.shape[0]), int(syn.shape[1])
    if hasattr(syn, "is_cuda") and syn.is_cuda:
        import torch
        dev = syn.device
        adj = torch.empty_like(syn) if adj is None else adj
        trace_misfit = torch.empty(ntr, dtype=torch.float64, device=dev) if trace_misfit is None else trace_misfit
        gather_misfit = torch.empty(ng, dtype=torch.float64, device=dev) if gather_misfit is None else gather_misfit
        _ready(syn, obs, weight, adj, trace_misfit, gather_misfit)
    else:
        syn = np.ascontiguousarray(syn, dtype=f32)
        obs = np.ascontiguousarray(obs, dtype=f32)
        weight = None if weight is None else np.ascontiguousarray(weight, dtype=f32)
        adj = np.empty_like(syn) if adj is None else adj
        trace_misfit = np.empty(ntr) if trace_misfit is None else trace_misfit
        gather_misfit = np.empty(ng) if gather_misfit is None else gather_misfit
    o = mopts.c()
    L.check(lib.owl_adjoint_source(C.byref(o), ng, gp.ctypes.data_as(C.POINTER(C.c_int)), nt, _ptr(syn), _ptr(obs),
                                   _ptr(weight) if weight is not None else None, _ptr(adj), _ptr(trace_misfit),
                                   _ptr(gather_misfit), _mem_kind(syn)))
    return adj, trace_misfit, gather_misfit


def dtw_time_shifts(mopts: MisfitOpts, gather_ptr, syn, obs, weight=None, tau=None):
    """Time shifts tau(t) of the DTW misfit (owl_dtw_time_shifts), obs(t + tau) ~
    syn(t), in seconds, rows like syn; numpy in -> numpy out, CUDA tensors in ->
    CUDA tensor out."""
    lib = L.load()
    gp = np.ascontiguousarray(np.asarray(gather_ptr, dtype=np.int32))
    ng = gp.size - 1
    if hasattr(syn, "is_cuda") and syn.is_cuda:
        import torch
        tau = torch.empty_like(syn) if tau is None else tau
        _ready(syn, obs, weight, tau)
    else:
        syn = np.ascontiguousarray(syn, dtype=f32)
        obs = np.ascontiguousarray(obs, dtype=f32)
        weight = None if weight is None else np.ascontiguousarray(weight, dtype=f32)
        tau = np.empty_like(syn) if tau is None else tau
    o = mopts.c()
    L.check(lib.owl_dtw_time_shifts(C.byref(o), ng, gp.ctypes.data_as(C.POINTER(C.c_int)), int(syn.shape[1]),
                                    _ptr(syn), _ptr(obs), _ptr(weight) if weight is not None else None, _ptr(tau),
                                    _mem_kind(syn)))
    return tau


def elastic_time_integration(mechanism: str) -> int:
    """STF time integration of the elastic media: explosion and moment-tensor
    sources inject the derivative of the wavelet as a stress drop."""
    return -1 if mechanism in ("explosion", "mt") else 0


def elastic_geometry(shots, desc, zmesh=None):
    """With a free surface, sources above the first row's spacing (z < dz_i(1):
    dz, or dz / free_surface_dz_refine on the refined mesh) are moved to that
    depth and their amplitude multiplied by 1.2 (module_vars.f90:463-466)."""
    if not desc.free_surface:
        return shots
    dz = np.float32(desc.dz) if zmesh is None else np.float32(zmesh.at(zmesh.dz_i, 1))
    out = []
    for sh in shots:
        srcs = [replace(q, z=float(dz), amp=float(np.float32(q.amp) * np.float32(1.2))) if np.float32(q.z) < dz else q
                for q in sh.sources]
        out.append(replace(sh, sources=srcs))
    return out


def mesh_is_refined(desc) -> bool:
    """A free-surface descriptor whose vertical mesh is not the uniform grid."""
    rr = desc.free_surface_dz_refine if desc.free_surface_dz_refine > 0 else 1.0
    cap = desc.dz_max if desc.dz_max > 0 else desc.dz
    return bool(desc.free_surface) and (rr != 1.0 or cap != desc.dz)


def vertical_mesh(desc) -> Optional[ZMesh]:
    """Rows of the depth-refined free-surface mesh of a descriptor
    (owl_vertical_mesh), None on the uniform grid."""
    if not mesh_is_refined(desc):
        return None
    lib = L.load()
    n = C.c_int()
    L.check(lib.owl_vertical_mesh(C.byref(desc), C.byref(n), None, None, None, None))
    arr = [np.zeros(n.value + 2 * desc.pml + 2, dtype=f32) for _ in range(4)]
    L.check(lib.owl_vertical_mesh(C.byref(desc), C.byref(n), *[a.ctypes.data_as(C.c_void_p) for a in arr]))
    return ZMesh(int(desc.pml), *arr)


def free_surface_refine_rows(desc, fields, f0_min: float) -> int:
    """refine_nz of the refined mesh from the model's surface row and the lowest
    source f0 (module_vars.f90:315-317); fields as owl_ssg_set_model takes them."""
    lib = L.load()
    keep = [np.asfortranarray(np.asarray(f, dtype=f32)) for f in fields]
    arr = (C.POINTER(C.c_float) * len(keep))()
    for i, f in enumerate(keep):
        arr[i] = f.ctypes.data_as(C.POINTER(C.c_float))
    rows = C.c_int()
    L.check(lib.owl_free_surface_refine_rows(C.byref(desc), len(keep), arr, float(f0_min), C.byref(rows)))
    return int(rows.value)


class SSGSolver:
    """One solver handle: grid, PML, time axis and model of one medium.

    Elastic 2D with a free surface may run on the reference's depth-refined
    vertical mesh: free_surface_dz_refine (rows dz / refine apart at the
    surface), dz_max (largest spacing) and refine_rows (the reference's
    refine_nz, free_surface_refine_rows()). The model and the gradient stay on
    the regular (nz, nx) grid; prepare() places sources and receivers on the
    mesh rows."""

    def __init__(self, medium: int, nx: int, nz: int, dx: float, dz: float, dt: float, nt: int,
                 pml: int = 15, fdhalf: int = 4, free_surface: bool = False, f0_max: float = 20.0,
                 max_shots: int = 1, ny: int = 1, dy: float = 0.0, ox: float = 0.0, oy: float = 0.0,
                 oz: float = 0.0, allow_dt_adjust: bool = False, aniso: int = 0,
                 free_surface_dz_refine: float = 0.0, dz_max: float = 0.0, refine_rows: int = 0):
        self.lib = L.load()
        d = L.OwlSsgDesc()
        d.medium = medium
        d.nx, d.ny, d.nz = nx, ny, nz
        d.dx, d.dy, d.dz = dx, (dy if dy else dx), dz
        d.ox, d.oy, d.oz = ox, oy, oz
        d.pml, d.fdhalf, d.free_surface = pml, fdhalf, int(bool(free_surface))
        d.dt, d.nt, d.f0_max = dt, nt, f0_max
        d.max_shots = max_shots
        d.allow_dt_adjust = int(bool(allow_dt_adjust))
        d.aniso = int(aniso)
        d.free_surface_dz_refine = float(free_surface_dz_refine)
        d.dz_max = float(dz_max)
        d.free_surface_refine_rows = int(refine_rows)
        self.desc = d
        self.grid = GridSpec(nx=nx, nz=nz, dx=dx, dz=dz, ox=ox, oz=oz, ny=ny, dy=(dy if dy else dx), oy=oy,
                             zmesh=vertical_mesh(d))
        h = C.c_void_p()
        L.check(self.lib.owl_ssg_create(C.byref(d), C.byref(h)))
        self.h = h
        self.ncomp = self.lib.owl_ssg_ncomp(medium)
        self.nparam = self.lib.owl_ssg_desc_nparam(C.byref(d))
        self.last_info = L.OwlRunInfo()
        self.data_nt, self.data_dt = 0, 0.0

    def close(self):
        if getattr(self, "h", None):
            self.lib.owl_ssg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dt_stable(self) -> float:
        return float(self.lib.owl_ssg_dt_stable(self.h))

    def set_model(self, *fields: np.ndarray) -> None:
        """fields: (nz, nx) [or (nz, ny, nx)] arrays in the order of owl_ssg_set_model."""
        self._model = [np.asfortranarray(np.asarray(f, dtype=f32)) for f in fields]
        arr = (C.POINTER(C.c_float) * len(self._model))()
        for i, f in enumerate(self._model):
            arr[i] = f.ctypes.data_as(C.POINTER(C.c_float))
        L.check(self.lib.owl_ssg_set_model(self.h, len(self._model), arr))

    def prepare(self, shots, f0factor: float = 1.0, time_integration=None) -> PreparedShots:
        """Sources and receivers on the grid (prepare_geometry / prepare_stf). For the
        elastic medium the STF of explosion and moment-tensor sources is
        differentiated (time_integration = -1) and, with a free surface, sources
        shallower than the first grid step move down to it with 1.2 x amplitude
        (src/solver/elastic_vhtiort_2d/module_vars.f90:466-477)."""
        if self.desc.medium in (L.OWL_ELASTIC_VHTIORT_2D, L.OWL_ELASTIC_VHTIORT_3D):
            shots = elastic_geometry(shots, self.desc, self.grid.zmesh)
            if time_integration is None:
                time_integration = elastic_time_integration
        return PreparedShots(shots, self.grid, self.desc.dt, f0factor,
                             0 if time_integration is None else time_integration)

    def set_data_sampling(self, data_nt: int, data_dt: float) -> None:
        """Traces in and out at data_nt samples of data_dt (data_nt <= 0: the time axis)."""
        L.check(self.lib.owl_ssg_set_data_sampling(self.h, int(data_nt), float(data_dt)))
        self.data_nt, self.data_dt = (int(data_nt), float(data_dt)) if data_nt > 0 else (0, 0.0)

    @property
    def trace_nt(self) -> int:
        """samples per trace of the seismograms the solver takes and returns"""
        return self.data_nt if self.data_nt > 0 else self.desc.nt

    def seis_size(self, ps: PreparedShots) -> int:
        return sum(ps.nrec(s) for s in range(ps.nshots)) * self.ncomp * self.trace_nt

    def split(self, ps: PreparedShots, flat) -> List:
        """flat seismogram buffer -> per-shot (ncomp, nrec, nt) views"""
        out, off = [], 0
        nt = self.trace_nt
        for s in range(ps.nshots):
            n = ps.nrec(s) * self.ncomp * nt
            out.append(flat[off:off + n].reshape(self.ncomp, ps.nrec(s), nt))
            off += n
        return out

    def forward(self, ps: PreparedShots, opts: Optional[RunOpts] = None, out=None):
        """Seismograms of all shots; returns the flat buffer (numpy or torch)."""
        opts = opts or RunOpts()
        if out is None:
            out = np.zeros(self.seis_size(ps), dtype=f32)
        o = opts.c()
        _ready(out)
        L.check(self.lib.owl_ssg_forward(self.h, ps.nshots, ps.arr, C.byref(o), _ptr(out), _mem_kind(out),
                                         C.byref(self.last_info)))
        return out

    def gradient(self, ps: PreparedShots, data, adj_kind: int = L.OWL_ADJ_L2_RESIDUAL,
                 opts: Optional[RunOpts] = None, grad=None, misfit=None, seis_out=None):
        """Stacked gradient of 0.5 * sum (syn - obs)^2 (or of <syn, adj> for OWL_ADJ_GIVEN).

        Returns (misfit per shot, gradient (nparam, nz*nx) flat buffer)."""
        opts = opts or RunOpts()
        nm = self.desc.nx * self.desc.nz * max(1, self.desc.ny)
        dev = _mem_kind(data) == L.OWL_MEM_DEVICE
        if grad is None:
            if dev:
                import torch
                grad = torch.zeros(self.nparam * nm, dtype=torch.float32, device=data.device)
                misfit = torch.zeros(ps.nshots, dtype=torch.float64, device=data.device)
            else:
                grad = np.zeros(self.nparam * nm, dtype=f32)
                misfit = np.zeros(ps.nshots, dtype=np.float64)
        o = opts.c()
        _ready(data, grad, misfit, seis_out)
        L.check(self.lib.owl_ssg_gradient(self.h, ps.nshots, ps.arr, _ptr(data), adj_kind, C.byref(o),
                                          _ptr(misfit) if misfit is not None else None, _ptr(grad),
                                          _ptr(seis_out) if seis_out is not None else None,
                                          _mem_kind(data), C.byref(self.last_info)))
        return misfit, grad

    def gradient_misfit(self, ps: PreparedShots, obs, mopts: MisfitOpts, opts: Optional[RunOpts] = None,
                        grad=None, misfit=None, seis_out=None):
        """Stacked gradient of 0.5 * the data-domain misfit `mopts` (the adjoint
        source and the trace selection of compute_adjoint_source, on the GPU).
        Returns (misfit per shot, gradient flat buffer)."""
        opts = opts or RunOpts()
        nm = self.desc.nx * self.desc.nz * max(1, self.desc.ny)
        if grad is None:
            if _mem_kind(obs) == L.OWL_MEM_DEVICE:
                import torch
                grad = torch.zeros(self.nparam * nm, dtype=torch.float32, device=obs.device)
                misfit = torch.zeros(ps.nshots, dtype=torch.float64, device=obs.device)
            else:
                grad = np.zeros(self.nparam * nm, dtype=f32)
                misfit = np.zeros(ps.nshots, dtype=np.float64)
        o, mo = opts.c(), mopts.c()
        _ready(obs, grad, misfit, seis_out)
        L.check(self.lib.owl_ssg_gradient_misfit(self.h, ps.nshots, ps.arr, _ptr(obs), C.byref(mo), C.byref(o),
                                                 _ptr(misfit) if misfit is not None else None, _ptr(grad),
                                                 _ptr(seis_out) if seis_out is not None else None,
                                                 _mem_kind(obs), C.byref(self.last_info)))
        return misfit, grad

    def gather_ptr(self, ps: PreparedShots) -> np.ndarray:
        """row ranges of the (shot, component) gathers in the seismogram layout"""
        gp = [0]
        for s in range(ps.nshots):
            for _ in range(self.ncomp):
                gp.append(gp[-1] + ps.nrec(s))
        return np.asarray(gp, dtype=np.int32)

    def grad_fields(self, grad) -> List[np.ndarray]:
        """flat gradient -> list of (nz, nx) [or (nz, ny, nx)] arrays (z fastest like OWL files)"""
        d = self.desc
        shape = (d.nz, d.nx) if d.ny <= 1 else (d.nz, d.ny, d.nx)
        nm = int(np.prod(shape))
        g = grad if isinstance(grad, np.ndarray) else grad.detach().cpu().numpy()
        return [g[i * nm:(i + 1) * nm].reshape(tuple(reversed(shape))).T for i in range(self.nparam)]

    def source_gradient(self, ps: PreparedShots, adj: np.ndarray, opts: Optional[RunOpts] = None):
        opts = opts or RunOpts()
        nsrc = sum(ps.arr[s].nsrc for s in range(ps.nshots))
        out = np.zeros(nsrc * self.desc.nt, dtype=f32)
        o = opts.c()
        L.check(self.lib.owl_ssg_source_gradient(self.h, ps.nshots, ps.arr, _ptr(adj), C.byref(o), _ptr(out),
                                                 L.OWL_MEM_HOST, C.byref(self.last_info)))
        return out

    def misfit(self, ps: PreparedShots, obs, opts: Optional[RunOpts] = None, traces: bool = False,
               seis_out=None):
        """Misfit-only forward (step-length trial forwards): per-shot sum over traces of
        (obs - syn)^2, and with traces=True also the per-trace misfits."""
        opts = opts or RunOpts()
        misfit = np.zeros(ps.nshots)
        tm = np.zeros(sum(ps.nrec(s) for s in range(ps.nshots)) * self.ncomp) if traces else None
        o = opts.c()
        L.check(self.lib.owl_ssg_misfit(self.h, ps.nshots, ps.arr, _ptr(obs), C.byref(o), _ptr(misfit),
                                        _ptr(tm) if tm is not None else None,
                                        _ptr(seis_out) if seis_out is not None else None, L.OWL_MEM_HOST,
                                        C.byref(self.last_info)))
        return (misfit, tm) if traces else misfit

    def mpml_ratios(self) -> np.ndarray:
        """The six M-PML face-ratio arrays of an elastic 3D model (left, right,
        front, back, top, bottom; the layout of owl_ssg_mpml_ratios)."""
        d = self.desc
        m = self.grid.zmesh  # on the refined free-surface mesh the faces span its planes
        nzm = d.nz if m is None else len(m.z_i) - 2 * d.pml - 2
        nx, ny, nz = d.nx + 2 * d.pml, d.ny + 2 * d.pml, nzm + 2 * d.pml
        out = np.zeros(2 * (ny * nz + nx * nz + nx * ny), dtype=f32)
        L.check(self.lib.owl_ssg_mpml_ratios(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def kernel_time(self, kernel_id: int, nlaunch: int = 20) -> Tuple[float, float]:
        """(mean ms per launch, algorithmic bytes per launch) of one kernel on the last batch state."""
        ms, b = C.c_double(), C.c_double()
        L.check(self.lib.owl_ssg_kernel_time(self.h, kernel_id, nlaunch, C.byref(ms), C.byref(b)))
        return ms.value, b.value
