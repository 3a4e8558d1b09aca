"""ctypes binding of the C ABI declared in include/owl_ssg.h.

The shared library ``owl_b200/lib/libowl_ssg.so`` is built in-tree by
``owl_b200.build.build_library()``. There is no fallback: if the library is
missing or has no usable sm_100a device, the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libowl_ssg.so")

OWL_OK = 0
OWL_ERR_INVALID = -1
OWL_ERR_CUDA = -2
OWL_ERR_OOM = -3
OWL_ERR_NONFINITE = -4
OWL_ERR_UNSTABLE = -5
OWL_ERR_TIMEOUT = -6
OWL_ERR_UNSUPPORTED = -7
OWL_ERR_NO_DEVICE = -8

OWL_ACOUSTIC_ISO_2D = 1
OWL_ACOUSTIC_ISO_3D = 2
OWL_ELASTIC_VHTIORT_2D = 3
OWL_ELASTIC_VHTIORT_3D = 4

OWL_ANISO_ISO = 0
OWL_ANISO_THOMSEN = 1
OWL_ANISO_AT = 2
OWL_ANISO_CIJ = 3

OWL_SRC_EXPLOSION = 0
OWL_SRC_FORCE = 1
OWL_SRC_MT = 2

OWL_MEM_HOST = 0
OWL_MEM_DEVICE = 1

OWL_CKPT_FP32 = 0
OWL_CKPT_FP16 = 1
OWL_CKPT_BF16 = 2

OWL_ADJ_L2_RESIDUAL = 0
OWL_ADJ_GIVEN = 1

OWL_MISFIT_WAVEFORM = 0
OWL_MISFIT_CORR = 1
OWL_MISFIT_ENVELOPE = 2
OWL_MISFIT_PHASE = 3
OWL_MISFIT_ADAPTIVE = 4
OWL_MISFIT_DTW = 5
OWL_MISFIT_LOCAL_ADAPTIVE = 6
OWL_MISFIT_ADAPTIVE_SPACETIME = 7
OWL_MISFIT_DTW_VECTOR = 8

OWL_DTW_PHASE = 0
OWL_DTW_AMP = 1
OWL_DTW_PHASE_AMP = 2

OWL_PENALTY_LINEAR = 0
OWL_PENALTY_POWER = 1
OWL_PENALTY_GAUSSIAN = 2
OWL_PENALTY_EXP = 3

#: misfit_type names of the reference's parameter file
MISFIT_NAMES = {"waveform": OWL_MISFIT_WAVEFORM, "corr": OWL_MISFIT_CORR, "envelope": OWL_MISFIT_ENVELOPE,
                "phase": OWL_MISFIT_PHASE, "adaptive": OWL_MISFIT_ADAPTIVE, "dtw": OWL_MISFIT_DTW,
                "local-adaptive": OWL_MISFIT_LOCAL_ADAPTIVE, "adaptive-spacetime": OWL_MISFIT_ADAPTIVE_SPACETIME,
                "dtw-vector": OWL_MISFIT_DTW_VECTOR}
#: dtw_form names of the reference's parameter file
DTW_FORM_NAMES = {"phase": OWL_DTW_PHASE, "amp": OWL_DTW_AMP, "phase+amp": OWL_DTW_PHASE_AMP}
PENALTY_NAMES = {"linear": OWL_PENALTY_LINEAR, "power": OWL_PENALTY_POWER, "gaussian": OWL_PENALTY_GAUSSIAN,
                 "exp": OWL_PENALTY_EXP}

MEDIUM_NAMES = {
    "acoustic-iso": OWL_ACOUSTIC_ISO_2D,
    "acoustic-iso-3d": OWL_ACOUSTIC_ISO_3D,
    "elastic-vhtiort": OWL_ELASTIC_VHTIORT_2D,
    "elastic-vhtiort-3d": OWL_ELASTIC_VHTIORT_3D,
}


class OwlSsgDesc(C.Structure):
    _fields_ = [
        ("medium", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
        ("pml", C.c_int),
        ("fdhalf", C.c_int),
        ("free_surface", C.c_int),
        ("dt", C.c_float),
        ("nt", C.c_int),
        ("f0_max", C.c_float),
        ("max_shots", C.c_int),
        ("allow_dt_adjust", C.c_int),
        ("aniso", C.c_int),
        ("free_surface_dz_refine", C.c_float),
        ("dz_max", C.c_float),
        ("free_surface_refine_rows", C.c_int),
    ]


_F9 = C.c_float * 9


class OwlSource(C.Structure):
    _fields_ = [
        ("mechanism", C.c_int),
        ("gx", C.c_int), ("gy", C.c_int), ("gz", C.c_int),
        ("hx", C.c_int), ("hy", C.c_int), ("hz", C.c_int),
        ("interp_ix", _F9), ("interp_iy", _F9), ("interp_iz", _F9),
        ("interp_hx", _F9), ("interp_hy", _F9), ("interp_hz", _F9),
        ("amp", C.c_float),
        ("polar", C.c_float), ("azimuth", C.c_float),
        ("mt", C.c_float * 6),
        ("nbeg", C.c_int),
        ("nt_stf", C.c_int),
        ("stf", C.POINTER(C.c_float)),
    ]


class OwlReceiver(C.Structure):
    _fields_ = [
        ("gx", C.c_int), ("gy", C.c_int), ("gz", C.c_int),
        ("hx", C.c_int), ("hy", C.c_int), ("hz", C.c_int),
        ("interp_ix", _F9), ("interp_iy", _F9), ("interp_iz", _F9),
        ("interp_hx", _F9), ("interp_hy", _F9), ("interp_hz", _F9),
        ("weight", C.c_float),
    ]


class OwlShot(C.Structure):
    _fields_ = [
        ("id", C.c_int),
        ("nsrc", C.c_int),
        ("src", C.POINTER(OwlSource)),
        ("nrec", C.c_int),
        ("rec", C.POINTER(OwlReceiver)),
    ]


class OwlRunOpts(C.Structure):
    _fields_ = [
        ("shots_per_launch", C.c_int),
        ("checkpoint_interval", C.c_int),
        ("checkpoint_precision", C.c_int),
        ("use_graph", C.c_int),
        ("shots_per_cta", C.c_int),
        ("tile_x", C.c_int), ("tile_z", C.c_int),
        ("check_every", C.c_int),
    ]


class OwlMisfitOpts(C.Structure):
    _fields_ = [
        ("misfit", C.c_int),
        ("dt", C.c_float),
        ("tlag_max", C.c_float),
        ("penalty", C.c_int),
        ("penalty_power", C.c_float),
        ("deconv_eps", C.c_float),
        ("discard_threshold", C.c_float),
        ("dtw_form", C.c_int),
        ("dtw_niter", C.c_int),
        ("dtw_trc", C.c_int),
        ("dtw_rinst", C.c_float),
        ("dtw_rcuml", C.c_float),
        ("dtw_epsabs", C.c_float),
        ("dtw_epsrel", C.c_float),
        ("dtw_loss_power", C.c_float),
        ("dtw_amp_weight", C.c_float),
        ("lawi_sigma", C.c_float),
        ("adaptive_half_window", C.c_int),
        ("ncomp", C.c_int),
        ("adj_nt", C.c_int),
    ]


class OwlRunInfo(C.Structure):
    _fields_ = [
        ("elapsed_ms", C.c_double),
        ("steps_cell_updates", C.c_double),
        ("gpu_launches", C.c_longlong),
        ("dt_used", C.c_float),
        ("dt_stable", C.c_float),
        ("shots_per_cta", C.c_int),
        ("tile_x", C.c_int), ("tile_z", C.c_int),
        ("batches", C.c_int),
        ("checkpoint_interval", C.c_int), ("shots_per_launch", C.c_int), ("tile_z_forward", C.c_int),
        ("shots_per_cta_forward", C.c_int),
    ]


#: every symbol include/owl_ssg.h declares
EXPORTED = [
    "owl_ssg_create", "owl_ssg_set_model", "owl_ssg_forward", "owl_ssg_gradient",
    "owl_ssg_source_gradient", "owl_ssg_destroy", "owl_last_error", "owl_ssg_abi_version",
    "owl_ssg_dt_stable", "owl_ssg_nparam", "owl_ssg_ncomp", "owl_ssg_device_ok", "owl_ssg_kernel_time",
    "owl_ssg_forward_noalloc", "owl_ssg_desc_nparam", "owl_ssg_misfit", "owl_ssg_gradient_misfit",
    "owl_adjoint_source", "owl_dtw_time_shifts", "owl_ssg_set_data_sampling", "owl_resample_traces",
    "owl_su_encode", "owl_su_decode", "owl_search_direction", "owl_grad_process",
    "owl_mpml_damp_ratio", "owl_ssg_mpml_ratios", "owl_vertical_mesh", "owl_free_surface_refine_rows",
]

OWL_SEARCH_SD = 0
OWL_SEARCH_CG = 1
OWL_SEARCH_LBFGS = 2
#: search_method names of the reference's parameter file
SEARCH_NAMES = {"sd": OWL_SEARCH_SD, "steepest-descent": OWL_SEARCH_SD, "cg": OWL_SEARCH_CG,
                "conjugate-gradient": OWL_SEARCH_CG, "l-bfgs": OWL_SEARCH_LBFGS}

OWL_GRAD_SMOOTH = 0
OWL_GRAD_TAPER = 1
OWL_GRAD_MASK = 2
OWL_GRAD_SCALE = 3
OWL_GRAD_MAX_BALANCE = 4
OWL_GRAD_RMS_BALANCE = 5
OWL_GRAD_RMS_BALANCE_AXIS = 6
OWL_GRAD_MEDIAN = 7

OWL_K_FWD_P = 0
OWL_K_FWD_V = 1
OWL_K_ADJ_P = 2
OWL_K_ADJ_V = 3
OWL_K_FWD_P_STORE = 4
OWL_K_FWD_V_STORE = 5


class OwlError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"owl status {code}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is not built; run owl_b200.build.build_library()")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    lib.owl_ssg_create.argtypes = [P(OwlSsgDesc), P(C.c_void_p)]
    lib.owl_ssg_set_model.argtypes = [C.c_void_p, C.c_int, P(P(C.c_float))]
    lib.owl_ssg_forward.argtypes = [C.c_void_p, C.c_int, P(OwlShot), P(OwlRunOpts), C.c_void_p, C.c_int,
                                    P(OwlRunInfo)]
    lib.owl_ssg_gradient.argtypes = [C.c_void_p, C.c_int, P(OwlShot), C.c_void_p, C.c_int, P(OwlRunOpts),
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, P(OwlRunInfo)]
    lib.owl_ssg_source_gradient.argtypes = [C.c_void_p, C.c_int, P(OwlShot), C.c_void_p, P(OwlRunOpts),
                                            C.c_void_p, C.c_int, P(OwlRunInfo)]
    lib.owl_ssg_kernel_time.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_double), P(C.c_double)]
    lib.owl_ssg_kernel_time.restype = C.c_int
    lib.owl_mpml_damp_ratio.argtypes = [P(C.c_float), C.c_int]
    lib.owl_mpml_damp_ratio.restype = C.c_float
    lib.owl_ssg_mpml_ratios.argtypes = [C.c_void_p, P(C.c_float)]
    lib.owl_ssg_mpml_ratios.restype = C.c_int
    lib.owl_ssg_forward_noalloc.argtypes = [P(OwlSsgDesc), C.c_int, P(P(C.c_float)), P(OwlShot), C.c_void_p]
    lib.owl_ssg_forward_noalloc.restype = C.c_int
    lib.owl_ssg_destroy.argtypes = [C.c_void_p]
    lib.owl_ssg_destroy.restype = None
    lib.owl_last_error.restype = C.c_char_p
    lib.owl_ssg_dt_stable.argtypes = [C.c_void_p]
    lib.owl_ssg_dt_stable.restype = C.c_float
    lib.owl_ssg_desc_nparam.argtypes = [P(OwlSsgDesc)]
    lib.owl_ssg_misfit.argtypes = [C.c_void_p, C.c_int, P(OwlShot), C.c_void_p, P(OwlRunOpts), C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_int, P(OwlRunInfo)]
    lib.owl_ssg_gradient_misfit.argtypes = [C.c_void_p, C.c_int, P(OwlShot), C.c_void_p, P(OwlMisfitOpts),
                                            P(OwlRunOpts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            P(OwlRunInfo)]
    lib.owl_adjoint_source.argtypes = [P(OwlMisfitOpts), C.c_int, P(C.c_int), C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    lib.owl_dtw_time_shifts.argtypes = [P(OwlMisfitOpts), C.c_int, P(C.c_int), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int]
    lib.owl_ssg_set_data_sampling.argtypes = [C.c_void_p, C.c_int, C.c_float]
    lib.owl_resample_traces.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_int, C.c_float,
                                        C.c_float, C.c_void_p, C.c_int]
    lib.owl_su_encode.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    lib.owl_su_decode.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    lib.owl_search_direction.argtypes = [C.c_int, C.c_longlong, C.c_int, P(C.c_void_p), P(C.c_void_p), C.c_void_p,
                                         C.c_void_p, C.c_int]
    lib.owl_grad_process.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_float), C.c_void_p, C.c_void_p,
                                     C.c_int]
    lib.owl_vertical_mesh.argtypes = [P(OwlSsgDesc), P(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.owl_free_surface_refine_rows.argtypes = [P(OwlSsgDesc), C.c_int, P(P(C.c_float)), C.c_float, P(C.c_int)]
    for fn in ("owl_vertical_mesh", "owl_free_surface_refine_rows", "owl_ssg_create", "owl_ssg_set_model", "owl_ssg_forward", "owl_ssg_gradient",
               "owl_ssg_source_gradient", "owl_ssg_abi_version", "owl_ssg_nparam", "owl_ssg_ncomp",
               "owl_ssg_device_ok", "owl_ssg_desc_nparam", "owl_ssg_misfit", "owl_ssg_gradient_misfit",
               "owl_adjoint_source", "owl_dtw_time_shifts", "owl_ssg_set_data_sampling", "owl_resample_traces",
               "owl_su_encode", "owl_su_decode", "owl_search_direction", "owl_grad_process"):
        getattr(lib, fn).restype = C.c_int
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != OWL_OK:
        msg = load().owl_last_error()
        raise OwlError(rc, msg.decode() if msg else "")
