"""owl_b200 -- B200-native standard-staggered-grid finite-difference modelling
and adjoint-state FWI gradients, a drop-in for the SSG solver path of LANL OWL.

The compute path is the CUDA library ``lib/libowl_ssg.so`` (sm_100a), reached
through the C ABI in ``include/owl_ssg.h``. This package holds the host-side
mirror of OWL's interfaces: geometry / source preparation, parameter and SU
files, and solver objects with OWL's forward / adjoint methods.
"""
from . import _lib
from .geometry import (GridSpec, PreparedShots, Receiver, Shot, Source, apply_offset_window,
                       kaiser_sinc_kernel, load_geometry, prepare_stf, write_geometry)
from .solver import RunOpts, SSGSolver

__all__ = [
    "GridSpec", "PreparedShots", "Receiver", "Shot", "Source", "apply_offset_window", "kaiser_sinc_kernel",
    "load_geometry", "prepare_stf", "write_geometry", "RunOpts", "SSGSolver", "_lib",
]
