"""CPU oracle: a C++ restatement of OWL's SSG loops (see oracle_ac2d.cpp).

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker. The product (owl_b200) never
imports it.
"""
from .oracle import (ORACLE_LIB, build, load, ac2d_forward, ac2d_gradient, ac2d_jvp, ac2d_ref_gradient,  # noqa: F401
                     ac3d_forward, ac3d_gradient, ac3d_jvp, el2d_forward, el2d_jvp, el2d_gradient, el2d_dt_stable,
                     el2d_damp_ratio, el2d_mesh, el3d_forward, el3d_jvp, el3d_gradient, el3d_dt_stable,
                     el3d_set_mpml)
