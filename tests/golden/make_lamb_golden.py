"""Generates tests/golden/lamb_flat.npz from the reference's own Python: the
2D Lamb half-space surface particle velocities of its elastic free-surface
test (test/lamb_reference.py, `lamb_halfspace_velocity`, discrete-wavenumber
integration) for the flat surface of test/test_elastic_lamb.py (vp 3000,
vs 1732, rho 2000 kg/m3, 20 Hz Ricker, surface-normal force at the surface,
surface receivers at offsets 150 .. 550 m, 1 ms samples to 0.6 s), and the
reference's Ricker wavelet (`ricker_owl`) at the simulation step.

Run from the repository root where the reference tree is present:
    python tests/golden/make_lamb_golden.py <path of the reference's test/>
The fixture travels with the repository; the tests never read the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

VP, VS, RHO = 3000.0, 1732.0, 2000.0
F0 = 20.0
DT = 2.0e-4
DATA_DT = 1.0e-3
TMAX = 0.6
OFFSETS = np.array([150.0, 250.0, 350.0, 450.0, 550.0])


def main(ref_test_dir: str) -> None:
    sys.path.insert(0, ref_test_dir)
    import lamb_reference as lr  # the reference's own module

    nt_data = int(round(TMAX / DATA_DT)) + 1
    ref_n, ref_t = lr.lamb_halfspace_velocity(OFFSETS, nt_data, DATA_DT, VP, VS, RHO, F0)
    nt_sim = int(round(TMAX / DT)) + 1
    stf = lr.ricker_owl(nt_sim, DT, F0)
    np.savez_compressed(os.path.join(HERE, "lamb_flat.npz"), ref_n=np.asarray(ref_n, dtype=np.float64),
                        ref_t=np.asarray(ref_t, dtype=np.float64), offsets=OFFSETS, vp=VP, vs=VS, rho=RHO, f0=F0,
                        dt=DT, data_dt=DATA_DT, tmax=TMAX, stf=np.asarray(stf, dtype=np.float64))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join("/root/reference", "test"))
