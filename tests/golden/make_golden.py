"""Generates tests/golden/ac2d_golden.npz: FP64 oracle seismograms, misfit and
exact gradient of a small fixed case (regression fixtures; the reference ships
no golden data). Run: python tests/golden/make_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def golden_case():
    from cases import desc, prepare, random_model, small_shots
    import oracle
    nx, nz, dx, dt, nt = 36, 30, 10.0, 1e-3, 160
    d = desc(nx, nz, dx, dt, nt, pml=8)
    vp, rho = random_model(nx, nz, seed=11)
    ps = prepare(small_shots(nx, nz, dx), nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp * np.float32(1.05), rho, ps, "f64")
    return d, vp, rho, ps, obs


if __name__ == "__main__":
    import oracle
    d, vp, rho, ps, obs = golden_case()
    seis = oracle.ac2d_forward(d, vp, rho, ps, "f64")
    mf, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=20)
    np.savez_compressed(os.path.join(HERE, "ac2d_golden.npz"), seis=seis, grad=g, misfit=mf)
    print("wrote", os.path.join(HERE, "ac2d_golden.npz"), seis.shape, g.shape)
