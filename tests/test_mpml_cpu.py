"""The library's M-PML damping-ratio search (owl_mpml_damp_ratio, host code:
the 27 x 27 split-field eigen-derivative reduced to the 3 x 3 Christoffel
problem) against the oracle's literal restatement of damp_ratio and
mpml_eigenvalue_derivative (src/solver/elastic_vhtiort_3d/module_cfspml.f90:
51-248, numpy.linalg.eig on the full 27 x 27 system). The search steps the
ratio by 2e-3 and its decisions are threshold comparisons of single- vs
double-precision derivatives, so the two may differ by one step."""
import numpy as np
import pytest

from oracle import oracle_mpml as M
from owl_b200 import _lib as L

STEP = 2.0e-3


def lib_ratio(c, axis):
    lib = L.load()
    cc = np.ascontiguousarray(c, dtype=np.float32)
    return float(lib.owl_mpml_damp_ratio(cc.ctypes.data_as(L.C.POINTER(L.C.c_float)), axis))


def ort(vp, vs, rho, f11=1.0, f22=1.0, f55=1.0, f66=1.0):
    lam, mu = rho * (vp ** 2 - 2 * vs ** 2), rho * vs ** 2
    return np.array([(lam + 2 * mu) * f11, lam, lam, (lam + 2 * mu) * f22, lam, lam + 2 * mu, mu, mu * f55, mu * f66],
                    dtype=np.float32)


def test_eigen_derivative_reduction_matches_27x27():
    """The literal derivative and the reduced form agree (the reduction the
    library evaluates), for random directions, axes and ratios."""
    rng = np.random.default_rng(4)
    c = ort(3000.0, 3000.0 / 1.73, 2300.0, 1.12, 1.05, 1.1, 1.15).astype(np.float64)
    for _ in range(8):
        k = rng.standard_normal(3)
        k /= np.linalg.norm(k)
        d, r = "xyz"[int(rng.integers(3))], float(0.3 * rng.random())
        lit = M.mpml_eigenvalue_derivative(c, d, r, *k)
        red = M.reduced_eigenvalue_derivative(c, d, r, *k)
        assert abs(lit - red) <= 1e-12 * max(1.0, abs(lit)), (lit, red)


@pytest.mark.parametrize("cell", [0, 1])
def test_damp_ratio_matches_literal_search(cell):
    if cell == 0:
        c = ort(3000.0, 3000.0 / 1.73, 2300.0, 1.12, 1.05, 1.1, 1.15)   # the benchmark's kind of ORT cell
    else:
        c = ort(2500.0, 2500.0 / 2.4, 2100.0, 1.3, 0.9, 1.4, 0.8)       # strong anisotropy
    for axis in range(3):
        want = M.damp_ratio(c, "xyz"[axis])
        got = lib_ratio(c, axis)
        assert abs(got - want) <= STEP + 1e-7, (axis, got, want)
        assert got >= STEP - 1e-7


def test_isotropic_stiffness():
    """An isotropic stiffness given as Cij still gets the search's ratio (the
    reference skips the search only for the iso parameterisation): directions
    almost perpendicular to the damped axis need ratio >= 0.01."""
    c = ort(3000.0, 1700.0, 2300.0)
    want = M.damp_ratio(c, "x")
    for axis in range(3):
        assert abs(lib_ratio(c, axis) - want) <= STEP + 1e-7


def test_bad_arguments():
    assert lib_ratio(ort(3000.0, 1700.0, 2300.0), 3) < 0
