"""Test infrastructure (the oracle): literal restatement of the reference's M-PML
damping-ratio search for 3D anisotropic elastic media,
src/solver/elastic_vhtiort_3d/module_cfspml.f90.

- mpml_eigenvalue_derivative (:51-186): the 27 x 27 split-field system of a
  plane wave with wavenumber direction (k1, k2, k3) -- 18 stress splits and 9
  velocity splits, stiffness scaled by 1e-9 -- its eigen-decomposition (LAPACK
  geev there, numpy.linalg.eig here), eigenvalues below 1e-2 of the largest
  set to zero, the first three negative real ones kept, and the largest
  derivative u^T B v / u^T v of them under the damping matrix B = -diag(1 on
  the splits of `direction`, ratio elsewhere).
- damp_ratio (:193-248): the ratio raised from 2e-3 in steps of 2e-3 (single
  precision, as the reference's real variables) until that derivative drops
  below -0.01 for every direction of a 60 x 60 (theta, phi) grid, or 1.
- face_ratio (:253-409): damp_ratio at every 10th cell of a face (at most
  min(10, n1, n2)) and linear interpolation to every cell of the face. FLIT's
  `interp` is not vendored: beyond the last sample the value is held
  (parity unpinned there).

The oracle is the checker of the library's own search (owl_mpml_damp_ratio,
owl_ssg_mpml_ratios); it is never called by the library.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
EIGENDERIV_MAX = F32(-0.01)
DRATIO = F32(2.0e-3)


def _system(c, k1, k2, k3):
    """The 27 x 27 matrix a of mpml_eigenvalue_derivative (:72-107) for the
    orthorhombic stiffness c = (c11, c12, c13, c22, c23, c33, c44, c55, c66)
    (every other Cij zero, as compute_damping_profile_ratio_face passes them)."""
    c11, c12, c13, c22, c23, c33, c44, c55, c66 = [float(v) for v in c]
    c14 = c15 = c16 = c24 = c25 = c26 = c34 = c35 = c36 = c45 = c46 = c56 = 0.0
    top = np.array([
        [c11 * k1, c16 * k1, c15 * k1] * 3,
        [c12 * k1, c26 * k1, c25 * k1] * 3,
        [c13 * k1, c36 * k1, c35 * k1] * 3,
        [c14 * k1, c46 * k1, c45 * k1] * 3,
        [c15 * k1, c56 * k1, c55 * k1] * 3,
        [c16 * k1, c66 * k1, c56 * k1] * 3,
        [c16 * k2, c12 * k2, c14 * k2] * 3,
        [c26 * k2, c22 * k2, c24 * k2] * 3,
        [c36 * k2, c23 * k2, c34 * k2] * 3,
        [c46 * k2, c24 * k2, c44 * k2] * 3,
        [c56 * k2, c25 * k2, c45 * k2] * 3,
        [c66 * k2, c26 * k2, c46 * k2] * 3,
        [c15 * k3, c14 * k3, c13 * k3] * 3,
        [c25 * k3, c24 * k3, c23 * k3] * 3,
        [c35 * k3, c34 * k3, c33 * k3] * 3,
        [c45 * k3, c44 * k3, c34 * k3] * 3,
        [c55 * k3, c45 * k3, c35 * k3] * 3,
        [c56 * k3, c46 * k3, c36 * k3] * 3,
    ]) / 1.0e9
    bot = np.zeros((9, 18))
    # rows: velocity splits (vx, vy, vz) x (x, y, z); columns: the three splits of
    # the stress component the row differentiates
    picks = [(k1, 0), (k1, 5), (k1, 4), (k2, 5), (k2, 1), (k2, 3), (k3, 4), (k3, 3), (k3, 2)]
    for r, (kk, comp) in enumerate(picks):
        for split in range(3):
            bot[r, comp + 6 * split] = kk
    a = np.zeros((27, 27))
    a[0:18, 18:27] = top
    a[18:27, 0:18] = bot
    return a


def _diag(direction, ratio):
    r = float(ratio)
    if direction == "x":
        d = [1.0] * 6 + [r] * 6 + [r] * 6 + [1.0] * 3 + [r] * 3 + [r] * 3
    elif direction == "y":
        d = [r] * 6 + [1.0] * 6 + [r] * 6 + [r] * 3 + [1.0] * 3 + [r] * 3
    else:
        d = [r] * 6 + [r] * 6 + [1.0] * 6 + [r] * 3 + [r] * 3 + [1.0] * 3
    return -np.diag(d)


def mpml_eigenvalue_derivative(c, direction, ratio, k1, k2, k3) -> float:
    """module_cfspml.f90:51-186."""
    a = _system(c, k1, k2, k3)
    b = _diag(direction, ratio)
    w, vr = np.linalg.eig(a)
    wl, vl_raw = np.linalg.eig(a.T)  # left eigenvectors: right eigenvectors of a^T
    # pair each right eigenvector with the left one of the same eigenvalue
    order = [int(np.argmin(np.abs(wl - lam))) for lam in w]
    vl = vl_raw[:, order]
    wr, wi = w.real.copy(), w.imag.copy()
    mx = np.max(np.abs(wr))
    wr[np.abs(wr) < 1.0e-2 * mx] = 0.0
    wi[np.abs(wi) < 1.0e-2 * mx] = 0.0
    psn = [i for i in range(27) if wr[i] < 0 and wi[i] == 0][:3]
    eigd = []
    for ind in sorted(psn):
        evl = vl[:, ind].real
        evr = vr[:, ind].real
        t = float(evl @ evr)
        t = t + (1.0e-15 if t == 0 else np.copysign(1.0e-15, t))
        eigd.append(float(evl @ b @ evr) / t)
    eigd = [e for e in eigd if not np.isnan(e)]
    return max(eigd)


def reduced_eigenvalue_derivative(c, direction, ratio, k1, k2, k3) -> float:
    """The same derivative from the 3 x 3 Christoffel problem: with P = the
    stress rate of a unit velocity summed over the splits (6 x 3), Q = the
    velocity rate of a unit stress (3 x 6), C_a and k_a D_a their split-a
    parts, gamma, e an eigenpair of Gamma = Q P, the eigenvalue -sqrt(gamma) of
    the 27 x 27 system has u^T B v / u^T v =
    -(1 / (2 gamma)) sum_a w_a (e^T Q C_a e + e^T k_a D_a P e), w_a = 1 on the
    damped axis and ratio elsewhere."""
    a = _system(c, k1, k2, k3)
    top, bot = a[0:18, 18:27], a[18:27, 0:18]
    Ca = [top[6 * s:6 * s + 6, 0:3] for s in range(3)]     # split s of the stress rate per unit velocity
    Da = [bot[3 * s:3 * s + 3, 0:6] for s in range(3)]     # split s of the velocity rate per unit stress
    P = sum(Ca)
    Q = sum(Da)
    G = Q @ P
    g, E = np.linalg.eigh(0.5 * (G + G.T))
    w = {"x": [1.0, ratio, ratio], "y": [ratio, 1.0, ratio], "z": [ratio, ratio, 1.0]}[direction]
    out = []
    for m in range(3):
        if g[m] <= 1e-4 * g.max():
            continue
        e = E[:, m]
        t = [e @ Q @ Ca[s] @ e + e @ Da[s] @ P @ e for s in range(3)]
        out.append(-sum(w[s] * t[s] for s in range(3)) / (2 * g[m]))
    return max(out)


def damp_ratio(c, direction) -> float:
    """module_cfspml.f90:193-248 (single-precision angles and ratio steps)."""
    ng1 = ng2 = 60
    pi = F32(np.pi)
    dtheta = F32(pi / F32(ng1))
    dphi = F32(pi / F32(ng2))
    ratio = DRATIO
    for i in range(1, ng1 + 1):
        for j in range(1, ng2 + 1):
            theta = F32(F32(i + 0.5) * dtheta)
            phi = F32(F32(j + 0.5) * dphi)
            kx = float(F32(np.sin(theta) * np.cos(phi)))
            ky = float(F32(np.sin(theta) * np.sin(phi)))
            kz = float(F32(np.cos(theta)))
            derig = mpml_eigenvalue_derivative(c, direction, ratio, kx, ky, kz)
            while derig >= EIGENDERIV_MAX and ratio < 1.0:
                ratio = F32(ratio + DRATIO)
                derig = mpml_eigenvalue_derivative(c, direction, ratio, kx, ky, kz)
    return float(ratio)


def sample_grid(n: int, interval: int):
    """Offsets of the sampled cells along a face axis of n cells (:290-308)."""
    m = 1
    for _ in range(1, n + 1, interval):
        m += 1
    if (m - 1) * interval > n - 1:
        m -= 1
    return [interval * q for q in range(m)]


def face_ratio(cface, direction, ratio_fn=damp_ratio):
    """cface: (n1, n2, 9) stiffness on a face (the model's cells at the face's
    edge, padded cells included); returns the (n1, n2) ratio array: ratio_fn at
    the sampled cells, linear interpolation between them, held beyond the last."""
    n1, n2 = cface.shape[:2]
    interval = min(10, n1, n2)
    s1, s2 = sample_grid(n1, interval), sample_grid(n2, interval)
    r = np.array([[ratio_fn(cface[i, j], direction) for j in s2] for i in s1], dtype=np.float64)
    return interp_linear_2d(r, s1, s2, n1, n2)


def interp_linear_2d(r, s1, s2, n1, n2):
    def axis_w(s, n):
        out = []
        for t in range(n):
            if t >= s[-1]:
                out.append((len(s) - 1, len(s) - 1, 0.0))
                continue
            q = t // (s[1] - s[0]) if len(s) > 1 else 0
            q = min(q, len(s) - 2)
            f = (t - s[q]) / (s[q + 1] - s[q])
            out.append((q, q + 1, f))
        return out
    w1, w2 = axis_w(s1, n1), axis_w(s2, n2)
    out = np.zeros((n1, n2))
    for i, (a0, a1, fa) in enumerate(w1):
        for j, (b0, b1, fb) in enumerate(w2):
            out[i, j] = ((1 - fa) * (1 - fb) * r[a0, b0] + fa * (1 - fb) * r[a1, b0] +
                         (1 - fa) * fb * r[a0, b1] + fa * fb * r[a1, b1])
    return out
