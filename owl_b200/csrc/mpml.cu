// mpml.cu -- M-PML damping ratios of the 3D anisotropic elastic solver (host).
//
// The reference (src/solver/elastic_vhtiort_3d/module_cfspml.f90) damps, inside
// the PML shell, every derivative along axis b with d_b + ratio_a d_a for the
// other axes a (Meza-Fajardo & Papageorgiou 2008), with one ratio per face
// cell. damp_ratio (:193-248) finds a face cell's ratio: starting at 2e-3 and in
// steps of 2e-3, the smallest ratio for which the eigenvalue derivative of the
// damped plane-wave system drops below -0.01 for every direction of a 60 x 60
// (theta, phi) grid (capped at 1). mpml_eigenvalue_derivative (:51-186) builds
// the 27 x 27 split-field system (18 stress splits, 9 velocity splits) and
// takes the largest u^T B v / u^T v over its three negative real eigenvalues
// (u, v left / right eigenvectors, B = -diag(1 on the damped axis' splits,
// ratio elsewhere)).
//
// That system reduces exactly to the 3 x 3 Christoffel problem: with P (6 x 3)
// the stress rate of a unit velocity summed over the splits, Q (3 x 6) the
// velocity rate of a unit stress, C_a and k_a D_a their split-a parts and
// Gamma = Q P, a nonzero eigenvalue is lambda = -sqrt(gamma) (gamma, e an
// eigenpair of the symmetric Gamma), its right eigenvector stacks C_a e / lambda
// and k_a D_a P e / lambda^2, its left one Q^T e / lambda and e on every split,
// u^T v = 2 and
//   u^T B v / u^T v = -(1 / (2 gamma)) sum_a w_a (e^T Q C_a e + e^T k_a D_a P e)
// with w_a = 1 on the damped axis and ratio on the others. This file evaluates
// that in double precision (Jacobi eigen-decomposition of Gamma); the literal
// 27 x 27 form is restated in the test oracle, which checks this one.
//
// Face arrays: damp_ratio at every min(10, n1, n2)-th cell of a face and linear
// interpolation in between (compute_damping_profile_ratio_face, :253-409; FLIT's
// interp, not vendored, restated as bilinear interpolation, the last sampled
// value held beyond the last sample).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "common.cuh"
#include "mpml.cuh"

namespace owl {

namespace {

// cyclic Jacobi: A (symmetric, overwritten) -> eigenvalues w, eigenvectors V[:, m]
void sym3_eig(double A[3][3], double w[3], double V[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const double dg = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-32 * dg) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A[p][q] == 0.0) continue;
                const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int m = 0; m < 3; ++m) w[m] = A[m][m];
}

}  // namespace

double mpml_eig_deriv(const double c[9], int axis, double ratio, double k1, double k2, double k3) {
    const double c11 = c[0], c12 = c[1], c13 = c[2], c22 = c[3], c23 = c[4], c33 = c[5], c44 = c[6], c55 = c[7],
                 c66 = c[8];
    // split parts of the stress rate per unit velocity (rows xx, yy, zz, yz, xz, xy; columns vx, vy, vz)
    double Ca[3][6][3] = {};
    Ca[0][0][0] = c11 * k1; Ca[0][1][0] = c12 * k1; Ca[0][2][0] = c13 * k1; Ca[0][4][2] = c55 * k1; Ca[0][5][1] = c66 * k1;
    Ca[1][0][1] = c12 * k2; Ca[1][1][1] = c22 * k2; Ca[1][2][1] = c23 * k2; Ca[1][3][2] = c44 * k2; Ca[1][5][0] = c66 * k2;
    Ca[2][0][2] = c13 * k3; Ca[2][1][2] = c23 * k3; Ca[2][2][2] = c33 * k3; Ca[2][3][1] = c44 * k3; Ca[2][4][0] = c55 * k3;
    // split parts of the velocity rate per unit stress: (vx, vy, vz) <- stresses
    const int pick[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};  // split a: vx, vy, vz read these stresses
    const double ka[3] = {k1, k2, k3};
    double P[6][3] = {}, Q[3][6] = {};
    for (int a = 0; a < 3; ++a) {
        for (int r = 0; r < 6; ++r)
            for (int j = 0; j < 3; ++j) P[r][j] += Ca[a][r][j];
        for (int i = 0; i < 3; ++i) Q[i][pick[a][i]] += ka[a];
    }
    double G[3][3] = {};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int r = 0; r < 6; ++r) G[i][j] += Q[i][r] * P[r][j];
    double A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = 0.5 * (G[i][j] + G[j][i]);
    double w[3], V[3][3];
    sym3_eig(A, w, V);
    const double gmax = std::max(w[0], std::max(w[1], w[2]));
    double best = -1e300;
    bool any = false;
    for (int m = 0; m < 3; ++m) {
        // eigenvalues below 1e-2 of the largest (in |lambda| = sqrt(gamma)) count as zero
        if (!(w[m] > 0.0) || w[m] < 1e-4 * gmax) continue;
        const double e[3] = {V[0][m], V[1][m], V[2][m]};
        double Pe[6] = {};
        for (int r = 0; r < 6; ++r)
            for (int j = 0; j < 3; ++j) Pe[r] += P[r][j] * e[j];
        double Qte[6] = {};
        for (int r = 0; r < 6; ++r)
            for (int i = 0; i < 3; ++i) Qte[r] += Q[i][r] * e[i];
        double sum = 0.0;
        for (int a = 0; a < 3; ++a) {
            double t1 = 0.0;  // e^T Q C_a e
            for (int r = 0; r < 6; ++r) {
                double ce = 0.0;
                for (int j = 0; j < 3; ++j) ce += Ca[a][r][j] * e[j];
                t1 += Qte[r] * ce;
            }
            double t2 = 0.0;  // e^T k_a D_a P e
            for (int i = 0; i < 3; ++i) t2 += e[i] * ka[a] * Pe[pick[a][i]];
            sum += (a == axis ? 1.0 : ratio) * (t1 + t2);
        }
        const double d = -sum / (2.0 * w[m]);
        if (!std::isnan(d)) { best = any ? std::max(best, d) : d; any = true; }
    }
    return any ? best : -1e300;
}

float mpml_damp_ratio(const float c[9], int axis) {
    double cd[9];
    for (int q = 0; q < 9; ++q) cd[q] = c[q];
    const int ng1 = 60, ng2 = 60;
    const float pi = 3.14159265358979323846f;
    const float dtheta = pi / (float)ng1, dphi = pi / (float)ng2;
    const float alpha = -0.01f, dratio = 2.0e-3f;
    float ratio = dratio;
    for (int i = 1; i <= ng1; ++i)
        for (int j = 1; j <= ng2; ++j) {
            const float theta = ((float)i + 0.5f) * dtheta, phi = ((float)j + 0.5f) * dphi;
            const float kx = std::sin(theta) * std::cos(phi), ky = std::sin(theta) * std::sin(phi), kz = std::cos(theta);
            double derig = mpml_eig_deriv(cd, axis, ratio, kx, ky, kz);
            while (derig >= alpha && ratio < 1.0f) {
                ratio = ratio + dratio;
                derig = mpml_eig_deriv(cd, axis, ratio, kx, ky, kz);
            }
        }
    return ratio;
}

std::vector<int> mpml_samples(int n, int interval) {
    int m = 1;
    for (int i = 1; i <= n; i += interval) ++m;
    if ((m - 1) * interval > n - 1) --m;
    std::vector<int> s(m);
    for (int q = 0; q < m; ++q) s[q] = q * interval;
    return s;
}

void mpml_face(int n1, int n2, int axis, const std::function<void(int, int, float*)>& cell_c, float* out, int ld) {
    const int interval = std::min(10, std::min(n1, n2));
    const std::vector<int> s1 = mpml_samples(n1, interval), s2 = mpml_samples(n2, interval);
    const int m1 = (int)s1.size(), m2 = (int)s2.size();
    std::vector<float> r((size_t)m1 * m2);
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int q = next++; q < m1 * m2; q = next++) {
            float c[9];
            cell_c(s1[q / m2], s2[q % m2], c);
            r[q] = mpml_damp_ratio(c, axis);
        }
    };
    const int nth = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int t = 1; t < std::min(nth, m1 * m2); ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    // bilinear interpolation, the last sample held beyond it
    auto wgt = [&](int t, const std::vector<int>& s, int& q0, int& q1, double& f) {
        const int m = (int)s.size();
        if (m == 1 || t >= s[m - 1]) { q0 = q1 = m - 1; f = 0.0; return; }
        q0 = std::min(t / interval, m - 2);
        q1 = q0 + 1;
        f = (double)(t - s[q0]) / (double)(s[q1] - s[q0]);
    };
    for (int i = 0; i < n1; ++i) {
        int a0, a1;
        double fa;
        wgt(i, s1, a0, a1, fa);
        for (int j = 0; j < n2; ++j) {
            int b0, b1;
            double fb;
            wgt(j, s2, b0, b1, fb);
            const double v = (1 - fa) * (1 - fb) * r[(size_t)a0 * m2 + b0] + fa * (1 - fb) * r[(size_t)a1 * m2 + b0] +
                             (1 - fa) * fb * r[(size_t)a0 * m2 + b1] + fa * fb * r[(size_t)a1 * m2 + b1];
            out[(size_t)j * ld + i] = (float)v;
        }
    }
}

}  // namespace owl

// ---- C ABI ----------------------------------------------------------------
extern "C" float owl_mpml_damp_ratio(const float* c9, int axis) {
    if (!c9 || axis < 0 || axis > 2) return -1.0f;
    return owl::mpml_damp_ratio(c9, axis);
}
