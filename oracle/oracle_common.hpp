// oracle_common.hpp -- shared pieces of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. The oracle is a plain C++ restatement of OWL's
// Fortran loops; it is used by tests/, by __graft_entry__.smoke() and by the
// CPU-baseline leg of bench.py as the checker. The product path (owl_b200/)
// never links, loads or calls it.
//
// Arrays follow the reference's conventions: Fortran-style lower bounds that
// may be negative, x (i) fastest after the transpose in prepare_modeling
// (src/solver/acoustic_iso_2d/module_vars.f90:109-111).
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/owl_ssg.h"

namespace oracle {

// real part / magnitude helpers so the same templates run on float, double and
// std::complex<double> (complex step differentiation).
inline double re(float v) { return v; }
inline double re(double v) { return v; }
inline double re(const std::complex<double>& v) { return v.real(); }

template <typename T>
struct Arr2 {
    // (i, j) with i in [i0, i1], j in [j0, j1], i fastest
    int i0 = 0, i1 = -1, j0 = 0, j1 = -1, ni = 0, nj = 0;
    std::vector<T> a;
    Arr2() = default;
    Arr2(int i0_, int i1_, int j0_, int j1_) { init(i0_, i1_, j0_, j1_); }
    void init(int i0_, int i1_, int j0_, int j1_) {
        i0 = i0_; i1 = i1_; j0 = j0_; j1 = j1_;
        ni = i1 - i0 + 1; nj = j1 - j0 + 1;
        a.assign((size_t)ni * nj, T(0));
    }
    inline T& operator()(int i, int j) { return a[(size_t)(j - j0) * ni + (i - i0)]; }
    inline const T& operator()(int i, int j) const { return a[(size_t)(j - j0) * ni + (i - i0)]; }
    void zero() { std::fill(a.begin(), a.end(), T(0)); }
};

template <typename T>
struct Arr1 {
    int i0 = 0, i1 = -1;
    std::vector<T> a;
    void init(int i0_, int i1_, T v) { i0 = i0_; i1 = i1_; a.assign(i1 - i0 + 1, v); }
    inline T& operator()(int i) { return a[i - i0]; }
    inline const T& operator()(int i) const { return a[i - i0]; }
};

// FD coefficients, src/lib/module_fdcoef.f90:59-62 (half-width 4) and :23-30 (half-width 8)
inline const float* fdcoefs(int half) {
    static const float c4[4] = {0.1217990e+1f, -0.9382142e-1f, 0.1507536e-1f, -0.1700324e-2f};
    static const float c8[8] = {0.1259312e+1f, -0.1280347e+0f, 0.3841945e-1f, -0.1473229e-1f,
                                0.5924913e-2f, -0.2248618e-2f, 0.7179226e-3f, -0.1400855e-3f};
    return half == 8 ? c8 : c4;
}

// CFS-PML coefficient for one node, restating damp_coef
// (src/solver/acoustic_iso_2d/module_cfspml.f90:37-56) in single precision.
inline void damp_coef(float bdvp, float d, float dist, int pml, float dt, float alphamax,
                      float& a, float& b, float& k) {
    const float R0 = 1.0e-5f, kmax = 1.0f;
    float nd = dist / ((float)pml * d);
    float alpha = std::max(alphamax * (1.0f - nd), 0.25f * alphamax);
    float damp = bdvp * (2.0f + 1.0f) * std::log(1.0f / R0) / (2.0f * (float)pml * d) * (nd * nd);
    k = 1.0f + (kmax - 1.0f) * (nd * nd);
    float adt = std::fabs(dt);
    a = -2.0f * adt * damp / k / (2.0f + adt * (alpha + damp / k));
    b = (2.0f - adt * (alpha + damp / k)) / (2.0f + adt * (alpha + damp / k));
}

// 1D CFS-PML coefficient arrays over [-pml+1, n+pml] at integer (i) and half (h)
// nodes, restating compute_cfspml_damping_coef (module_cfspml.f90:61-133).
struct Pml1D {
    Arr1<float> ai, bi, ki, ah, bh, kh;
    void build(int n, int pml, float d, float dt, float pmlvp, float alphamax) {
        ai.init(-pml + 1, n + pml, 0.f); bi.init(-pml + 1, n + pml, 0.f); ki.init(-pml + 1, n + pml, 1.f);
        ah.init(-pml + 1, n + pml, 0.f); bh.init(-pml + 1, n + pml, 0.f); kh.init(-pml + 1, n + pml, 1.f);
        for (int i = -pml + 1; i <= n + pml; ++i) {
            float disti = 0.f, disth = 0.f;
            if (i <= 1) {
                disti = std::fabs((float)(i - 1) * d);
                disth = std::fabs(((float)(i - 1) - 0.5f) * d);
            } else if (i >= n + 1) {
                disti = std::fabs((float)(i - n) * d);
                disth = std::fabs(((float)(i - n) - 0.5f) * d);
            }
            if (i <= 1 || i >= n + 1) {
                damp_coef(pmlvp, d, disti, pml, dt, alphamax, ai(i), bi(i), ki(i));
                damp_coef(pmlvp, d, disth, pml, dt, alphamax, ah(i), bh(i), kh(i));
            }
        }
    }
};

}  // namespace oracle
