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
#include <algorithm>
#include <stdexcept>
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

// ---------------------------------------------------------------------------
// Depth-refined vertical mesh of the elastic solvers with a free surface
// (src/solver/elastic_vhtiort_2d/module_vars.f90:313-376). FLIT (not vendored)
// supplies regspace and deriv, restated from their use: regspace(a, h, b) =
// a + (i - 1) h for i = 1 .. floor((b - a) / h) + 1 (a quotient within 1e-5 of
// an integer taken as that integer); deriv(x, 'center') the centred
// difference, one-sided at the two ends.
// ---------------------------------------------------------------------------
struct ZMesh {
    bool refined = false;
    int n = 0, pml = 0;
    Arr1<float> zi, zh, dzi, dzh, si, sh;  // rows [-pml, n + pml + 1]
};

inline ZMesh zmesh_build(const owl_ssg_desc& d) {
    ZMesh m;
    m.n = d.nz;
    m.pml = d.pml;
    const float rr = d.free_surface_dz_refine > 0.f ? d.free_surface_dz_refine : 1.f;
    const float dz_cap = d.dz_max > 0.f ? d.dz_max : d.dz;
    if (!d.free_surface || (rr == 1.f && dz_cap == d.dz)) return m;
    if (d.free_surface_refine_rows < 1) throw std::runtime_error("refine rows");
    m.refined = true;
    const float dz = d.dz;
    float dz_max = dz / rr;
    // zz_i = regspace(0.0, dz_max, (refine_nz - 1)*dz)
    const float b = (float)(d.free_surface_refine_rows - 1) * dz;
    const double q = (double)(b / dz_max);
    const double qr = std::floor(q + 0.5);
    const int cnt = (int)(std::fabs(q - qr) <= 1e-5 ? qr : std::floor(q)) + 1;
    std::vector<float> zz_i;
    for (int i = 1; i <= cnt; ++i) zz_i.push_back(0.0f + (float)(i - 1) * dz_max);
    size_t l = zz_i.size();
    while (zz_i[l - 1] < (float)(d.nz - 1) * dz) {
        dz_max = std::min(dz_max * 1.025f, dz_cap);
        zz_i.push_back(zz_i[l - 1] + dz_max);
        l = l + 1;
    }
    const int nz = (int)zz_i.size();
    m.n = nz;
    std::vector<float> zz_h(nz, 0.f);
    zz_h[0] = -0.5f * dz / rr;
    for (int i = 1; i <= nz - 1; ++i) zz_h[i] = 0.5f * (zz_i[i - 1] + zz_i[i]);
    auto deriv_center = [](const std::vector<float>& x) {
        const int k = (int)x.size();
        std::vector<float> g(k);
        for (int i = 1; i < k - 1; ++i) g[i] = (x[i + 1] - x[i - 1]) * 0.5f;
        g[0] = x[1] - x[0];
        g[k - 1] = x[k - 1] - x[k - 2];
        return g;
    };
    const std::vector<float> dz_i = deriv_center(zz_i), dz_h = deriv_center(zz_h);
    const int P = d.pml;
    for (Arr1<float>* a : {&m.zi, &m.zh, &m.dzi, &m.dzh, &m.si, &m.sh}) a->init(-P, nz + P + 1, 0.f);
    // pad_array by pml + 1 (edge values), then the positions past both ends
    for (int j = -P; j <= nz + P + 1; ++j) {
        const int e = std::min(std::max(j, 1), nz) - 1;
        m.dzi(j) = dz_i[e];
        m.dzh(j) = dz_h[e];
        m.si(j) = dz / dz_i[e];
        m.sh(j) = dz / dz_h[e];
        m.zi(j) = zz_i[e];
        m.zh(j) = zz_h[e];
    }
    for (int i = 1; i <= P + 1; ++i) {
        m.zi(1 - i) = zz_i[0] - (float)i * dz / rr;
        m.zi(nz + i) = zz_i[nz - 1] + (float)i * dz_max;
        m.zh(1 - i) = zz_h[0] - (float)i * dz / rr;
        m.zh(nz + i) = zz_h[nz - 1] + (float)i * dz_max;
    }
    return m;
}

// map_regular_to_irregular (module_vars.f90:139-169): regular padded rows at
// depths (j - 1) dz, j = -pml .. nzm + pml + 1, interpolated linearly at the
// mesh rows zi(f); j0(f) the upper bracketing regular row, w(f) the weight of
// the lower one (constant extension past the ends, where the padding is
// constant anyway).
struct ZLinear {
    Arr1<int> j0;
    Arr1<float> w;
};

inline ZLinear zlinear_build(const ZMesh& m, int nzm, float dz) {
    ZLinear t;
    const int P = m.pml;
    t.j0.init(-P, m.n + P + 1, 0);
    t.w.init(-P, m.n + P + 1, 0.f);
    for (int f = -P; f <= m.n + P + 1; ++f) {
        const float z = m.zi(f);
        int j = (int)std::floor(z / dz) + 1;
        float w;
        if (j < -P) {
            j = -P;
            w = 0.f;
        } else if (j > nzm + P) {
            j = nzm + P;
            w = 1.f;
        } else {
            const float z0 = (float)(j - 1) * dz, z1 = (float)j * dz;
            w = std::min(std::max((z - z0) / (z1 - z0), 0.f), 1.f);
        }
        t.j0(f) = j;
        t.w(f) = w;
    }
    return t;
}

}  // namespace oracle
