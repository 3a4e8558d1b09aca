// vmesh.hpp -- the depth-refined vertical mesh of the elastic solvers with a
// free surface (prepare_modeling, src/solver/elastic_vhtiort_2d/module_vars.f90:
// 313-376; the same construction in elastic_vhtiort_3d/module_vars.f90:424-490).
// Host only.
//
// Integer rows z_i start at the surface (z_i(1) = 0) with spacing dz / rr down
// to (refine_rows - 1) dz; below, each new row lies min(1.025 h, dz_max) under
// the previous one (h the previous spacing) until the model's depth
// (nz - 1) dz is reached; the number of rows is the computational nz. Half rows
// z_h(1) = -dz / (2 rr), z_h(j + 1) = (z_i(j) + z_i(j + 1)) / 2. Local spacings
// dz_i, dz_h are centred differences of z_i, z_h (one-sided at the ends), and
// every z derivative of a row is scaled by dz / dz_i (integer rows) or dz / dz_h
// (half rows). The arrays extend pml + 1 rows past both ends: spacings and
// scalings by their end values, positions by dz / rr above the surface and the
// last spacing below the bottom.
//
// FLIT (github.com/lanl/flit, not vendored, no version pinned) supplies
// regspace and deriv; they are restated here from their use: regspace(a, h, b)
// = a, a + h, ... while <= b (a quotient (b - a) / h within 1e-5 of an integer
// counts as that integer), deriv(x, 'center') the centred difference above.
#pragma once

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/owl_ssg.h"

namespace owl {

struct VMesh {
    bool refined = false;  // false: the uniform grid, no mesh arrays needed
    int nz = 0;            // computational rows
    int pml = 0;
    float rr = 1.f;
    // rows -pml .. nz + pml + 1, at index j + pml
    std::vector<float> zi, zh, dzi, dzh, si, sh;
    float get(const std::vector<float>& v, int j) const { return v[(size_t)(j + pml)]; }
    size_t len() const { return (size_t)nz + 2 * pml + 2; }
};

// refinement factor and spacing cap of a descriptor (0 = unset: 1 and dz)
inline float vmesh_rr(const owl_ssg_desc& d) { return d.free_surface_dz_refine > 0.f ? d.free_surface_dz_refine : 1.f; }
inline float vmesh_dzmax(const owl_ssg_desc& d) { return d.dz_max > 0.f ? d.dz_max : d.dz; }

// a free-surface descriptor whose mesh is not the uniform grid
inline bool vmesh_is_refined(const owl_ssg_desc& d) {
    return d.free_surface != 0 && (vmesh_rr(d) != 1.f || vmesh_dzmax(d) != d.dz);
}

// throws std::invalid_argument with the reason on a descriptor the mesh cannot take
inline VMesh build_vmesh(const owl_ssg_desc& d) {
    VMesh m;
    m.nz = d.nz;
    m.pml = d.pml;
    if (!vmesh_is_refined(d)) return m;
    const float dz = d.dz, rr = vmesh_rr(d), cap = vmesh_dzmax(d);
    if (!(rr >= 1.f) || !std::isfinite(rr)) throw std::invalid_argument("free_surface_dz_refine must be >= 1");
    if (!(cap >= dz / rr) || !std::isfinite(cap))
        throw std::invalid_argument("dz_max must be at least dz / free_surface_dz_refine");
    if (d.free_surface_refine_rows < 1)
        throw std::invalid_argument("free_surface_refine_rows must be >= 1 with a refined free-surface mesh "
                                    "(owl_free_surface_refine_rows computes it)");
    m.refined = true;
    m.rr = rr;
    // regspace(0, dz / rr, (refine_rows - 1) dz)
    float h = dz / rr;
    const float last = (float)(d.free_surface_refine_rows - 1) * dz;
    const double q = (double)(last / h);
    const double qn = std::floor(q + 0.5);
    const long n0 = (long)(std::fabs(q - qn) <= 1e-5 ? qn : std::floor(q)) + 1;
    const long limit = 4L * 1000 * 1000;
    if (n0 > limit) throw std::invalid_argument("refined mesh too large");
    std::vector<float> z((size_t)n0);
    for (long i = 0; i < n0; ++i) z[(size_t)i] = 0.0f + (float)i * h;
    const float depth = (float)(d.nz - 1) * dz;
    while (z.back() < depth) {
        h = std::min(h * 1.025f, cap);
        z.push_back(z.back() + h);
        if ((long)z.size() > limit) throw std::invalid_argument("refined mesh too large");
    }
    const int n = (int)z.size();
    if (n < 2) throw std::invalid_argument("refined mesh needs at least two rows");
    m.nz = n;
    std::vector<float> zh((size_t)n);
    zh[0] = -0.5f * dz / rr;
    for (int i = 0; i + 1 < n; ++i) zh[(size_t)i + 1] = 0.5f * (z[(size_t)i] + z[(size_t)i + 1]);
    auto deriv = [](const std::vector<float>& x) {
        const size_t k = x.size();
        std::vector<float> g(k);
        g[0] = x[1] - x[0];
        g[k - 1] = x[k - 1] - x[k - 2];
        for (size_t i = 1; i + 1 < k; ++i) g[i] = 0.5f * (x[i + 1] - x[i - 1]);
        return g;
    };
    const std::vector<float> dzi = deriv(z), dzh = deriv(zh);
    const int P = d.pml;
    const size_t L = (size_t)n + 2 * P + 2;
    m.zi.assign(L, 0.f); m.zh.assign(L, 0.f); m.dzi.assign(L, 0.f); m.dzh.assign(L, 0.f);
    m.si.assign(L, 0.f); m.sh.assign(L, 0.f);
    for (int j = -P; j <= n + P + 1; ++j) {
        const int c = std::min(std::max(j, 1), n) - 1;  // edge value of the padded arrays
        const size_t o = (size_t)(j + P);
        m.dzi[o] = dzi[(size_t)c];
        m.dzh[o] = dzh[(size_t)c];
        m.si[o] = dz / dzi[(size_t)c];
        m.sh[o] = dz / dzh[(size_t)c];
        if (j >= 1 && j <= n) {
            m.zi[o] = z[(size_t)j - 1];
            m.zh[o] = zh[(size_t)j - 1];
        } else if (j < 1) {
            const int i = 1 - j;
            m.zi[o] = z[0] - (float)i * dz / rr;
            m.zh[o] = zh[0] - (float)i * dz / rr;
        } else {
            const int i = j - n;
            m.zi[o] = z[(size_t)n - 1] + (float)i * h;
            m.zh[o] = zh[(size_t)n - 1] + (float)i * h;
        }
    }
    return m;
}

// Linear interpolation of the padded regular rows (depths (j - 1) dz, j = -pml ..
// nz + pml + 1) at the mesh's integer rows (map_regular_to_irregular,
// module_vars.f90:139-169): row f takes (1 - w) of regular row r0(f) and w of
// r0(f) + 1, as y(r0) + w (y(r0 + 1) - y(r0)); outside the regular rows the end
// values (the padding is constant there).
struct ZInterp {
    std::vector<int> r0;   // regular padded row of each mesh row (rows -pml .. n + pml + 1)
    std::vector<float> w;
};

inline ZInterp build_zinterp(const VMesh& m, int nz_reg, float dz) {
    ZInterp t;
    const int P = m.pml;
    t.r0.resize(m.len());
    t.w.resize(m.len());
    for (int f = -P; f <= m.nz + P + 1; ++f) {
        const float zf = m.get(m.zi, f);
        // regular padded row j sits at (j - 1) dz
        int j = (int)std::floor(zf / dz) + 1;
        float w;
        if (j < -P) {
            j = -P;
            w = 0.f;
        } else if (j >= nz_reg + P + 1) {
            j = nz_reg + P;
            w = 1.f;
        } else {
            const float za = (float)(j - 1) * dz, zb = (float)j * dz;
            w = (zf - za) / (zb - za);
            w = std::min(std::max(w, 0.f), 1.f);
        }
        t.r0[(size_t)(f + P)] = j;
        t.w[(size_t)(f + P)] = w;
    }
    return t;
}

template <typename T>
inline T zinterp_apply(const ZInterp& t, int f, int P, const T& y0, const T& y1) {
    return y0 + T(t.w[(size_t)(f + P)]) * (y1 - y0);
}

}  // namespace owl
