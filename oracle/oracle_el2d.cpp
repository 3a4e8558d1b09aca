// oracle_el2d.cpp -- CPU oracle for the 2D elastic VTI/TTI SSG solver.
//
// TEST INFRASTRUCTURE ONLY (see oracle_common.hpp). Restates, loop by loop:
//   model set-up (Cij from iso / Thomsen / Alkhalifah-Tsvankin / Cij, padding,
//   pmlvp, dt_stable)           src/solver/elastic_vhtiort_2d/module_vars.f90:208-420
//   thomsen_to_cij2d, alkhalifah_tsvankin_to_cij2d
//                               src/lib/module_anisotropy.f90:310-402
//   M-PML damping ratios and 2D CFS-MPML coefficients
//                               src/solver/elastic_vhtiort_2d/module_cfspml.f90:76-577
//   update_wavefield            src/solver/elastic_vhtiort_2d/module_wavefield.f90:42-138
//   update_wavefield_free_surface                    module_wavefield.f90:143-289
//   add_source                  src/solver/elastic_vhtiort_2d/module_wavefield.f90:294-403
//   time loop, surface images and sampling
//                               src/solver/elastic_vhtiort_2d/submodule_forward_modeling.f90:58-197
// on the uniform grid and on the depth-refined free-surface mesh
// (module_vars.f90:313-376: Cij interpolated linearly to the mesh rows, every z
// derivative scaled by dz / dz_i or dz / dz_h, the z PML and the explosion
// source on the row's own dz_i), plus the exact discrete adjoint of that loop
// and the chain rule from (c11, c13, c33, c55, rho) to the model parameters (on
// the refined mesh through the transpose of the row interpolation, back to the
// regular rows).
//
// Templated on T: float (forward parity oracle), double (FP64 gradient oracle),
// std::complex<double> (complex-step Jacobian-vector products). The PML
// coefficients and M-PML ratios depend on the model only through max / threshold
// operations; they are computed in float from the real part and held constant.
#include <algorithm>
#include <array>
#include <cstdio>
#include <stdexcept>

#include "oracle_common.hpp"

namespace oracle {

template <typename T>
inline T cs_abs(const T& x) { return re(x) < 0 ? -x : x; }

// Cij of one cell from the model parameters (desc.aniso), in T arithmetic with
// the reference's operation order. Rotation by the tilt: closed form of the
// Bond rotation about y restricted to c11, c13, c33, c55 (c15, c35 are dropped
// by the 2D stencils, module_wavefield.f90:71-72,92).
template <typename T>
void to_cij(int aniso, const T* p, T& c11, T& c13, T& c33, T& c55, T& rho) {
    T the = T(0);
    if (aniso == OWL_ANISO_ISO) {
        const T vp = p[0], vs = p[1];
        rho = p[2];
        c33 = rho * (vp * vp);
        c55 = rho * (vs * vs);
        c11 = c33;
        c13 = c33 - T(2) * c55;
        return;
    } else if (aniso == OWL_ANISO_THOMSEN) {
        const T vp = p[0], vs = p[1], eps = p[2], del = p[3];
        the = p[4];
        rho = p[5];
        c33 = (vp * vp) * rho;
        c55 = (vs * vs) * rho;
        c11 = c33 * (T(1) + T(2) * eps);
        T tmp = T(2) * c33 * (c33 - c55) * del + (c33 - c55) * (c33 - c55);
        c13 = std::sqrt(cs_abs(tmp)) - c55;
    } else if (aniso == OWL_ANISO_AT) {
        const T vp = p[0], vs = p[1], eps = p[2], eta = p[3];
        the = p[4];
        rho = p[5];
        c11 = (vp * vp) * rho;
        c55 = (vs * vs) * rho;
        c33 = c11 / (T(1) + T(2) * eps);
        c13 = rho * (std::sqrt(cs_abs(((vp * vp) / (T(1) + T(2) * eps) - vs * vs) *
                                      ((vp * vp) / (T(1) + T(2) * eta) - vs * vs))) - vs * vs);
    } else {
        c11 = p[0]; c13 = p[1]; c33 = p[2]; c55 = p[3];
        rho = p[4];
        return;
    }
    if (re(the) != 0) {
        const T cs = std::cos(-the), sn = std::sin(-the);
        const T c2 = cs * cs, s2 = sn * sn, cs2s2 = c2 * s2, c4 = c2 * c2, s4 = s2 * s2;
        const T a11 = c11, a13 = c13, a33 = c33, a55 = c55;
        c11 = a11 * c4 + T(2) * (a13 + T(2) * a55) * cs2s2 + a33 * s4;
        c33 = a11 * s4 + T(2) * (a13 + T(2) * a55) * cs2s2 + a33 * c4;
        c13 = (a11 + a33 - T(4) * a55) * cs2s2 + a13 * (c4 + s4);
        c55 = (a11 + a33 - T(2) * a13 - T(2) * a55) * cs2s2 + a55 * (c4 + s4);
    }
}

inline int aniso_nparam(int aniso) {
    switch (aniso) {
        case OWL_ANISO_ISO: return 3;
        case OWL_ANISO_THOMSEN: return 6;
        case OWL_ANISO_AT: return 6;
        case OWL_ANISO_CIJ: return 5;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// M-PML damping ratio (damp_ratio, module_cfspml.f90:174-223) with c15 = c35 = 0
// as the 2D solver calls it (:240-270). With those zeros the eigenvalues are
// purely imaginary and every complex operation reduces to the real one below.
// ---------------------------------------------------------------------------
// squared eigenvalue of mode 1 / 2 of the Christoffel problem (mpml_eigenvalue, :79-103)
inline float mpml_eig2(float c11, float c13, float c33, float c55, float rho, int mode, float k1, float k3) {
    const float A = (c11 + c55) * (k1 * k1) + (c33 + c55) * (k3 * k3);
    const float k14 = (k1 * k1) * (k1 * k1), k34 = (k3 * k3) * (k3 * k3);
    const float B = -(c11 * c55) * k14 + (c13 * c13 - c11 * c33 + 2 * c13 * c55) * (k1 * k1) * (k3 * k3) -
                    (c33 * c55) * k34;
    const float s = std::sqrt((A * A + 4 * B) * (rho * rho));
    const float x = mode == 1 ? -((A * rho + s) / (rho * rho)) : (-(A * rho) + s) / (rho * rho);
    // -(csqrt(x) / sqrt(2)) squared: purely imaginary for x <= 0
    const float b = (x <= 0 ? std::sqrt(-x) : std::sqrt(x)) / std::sqrt(2.0f);
    return x <= 0 ? -(b * b) : b * b;
}

// real part of mpml_eigenvalue_derivative (:108-168) given E2 = eigval^2
inline float mpml_deriv(float c11, float c13, float c33, float c55, float rho, char dir, float E2, float r,
                        float k1, float k3) {
    const float E4 = E2 * E2;
    const float k12 = k1 * k1, k32 = k3 * k3;
    const float A = (c11 + c55) * k12 + (c33 + c55) * k32;
    const float B = -(c11 * c55) * (k12 * k12) + (c13 * c13 - c11 * c33 + 2 * c13 * c55) * k12 * k32 -
                    (c33 * c55) * (k32 * k32);
    const float den = 2 * B - 3 * E2 * A * rho - 4 * E4 * (rho * rho);
    float num;
    if (dir == 'x') {
        num = 2 * c33 * c55 * (k32 * k32) - c13 * c13 * k12 * k32 * (1 + r) - c13 * k1 * k3 * (k3 * (2 * c55 * k1 * (1 + r))) +
              E2 * (k3 * (c33 * k3 * (2 + r)) + c55 * (k32 * (2 + r) + k12 * (1 + 2 * r))) * rho +
              2 * E4 * (1 + r) * (rho * rho) + c11 * k12 * (2 * c55 * k12 * r + c33 * k32 * (1 + r) + E2 * (1 + 2 * r) * rho);
    } else {
        num = k32 * (-(2 * (-(c33 * c55)) * k32 * r) - c13 * c13 * k12 * (1 + r) - c13 * k1 * (2 * c55 * k1 * (1 + r))) +
              E2 * (k3 * (c33 * k3 * (1 + 2 * r)) + c55 * (k12 * (2 + r) + k32 * (1 + 2 * r))) * rho +
              2 * E4 * (1 + r) * (rho * rho) + c11 * k12 * (2 * c55 * k12 + k3 * (c33 * k3 * (1 + r)) + E2 * (2 + r) * rho);
    }
    return num / den;
}

inline float damp_ratio(float c11, float c13, float c33, float c55, float rho, char dir) {
    const float dtheta = (float)(3.14159265358979323846 / 180.0);
    const float alpha = -0.01f, dratio = 0.002f, sc = 1.0e-9f;
    float ratio = 0.f;
    for (int i = 1; i <= 180; ++i) {
        const float theta = ((float)i + 0.5f) * dtheta;
        const float kx = std::sin(theta), kz = std::cos(theta);
        const float e1 = mpml_eig2(c11, c13, c33, c55, rho, 1, kx, kz);
        const float e2 = mpml_eig2(c11, c13, c33, c55, rho, 2, kx, kz);
        auto deriv = [&](float E2) {
            return mpml_deriv(c11 * sc, c13 * sc, c33 * sc, c55 * sc, rho * sc, dir, E2, ratio, kx, kz);
        };
        float d = std::max(deriv(e1), deriv(e2));
        while (d >= alpha && ratio < 1.0f) {
            ratio = ratio + dratio;
            d = std::max(deriv(e1), deriv(e2));
        }
    }
    return ratio;
}

// elastic damp_coef (module_cfspml.f90:286-327) with kmax = 1; distances are
// already normalised by the PML width
inline void el_damp_coef(float vp, float xdist, float zdist, float dx, float dz, int pml, float dt, float alphamax,
                         float ratiox, float ratioz, float& ax, float& bx, float& az, float& bz) {
    const float R0 = 1.0e-5f;
    float dampx = vp * 3.0f * std::log(1.0f / R0) / (2.0f * (float)pml * dx) * (xdist * xdist);
    float dampz = vp * 3.0f * std::log(1.0f / R0) / (2.0f * (float)pml * dz) * (zdist * zdist);
    const float wx = dampx + ratioz * dampz, wz = dampz + ratiox * dampx;
    dampx = wx;
    dampz = wz;
    const float adt = std::fabs(dt);
    const float alx = std::max(alphamax * (1.0f - xdist), 0.25f * alphamax);
    ax = -2.0f * adt * dampx / 1.0f / (2.0f + adt * (alx + dampx / 1.0f));
    bx = (2.0f - adt * (alx + dampx / 1.0f)) / (2.0f + adt * (alx + dampx / 1.0f));
    const float alz = std::max(alphamax * (1.0f - zdist), 0.25f * alphamax);
    az = -2.0f * adt * dampz / 1.0f / (2.0f + adt * (alz + dampz / 1.0f));
    bz = (2.0f - adt * (alz + dampz / 1.0f)) / (2.0f + adt * (alz + dampz / 1.0f));
}

// 2D coefficient set of one staggered position (ii, hh, hi, ih)
struct Mp2 {
    Arr2<float> ax, bx, az, bz;
    void init(int i0, int i1, int j0, int j1) {
        ax.init(i0, i1, j0, j1); bx.init(i0, i1, j0, j1); az.init(i0, i1, j0, j1); bz.init(i0, i1, j0, j1);
    }
};

template <typename T>
struct El2dState {
    Arr2<T> sxx, szz, sxz, vx, vz;
    Arr2<T> m_dxvx, m_dzvz, m_dzvx, m_dxvz, m_dxxx, m_dzxz, m_dxxz, m_dzzz;
    void init(int a, int b, int c, int d) {
        for (Arr2<T>* x : {&sxx, &szz, &sxz, &vx, &vz, &m_dxvx, &m_dzvz, &m_dzvx, &m_dxvz, &m_dxxx, &m_dzxz,
                           &m_dxxz, &m_dzzz})
            x->init(a, b, c, d);
    }
};

template <typename T>
struct El2d {
    int nx, nz, pml, R, nt, aniso, np;
    int nzm;                          // regular (model) rows; nz: the mesh's rows
    float dx, dz, dt, idx, idz;
    bool fs;
    const float* c;
    ZMesh zm;
    ZLinear zl;
    Arr2<T> c11, c13, c33, c55, rho;  // padded by pml+1, on the mesh's rows
    Arr2<T> c55e;                     // harmonic c55 at the sigma_xz nodes
    std::vector<Arr2<T>> par;         // padded model parameters, regular rows
    Mp2 ii, hh, hi, ih;
    int lo_x, hi_x, lo_z, hi_z;
    float dt_stable = 0;

    El2d(const owl_ssg_desc& d, const T* const* fields) {
        nx = d.nx; nzm = d.nz; pml = d.pml; R = d.fdhalf; nt = d.nt; aniso = d.aniso;
        dx = d.dx; dz = d.dz; dt = d.dt; fs = d.free_surface != 0;
        np = aniso_nparam(aniso);
        if (np < 0) throw std::runtime_error("bad aniso");
        idx = (float)(1.0 / (double)dx);
        idz = (float)(1.0 / (double)dz);
        c = fdcoefs(R);
        const int P = pml;
        zm = zmesh_build(d);
        nz = zm.n;
        if (zm.refined) zl = zlinear_build(zm, nzm, dz);
        // Cij of the regular padded rows
        Arr2<T> r11(-P, nx + P + 1, -P, nzm + P + 1), r13 = r11, r33 = r11, r55 = r11, rr_ = r11;
        par.resize(np);
        for (auto& a : par) a.init(-P, nx + P + 1, -P, nzm + P + 1);
        for (int j = -P; j <= nzm + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                int ii_ = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nzm);
                size_t src = (size_t)(ii_ - 1) * nzm + (jj - 1);
                std::vector<T> p(np);
                for (int q = 0; q < np; ++q) p[q] = par[q](i, j) = fields[q][src];
                to_cij(aniso, p.data(), r11(i, j), r13(i, j), r33(i, j), r55(i, j), rr_(i, j));
            }
        // the mesh's rows (map_regular_to_irregular, module_vars.f90:139-169)
        for (Arr2<T>* a : {&c11, &c13, &c33, &c55, &rho}) a->init(-P, nx + P + 1, -P, nz + P + 1);
        for (int j = -P; j <= nz + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                if (!zm.refined) {
                    c11(i, j) = r11(i, j); c13(i, j) = r13(i, j); c33(i, j) = r33(i, j); c55(i, j) = r55(i, j);
                    rho(i, j) = rr_(i, j);
                    continue;
                }
                const int j0 = zl.j0(j);
                const T w = T(zl.w(j));
                c11(i, j) = r11(i, j0) + w * (r11(i, j0 + 1) - r11(i, j0));
                c13(i, j) = r13(i, j0) + w * (r13(i, j0 + 1) - r13(i, j0));
                c33(i, j) = r33(i, j0) + w * (r33(i, j0 + 1) - r33(i, j0));
                c55(i, j) = r55(i, j0) + w * (r55(i, j0 + 1) - r55(i, j0));
                rho(i, j) = rr_(i, j0) + w * (rr_(i, j0 + 1) - rr_(i, j0));
            }
        c55e.init(-P + 1, nx + P, -P + 1, nz + P);
        for (int n = -P + 1; n <= nz + P; ++n)
            for (int m = -P + 1; m <= nx + P; ++m) {
                T s = T(1) / c55(m - 1, n - 1) + T(1) / c55(m, n - 1) + T(1) / c55(m - 1, n) + T(1) / c55(m, n);
                c55e(m, n) = T(4) / s;
            }
        // pmlvp of the regular model's edges (module_vars.f90:298-302) and dt_stable
        // (:381-420: on the refined mesh the least over the cells, each with its
        // row's smaller spacing)
        float pv = -1e30f, maxv = 0.f;
        for (int j = 1; j <= nzm; ++j)
            for (int i : {1, nx}) {
                pv = std::max(pv, (float)re(r11(i, j)) / (float)re(rr_(i, j)));
                pv = std::max(pv, (float)re(r33(i, j)) / (float)re(rr_(i, j)));
            }
        for (int i = 1; i <= nx; ++i)
            for (int j : {1, nzm}) {
                pv = std::max(pv, (float)re(r11(i, j)) / (float)re(rr_(i, j)));
                pv = std::max(pv, (float)re(r33(i, j)) / (float)re(rr_(i, j)));
            }
        const float pmlvp = std::sqrt(pv);
        float temp = 0.f;
        for (int k = 0; k < R; ++k) temp += std::fabs(c[k]);
        if (!zm.refined) {
            for (int j = 1; j <= nz; ++j)
                for (int i = 1; i <= nx; ++i)
                    maxv = std::max({maxv, std::sqrt((float)re(c11(i, j)) / (float)re(rho(i, j))),
                                     std::sqrt((float)re(c33(i, j)) / (float)re(rho(i, j)))});
            dt_stable = 1.0f / (temp * maxv * std::sqrt(1.0f / (dx * dx) + 1.0f / (dz * dz)));
        } else {
            float best = 3.0e38f;
            for (int j = 1; j <= nz; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const float mv = std::max(std::sqrt((float)re(c11(i, j)) / (float)re(rho(i, j))),
                                              std::sqrt((float)re(c33(i, j)) / (float)re(rho(i, j))));
                    const float h = std::min(zm.dzi(j), zm.dzh(j));
                    best = std::min(best, 1.0f / (temp * mv * std::sqrt(1.0f / (dx * dx) + 1.0f / (h * h))));
                }
            dt_stable = best;
        }
        // M-PML ratios (module_cfspml.f90:229-276), zero for the isotropic parameterisation
        Arr1<float> rl, rr, rt, rb;
        rl.init(-P, nz + P + 1, 0.f); rr.init(-P, nz + P + 1, 0.f);
        rt.init(-P, nx + P + 1, 0.f); rb.init(-P, nx + P + 1, 0.f);
        if (aniso != OWL_ANISO_ISO) {
            auto f = [&](int i, int j, char dir) {
                return damp_ratio((float)re(c11(i, j)), (float)re(c13(i, j)), (float)re(c33(i, j)),
                                  (float)re(c55(i, j)), (float)re(rho(i, j)), dir);
            };
            for (int j = -P; j <= nz + P + 1; ++j) { rl(j) = f(1, j, 'x'); rr(j) = f(nx, j, 'x'); }
            for (int i = -P; i <= nx + P + 1; ++i) { rt(i) = f(i, 1, 'z'); rb(i) = f(i, nz, 'z'); }
        }
        // 2D CFS-MPML coefficients (module_cfspml.f90:329-575)
        const float alphamax = (float)(1.0 * (double)d.f0_max * 3.14159265358979323846);
        for (Mp2* m : {&ii, &hh, &hi, &ih}) m->init(-P + 1, nx + P, -P + 1, nz + P);
        for (int j = -P + 1; j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                float xdi = 0.f, xdh = 0.f, zdi = 0.f, zdh = 0.f;
                if (i <= 1) {
                    xdi = (float)std::fabs((i - 1 + 0.0) / P);
                    xdh = (float)std::fabs((i - 1 - 0.5) / P);
                } else if (i >= nx) {
                    xdi = (float)std::fabs((i - nx + 0.0) / P);
                    xdh = (float)std::fabs((i - nx - 0.5) / P);
                }
                if (j <= 1) {
                    zdi = (float)std::fabs((j - 1 + 0.0) / P);
                    zdh = (float)std::fabs((j - 1 - 0.5) / P);
                } else if (j >= nz) {
                    zdi = (float)std::fabs((j - nz + 0.0) / P);
                    zdh = (float)std::fabs((j - nz - 0.5) / P);
                }
                if (i > 1 && i < nx && j > 1 && j < nz) continue;
                float rx = 0.f, rz = 0.f;
                if (i <= 1) rx = rl(j); else if (i >= nx) rx = rr(j);
                if (j <= 1) rz = rt(i); else if (j >= nz) rz = rb(i);
                // the row's own dz_i(j) on the refined mesh (module_cfspml.f90:446-473)
                const float dzj = zm.refined ? zm.dzi(j) : dz;
                auto set = [&](Mp2& m, float xd, float zd) {
                    el_damp_coef(pmlvp, xd, zd, dx, dzj, P, dt, alphamax, rx, rz, m.ax(i, j), m.bx(i, j), m.az(i, j),
                                 m.bz(i, j));
                };
                set(ii, xdi, zdi);
                set(ih, xdi, zdh);
                set(hi, xdh, zdi);
                set(hh, xdh, zdh);
            }
        lo_x = -P - R + 1; hi_x = nx + P + R;
        lo_z = -P - R + 1; hi_z = nz + P + R;
    }

    // dz scalings of the z derivatives at integer / half rows (1 on the uniform grid)
    T zsi(int j) const { return zm.refined ? T(zm.si(j)) : T(1); }
    T zsh(int j) const { return zm.refined ? T(zm.sh(j)) : T(1); }
    // local spacing of an explosion / moment-tensor source's row (dz_s, module_wavefield.f90:305-309)
    float dz_src(int gz) const { return zm.refined ? zm.dzi(gz) : dz; }

    // PML membership of the owner node of each field
    bool in_ii(int i, int j) const { return i <= 0 || i >= nx + 1 || (!fs && j <= 0) || j >= nz + 1; }
    bool in_hh(int m, int n) const { return m <= 1 || m >= nx + 1 || (!fs && n <= 1) || n >= nz + 1; }
    bool in_hi(int m, int j) const { return m <= 1 || m >= nx + 1 || (!fs && j <= 0) || j >= nz + 1; }
    bool in_ih(int i, int n) const { return i <= 0 || i >= nx + 1 || (!fs && n <= 1) || n >= nz + 1; }

    // first owner row of each field
    int js() const { return fs ? 1 : -pml + 1; }   // sigma_xx, sigma_zz
    int jxz() const { return fs ? 2 : -pml + 1; }  // sigma_xz (n)
    int jvx() const { return fs ? 1 : -pml + 1; }  // vx
    int jvz() const { return fs ? 2 : -pml + 1; }  // vz (n)

    // one forward update. S (optional): 5 stored stencil terms (see header of the file)
    void update(El2dState<T>& s, Arr2<T>* S) const {
        const int P = pml;
        if (fs) {
            for (int j = 1; j <= R; ++j)
                for (int i = lo_x; i <= hi_x; ++i) {
                    s.vx(i, 1 - j) = T(0);
                    s.vz(i, 2 - j) = T(0);
                }
        }
        // sigma_xx, sigma_zz
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = js(); j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T sx = T(0), sz = T(0);
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.vx(i + k, j) - s.vx(i - k + 1, j));
                T pdxvx = T(idx) * sx, pdzvz;
                if (fs && j == 1) {
                    if (i <= 0 || i >= nx + 1) {
                        s.m_dxvx(i, j) = T(ii.ax(i, j)) * pdxvx + T(ii.bx(i, j)) * s.m_dxvx(i, j);
                        pdxvx = pdxvx + s.m_dxvx(i, j);
                    }
                    pdzvz = -(c13(i, j) / c33(i, j) * pdxvx);
                } else {
                    for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.vz(i, j + k) - s.vz(i, j - k + 1));
                    pdzvz = T(idz) * sz * zsi(j);
                    if (in_ii(i, j)) {
                        s.m_dxvx(i, j) = T(ii.ax(i, j)) * pdxvx + T(ii.bx(i, j)) * s.m_dxvx(i, j);
                        pdxvx = pdxvx + s.m_dxvx(i, j);
                        s.m_dzvz(i, j) = T(ii.az(i, j)) * pdzvz + T(ii.bz(i, j)) * s.m_dzvz(i, j);
                        pdzvz = pdzvz + s.m_dzvz(i, j);
                    }
                }
                s.sxx(i, j) = s.sxx(i, j) + T(dt) * (c11(i, j) * pdxvx + c13(i, j) * pdzvz);
                s.szz(i, j) = s.szz(i, j) + T(dt) * (c13(i, j) * pdxvx + c33(i, j) * pdzvz);
                if (S) { S[0](i, j) = pdxvx; S[1](i, j) = pdzvz; }
            }
        // sigma_xz at (m, n) = (i+1, j+1)
#pragma omp parallel for collapse(2) schedule(static)
        for (int n = jxz(); n <= nz + P; ++n)
            for (int m = -P + 1; m <= nx + P; ++m) {
                T sz = T(0), sx = T(0);
                for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.vx(m, n - 1 + k) - s.vx(m, n - k));
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.vz(m - 1 + k, n) - s.vz(m - k, n));
                T pdzvx = T(idz) * sz * zsh(n), pdxvz = T(idx) * sx;
                if (in_hh(m, n)) {
                    s.m_dxvz(m, n) = T(hh.ax(m, n)) * pdxvz + T(hh.bx(m, n)) * s.m_dxvz(m, n);
                    pdxvz = pdxvz + s.m_dxvz(m, n);
                    s.m_dzvx(m, n) = T(hh.az(m, n)) * pdzvx + T(hh.bz(m, n)) * s.m_dzvx(m, n);
                    pdzvx = pdzvx + s.m_dzvx(m, n);
                }
                s.sxz(m, n) = s.sxz(m, n) + T(dt) * c55e(m, n) * (pdzvx + pdxvz);
                if (S) S[2](m, n) = pdzvx + pdxvz;
            }
        if (fs) {
            for (int j = 1; j <= R; ++j)
                for (int i = lo_x; i <= hi_x; ++i) {
                    s.szz(i, 1 - j) = -s.szz(i, 1 + j);
                    s.szz(i, 1) = T(0);
                    s.sxx(i, 1 - j) = -s.sxx(i, 1 + j);
                    s.sxz(i, 2 - j) = -s.sxz(i, 1 + j);
                }
        }
        // vx at (m, j)
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = jvx(); j <= nz + P; ++j)
            for (int m = -P + 1; m <= nx + P; ++m) {
                T sx = T(0), sz = T(0);
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.sxx(m - 1 + k, j) - s.sxx(m - k, j));
                for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.sxz(m, j + k) - s.sxz(m, j - k + 1));
                T pdxxx = T(idx) * sx, pdzxz = T(idz) * sz * zsi(j);
                if (in_hi(m, j)) {
                    s.m_dxxx(m, j) = T(hi.ax(m, j)) * pdxxx + T(hi.bx(m, j)) * s.m_dxxx(m, j);
                    pdxxx = pdxxx + s.m_dxxx(m, j);
                    s.m_dzxz(m, j) = T(hi.az(m, j)) * pdzxz + T(hi.bz(m, j)) * s.m_dzxz(m, j);
                    pdzxz = pdzxz + s.m_dzxz(m, j);
                }
                T rx = T(0.5f) * (rho(m - 1, j) + rho(m, j));
                s.vx(m, j) = s.vx(m, j) + T(dt) / rx * (pdxxx + pdzxz);
                if (S) S[3](m, j) = pdxxx + pdzxz;
            }
        // vz at (i, n)
#pragma omp parallel for collapse(2) schedule(static)
        for (int n = jvz(); n <= nz + P; ++n)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T sx = T(0), sz = T(0);
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.sxz(i + k, n) - s.sxz(i - k + 1, n));
                for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.szz(i, n - 1 + k) - s.szz(i, n - k));
                T pdxxz = T(idx) * sx, pdzzz = T(idz) * sz * zsh(n);
                if (in_ih(i, n)) {
                    s.m_dxxz(i, n) = T(ih.ax(i, n)) * pdxxz + T(ih.bx(i, n)) * s.m_dxxz(i, n);
                    pdxxz = pdxxz + s.m_dxxz(i, n);
                    s.m_dzzz(i, n) = T(ih.az(i, n)) * pdzzz + T(ih.bz(i, n)) * s.m_dzzz(i, n);
                    pdzzz = pdzzz + s.m_dzzz(i, n);
                }
                T rz = T(0.5f) * (rho(i, n - 1) + rho(i, n));
                s.vz(i, n) = s.vz(i, n) + T(dt) / rz * (pdxxz + pdzzz);
                if (S) S[4](i, n) = pdxxz + pdzzz;
            }
    }

    // source amplitude of step t (0 outside the STF window)
    static bool amp_at(const owl_source& q, int t, float dt, T& amp) {
        if (t < q.nbeg || t > q.nbeg + q.nt_stf - 1) return false;
        amp = T(q.stf[t - q.nbeg]) * T(q.amp) * T(dt);
        return true;
    }

    void add_source(int t, const owl_shot& sh, El2dState<T>& s) const {
        for (int k = 0; k < sh.nsrc; ++k) {
            const owl_source& q = sh.src[k];
            T amp;
            if (!amp_at(q, t, dt, amp)) continue;
            if (q.mechanism == OWL_SRC_FORCE) {
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx) {
                        if (!fs || q.gz + irz >= 2)
                            s.vx(q.hx + irx, q.gz + irz) = s.vx(q.hx + irx, q.gz + irz) +
                                T(std::sin(q.polar)) * amp / rho(q.hx, q.gz) * T(q.interp_hx[irx + 4]) * T(q.interp_iz[irz + 4]);
                        if (!fs || q.hz + irz >= 2)
                            s.vz(q.gx + irx, q.hz + irz) = s.vz(q.gx + irx, q.hz + irz) +
                                T(std::cos(q.polar)) * amp / rho(q.gx, q.hz) * T(q.interp_ix[irx + 4]) * T(q.interp_hz[irz + 4]);
                    }
            } else {
                const T a = amp / (T(dx) * T(dz_src(q.gz)));
                const bool mt = q.mechanism == OWL_SRC_MT;
                const T mxx = mt ? T(q.mt[0]) : T(1), mzz = mt ? T(q.mt[2]) : T(1), mxz = T(q.mt[4]);
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx) {
                        if (!fs || q.gz + irz >= 2) {
                            T w = T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]);
                            s.sxx(q.gx + irx, q.gz + irz) = s.sxx(q.gx + irx, q.gz + irz) - a * mxx * w;
                            s.szz(q.gx + irx, q.gz + irz) = s.szz(q.gx + irx, q.gz + irz) - a * mzz * w;
                        }
                        if (mt && (!fs || q.hz + irz >= 2))
                            s.sxz(q.hx + irx, q.hz + irz) = s.sxz(q.hx + irx, q.hz + irz) -
                                a * mxz * T(q.interp_hx[irx + 4]) * T(q.interp_hz[irz + 4]);
                    }
            }
        }
    }

    // near-surface images before sampling (submodule_forward_modeling.f90:75-83)
    void images(El2dState<T>& s) const {
        for (int j = 1; j <= R; ++j)
            for (int i = lo_x; i <= hi_x; ++i) {
                s.vx(i, 1 - j) = s.vx(i, 1 + j);
                s.vz(i, 2 - j) = s.vz(i, 1 + j);
            }
    }

    // sampling of step t: out[(comp*nrec + r)*nt + t-1], comp 0 = vx, 1 = vz
    void sample(int t, const owl_shot& sh, const El2dState<T>& s, T* out) const {
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T ax = T(0), az = T(0);
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx)
                    ax = ax + s.vx(q.hx + irx, q.gz + irz) * T(q.interp_hx[irx + 4]) * T(q.interp_iz[irz + 4]) * T(q.weight);
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx)
                    az = az + s.vz(q.gx + irx, q.hz + irz) * T(q.interp_ix[irx + 4]) * T(q.interp_hz[irz + 4]) * T(q.weight);
            out[(size_t)r * nt + (t - 1)] = ax;
            out[((size_t)sh.nrec + r) * nt + (t - 1)] = az;
        }
    }

    void forward_shot(const owl_shot& sh, T* seis, std::vector<El2dState<T>>* ckpt, int k) const {
        El2dState<T> s;
        s.init(lo_x, hi_x, lo_z, hi_z);
        std::fill(seis, seis + (size_t)2 * sh.nrec * nt, T(0));
        for (int t = 1; t <= nt; ++t) {
            if (ckpt && (t - 1) % k == 0) ckpt->push_back(s);
            if (fs) images(s);
            sample(t, sh, s, seis);
            update(s, nullptr);
            add_source(t, sh, s);
        }
    }

    // ---------------- exact discrete adjoint -----------------------------------
    struct Grad {
        Arr2<T> g11, g13, g33, g55, grho;  // d J / d (c11, c13, c33, c55, rho), padded model grid
        std::vector<Arr2<T>> gpar;
    };

    // adjoint PML term of one derivative: q = adjoint of the PML-corrected
    // derivative, psi^ = adjoint of its memory variable
    static T pml_e(T q, float a, float b, T& psih) {
        T u = q + psih;
        psih = T(b) * u;
        return q + T(a) * u;
    }

    void adjoint_step(int t, const owl_shot& sh, El2dState<T>& a, Arr2<T>* S, const T* res, Grad& g,
                      T* stf_grad) const {
        const int P = pml;
        // add_source(t)
        for (int kk = 0; kk < sh.nsrc; ++kk) {
            const owl_source& q = sh.src[kk];
            T amp;
            if (!amp_at(q, t, dt, amp)) continue;
            T dstf = T(0);
            if (q.mechanism == OWL_SRC_FORCE) {
                T ax = T(0), az = T(0);
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx) {
                        if (!fs || q.gz + irz >= 2)
                            ax = ax + a.vx(q.hx + irx, q.gz + irz) * T(q.interp_hx[irx + 4]) * T(q.interp_iz[irz + 4]);
                        if (!fs || q.hz + irz >= 2)
                            az = az + a.vz(q.gx + irx, q.hz + irz) * T(q.interp_ix[irx + 4]) * T(q.interp_hz[irz + 4]);
                    }
                T sx = T(std::sin(q.polar)), sz = T(std::cos(q.polar));
                dstf = (sx * ax / rho(q.hx, q.gz) + sz * az / rho(q.gx, q.hz)) * T(q.amp) * T(dt);
                g.grho(q.hx, q.gz) = g.grho(q.hx, q.gz) - sx * amp * ax / (rho(q.hx, q.gz) * rho(q.hx, q.gz));
                g.grho(q.gx, q.hz) = g.grho(q.gx, q.hz) - sz * amp * az / (rho(q.gx, q.hz) * rho(q.gx, q.hz));
            } else {
                const bool mt = q.mechanism == OWL_SRC_MT;
                const T mxx = mt ? T(q.mt[0]) : T(1), mzz = mt ? T(q.mt[2]) : T(1), mxz = T(q.mt[4]);
                T acc = T(0);
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx) {
                        if (!fs || q.gz + irz >= 2) {
                            T w = T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]);
                            acc = acc + (mxx * a.sxx(q.gx + irx, q.gz + irz) + mzz * a.szz(q.gx + irx, q.gz + irz)) * w;
                        }
                        if (mt && (!fs || q.hz + irz >= 2))
                            acc = acc + mxz * a.sxz(q.hx + irx, q.hz + irz) * T(q.interp_hx[irx + 4]) * T(q.interp_hz[irz + 4]);
                    }
                dstf = -acc * T(q.amp) * T(dt) / (T(dx) * T(dz_src(q.gz)));
            }
            if (stf_grad) stf_grad[(size_t)kk * nt + (t - 1)] = stf_grad[(size_t)kk * nt + (t - 1)] + dstf;
        }
        // reverse the vz update
        for (int n = jvz(); n <= nz + P; ++n)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T rz = T(0.5f) * (rho(i, n - 1) + rho(i, n));
                T zh = a.vz(i, n);
                T gr = -zh * S[4](i, n) * T(dt) * T(0.5f) / (rz * rz);
                g.grho(i, n - 1) = g.grho(i, n - 1) + gr;
                g.grho(i, n) = g.grho(i, n) + gr;
                T q = T(dt) / rz * zh;
                T ex = q, ez = q;
                if (in_ih(i, n)) {
                    ex = pml_e(q, ih.ax(i, n), ih.bx(i, n), a.m_dxxz(i, n));
                    ez = pml_e(q, ih.az(i, n), ih.bz(i, n), a.m_dzzz(i, n));
                }
                ex = T(idx) * ex;
                ez = T(idz) * zsh(n) * ez;
                for (int k = 1; k <= R; ++k) {
                    a.sxz(i + k, n) = a.sxz(i + k, n) + T(c[k - 1]) * ex;
                    a.sxz(i - k + 1, n) = a.sxz(i - k + 1, n) - T(c[k - 1]) * ex;
                    a.szz(i, n - 1 + k) = a.szz(i, n - 1 + k) + T(c[k - 1]) * ez;
                    a.szz(i, n - k) = a.szz(i, n - k) - T(c[k - 1]) * ez;
                }
            }
        // reverse the vx update
        for (int j = jvx(); j <= nz + P; ++j)
            for (int m = -P + 1; m <= nx + P; ++m) {
                T rx = T(0.5f) * (rho(m - 1, j) + rho(m, j));
                T xh = a.vx(m, j);
                T gr = -xh * S[3](m, j) * T(dt) * T(0.5f) / (rx * rx);
                g.grho(m - 1, j) = g.grho(m - 1, j) + gr;
                g.grho(m, j) = g.grho(m, j) + gr;
                T q = T(dt) / rx * xh;
                T ex = q, ez = q;
                if (in_hi(m, j)) {
                    ex = pml_e(q, hi.ax(m, j), hi.bx(m, j), a.m_dxxx(m, j));
                    ez = pml_e(q, hi.az(m, j), hi.bz(m, j), a.m_dzxz(m, j));
                }
                ex = T(idx) * ex;
                ez = T(idz) * zsi(j) * ez;
                for (int k = 1; k <= R; ++k) {
                    a.sxx(m - 1 + k, j) = a.sxx(m - 1 + k, j) + T(c[k - 1]) * ex;
                    a.sxx(m - k, j) = a.sxx(m - k, j) - T(c[k - 1]) * ex;
                    a.sxz(m, j + k) = a.sxz(m, j + k) + T(c[k - 1]) * ez;
                    a.sxz(m, j - k + 1) = a.sxz(m, j - k + 1) - T(c[k - 1]) * ez;
                }
            }
        // reverse the surface mirror and sigma_zz(., 1) = 0
        if (fs) {
            for (int j = R; j >= 1; --j)
                for (int i = lo_x; i <= hi_x; ++i) {
                    a.sxz(i, 1 + j) = a.sxz(i, 1 + j) - a.sxz(i, 2 - j);
                    a.sxz(i, 2 - j) = T(0);
                    a.sxx(i, 1 + j) = a.sxx(i, 1 + j) - a.sxx(i, 1 - j);
                    a.sxx(i, 1 - j) = T(0);
                    a.szz(i, 1) = T(0);
                    a.szz(i, 1 + j) = a.szz(i, 1 + j) - a.szz(i, 1 - j);
                    a.szz(i, 1 - j) = T(0);
                }
        }
        // reverse the sigma_xz update
        for (int n = jxz(); n <= nz + P; ++n)
            for (int m = -P + 1; m <= nx + P; ++m) {
                T sh_ = a.sxz(m, n);
                T g55e = T(dt) * sh_ * S[2](m, n);
                // c55e = 4 / sum(1/c55) over the 4 surrounding cells
                const int cm[4] = {m - 1, m, m - 1, m}, cn[4] = {n - 1, n - 1, n, n};
                if (re(c55e(m, n)) != 0)
                    for (int q = 0; q < 4; ++q) {
                        T cc = c55(cm[q], cn[q]);
                        g.g55(cm[q], cn[q]) = g.g55(cm[q], cn[q]) + g55e * c55e(m, n) * c55e(m, n) / (T(4) * cc * cc);
                    }
                T q = T(dt) * c55e(m, n) * sh_;
                T ez = q, ex = q;
                if (in_hh(m, n)) {
                    ex = pml_e(q, hh.ax(m, n), hh.bx(m, n), a.m_dxvz(m, n));
                    ez = pml_e(q, hh.az(m, n), hh.bz(m, n), a.m_dzvx(m, n));
                }
                ez = T(idz) * zsh(n) * ez;
                ex = T(idx) * ex;
                for (int k = 1; k <= R; ++k) {
                    a.vx(m, n - 1 + k) = a.vx(m, n - 1 + k) + T(c[k - 1]) * ez;
                    a.vx(m, n - k) = a.vx(m, n - k) - T(c[k - 1]) * ez;
                    a.vz(m - 1 + k, n) = a.vz(m - 1 + k, n) + T(c[k - 1]) * ex;
                    a.vz(m - k, n) = a.vz(m - k, n) - T(c[k - 1]) * ex;
                }
            }
        // reverse the sigma_xx / sigma_zz update
        for (int j = js(); j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T xh = a.sxx(i, j), zh = a.szz(i, j);
                T ex, ez = T(0);
                if (fs && j == 1) {
                    // pdzvz = -(c13 / c33) pdxvx; sigma_zz(., 1) is overwritten by 0
                    const T r = c13(i, j) / c33(i, j);
                    g.g11(i, j) = g.g11(i, j) + T(dt) * xh * S[0](i, j);
                    g.g13(i, j) = g.g13(i, j) - T(dt) * xh * T(2) * r * S[0](i, j);
                    g.g33(i, j) = g.g33(i, j) + T(dt) * xh * r * r * S[0](i, j);
                    T q = T(dt) * c11(i, j) * xh - r * (T(dt) * c13(i, j) * xh);
                    ex = q;
                    if (i <= 0 || i >= nx + 1) ex = pml_e(q, ii.ax(i, j), ii.bx(i, j), a.m_dxvx(i, j));
                } else {
                    g.g11(i, j) = g.g11(i, j) + T(dt) * xh * S[0](i, j);
                    g.g13(i, j) = g.g13(i, j) + T(dt) * (xh * S[1](i, j) + zh * S[0](i, j));
                    g.g33(i, j) = g.g33(i, j) + T(dt) * zh * S[1](i, j);
                    T qx = T(dt) * (c11(i, j) * xh + c13(i, j) * zh);
                    T qz = T(dt) * (c13(i, j) * xh + c33(i, j) * zh);
                    ex = qx;
                    ez = qz;
                    if (in_ii(i, j)) {
                        ex = pml_e(qx, ii.ax(i, j), ii.bx(i, j), a.m_dxvx(i, j));
                        ez = pml_e(qz, ii.az(i, j), ii.bz(i, j), a.m_dzvz(i, j));
                    }
                }
                ex = T(idx) * ex;
                ez = T(idz) * zsi(j) * ez;
                for (int k = 1; k <= R; ++k) {
                    a.vx(i + k, j) = a.vx(i + k, j) + T(c[k - 1]) * ex;
                    a.vx(i - k + 1, j) = a.vx(i - k + 1, j) - T(c[k - 1]) * ex;
                    a.vz(i, j + k) = a.vz(i, j + k) + T(c[k - 1]) * ez;
                    a.vz(i, j - k + 1) = a.vz(i, j - k + 1) - T(c[k - 1]) * ez;
                }
            }
        // the surface rows zeroed at the top of update() and everything outside
        // each field's update range are constants: their adjoint is dropped
        clear_outside(a);
        // sampling of step t, with the surface images folded back
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T rvx = res[(size_t)r * nt + (t - 1)], rvz = res[((size_t)sh.nrec + r) * nt + (t - 1)];
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx) {
                    a.vx(q.hx + irx, q.gz + irz) = a.vx(q.hx + irx, q.gz + irz) +
                        rvx * T(q.interp_hx[irx + 4]) * T(q.interp_iz[irz + 4]) * T(q.weight);
                    a.vz(q.gx + irx, q.hz + irz) = a.vz(q.gx + irx, q.hz + irz) +
                        rvz * T(q.interp_ix[irx + 4]) * T(q.interp_hz[irz + 4]) * T(q.weight);
                }
        }
        if (fs) {
            for (int j = R; j >= 1; --j)
                for (int i = lo_x; i <= hi_x; ++i) {
                    a.vx(i, 1 + j) = a.vx(i, 1 + j) + a.vx(i, 1 - j);
                    a.vx(i, 1 - j) = T(0);
                    a.vz(i, 1 + j) = a.vz(i, 1 + j) + a.vz(i, 2 - j);
                    a.vz(i, 2 - j) = T(0);
                }
        }
        clear_outside(a);
    }

    void clear_outside(El2dState<T>& a) const {
        const int P = pml;
        for (int j = lo_z; j <= hi_z; ++j)
            for (int i = lo_x; i <= hi_x; ++i) {
                bool inx = i >= -P + 1 && i <= nx + P, inz = j <= nz + P;
                if (!(inx && inz && j >= js())) { a.sxx(i, j) = T(0); a.szz(i, j) = T(0); }
                if (!(inx && inz && j >= jxz())) a.sxz(i, j) = T(0);
                if (!(inx && inz && j >= jvx())) a.vx(i, j) = T(0);
                if (!(inx && inz && j >= jvz())) a.vz(i, j) = T(0);
            }
    }

    void adjoint_shot(const owl_shot& sh, const T* res, int k, Grad& g, T* stf_grad) const {
        std::vector<El2dState<T>> ck;
        std::vector<T> dummy((size_t)2 * sh.nrec * nt);
        forward_shot(sh, dummy.data(), &ck, k);
        El2dState<T> a;
        a.init(lo_x, hi_x, lo_z, hi_z);
        int nseg = (int)ck.size();
        std::vector<std::array<Arr2<T>, 5>> Sbuf((size_t)k);
        for (auto& s5 : Sbuf)
            for (auto& arr : s5) arr.init(lo_x, hi_x, lo_z, hi_z);
        for (int sg = nseg - 1; sg >= 0; --sg) {
            int n0 = sg * k, n1 = std::min(nt, n0 + k);
            El2dState<T> s = ck[sg];
            for (int t = n0 + 1; t <= n1; ++t) {
                if (fs) images(s);
                update(s, Sbuf[t - n0 - 1].data());
                add_source(t, sh, s);
            }
            for (int t = n1; t >= n0 + 1; --t) adjoint_step(t, sh, a, Sbuf[t - n0 - 1].data(), res, g, stf_grad);
        }
    }

    // parameter gradients on the padded grid from d J / d (c11, c13, c33, c55, rho):
    // the Jacobian of to_cij by complex-step differentiation of each parameter
    // (on the refined mesh: first the transpose of the row interpolation, from
    // the mesh rows to the regular rows)
    void chain(Grad& g) const {
        typedef std::complex<double> C;
        const int P = pml;
        std::array<Arr2<T>, 5> rg;
        const Arr2<T>* src[5] = {&g.g11, &g.g13, &g.g33, &g.g55, &g.grho};
        if (zm.refined) {
            for (auto& a : rg) a.init(-P, nx + P + 1, -P, nzm + P + 1);
            for (int f = -P; f <= nz + P + 1; ++f) {
                const int j0 = zl.j0(f);
                const T w = T(zl.w(f));
                for (int q = 0; q < 5; ++q)
                    for (int i = -P; i <= nx + P + 1; ++i) {
                        const T v = (*src[q])(i, f);
                        rg[q](i, j0) = rg[q](i, j0) + (T(1) - w) * v;
                        rg[q](i, j0 + 1) = rg[q](i, j0 + 1) + w * v;
                    }
            }
            for (int q = 0; q < 5; ++q) src[q] = &rg[q];
        }
        g.gpar.assign(np, Arr2<T>(-P, nx + P + 1, -P, nzm + P + 1));
        for (int j = -P; j <= nzm + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                const T dc[5] = {(*src[0])(i, j), (*src[1])(i, j), (*src[2])(i, j), (*src[3])(i, j), (*src[4])(i, j)};
                for (int q = 0; q < np; ++q) {
                    std::vector<C> p(np);
                    for (int r = 0; r < np; ++r) p[r] = C(re(par[r](i, j)), r == q ? 1e-30 : 0.0);
                    C o[5];
                    to_cij(aniso, p.data(), o[0], o[1], o[2], o[3], o[4]);
                    T acc = T(0);
                    for (int r = 0; r < 5; ++r) acc = acc + dc[r] * T(o[r].imag() / 1e-30);
                    g.gpar[q](i, j) = acc;
                }
            }
    }

    void fold(const Arr2<T>& gp, T* out) const {
        std::fill(out, out + (size_t)nx * nzm, T(0));
        for (int j = gp.j0; j <= gp.j1; ++j)
            for (int i = gp.i0; i <= gp.i1; ++i) {
                int ii_ = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nzm);
                out[(size_t)(ii_ - 1) * nzm + (jj - 1)] += gp(i, j);
            }
    }
};

}  // namespace oracle

// ---------------------------------------------------------------------------
// C entry points used by the Python test harness (ctypes)
// ---------------------------------------------------------------------------
using namespace oracle;

static size_t seis_len(const owl_ssg_desc* d, int nshots, const owl_shot* shots) {
    size_t n = 0;
    for (int s = 0; s < nshots; ++s) n += (size_t)2 * shots[s].nrec * d->nt;
    return n;
}

template <typename T>
static int el_fwd_impl(const owl_ssg_desc* d, const T* const* f, int nshots, const owl_shot* shots, T* seis) {
    try {
        El2d<T> m(*d, f);
        size_t off = 0;
        for (int s = 0; s < nshots; ++s) {
            m.forward_shot(shots[s], seis + off, nullptr, 1 << 30);
            off += (size_t)2 * shots[s].nrec * d->nt;
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" int oracle_el2d_forward_f32(const owl_ssg_desc* d, const float* const* f, int nshots,
                                       const owl_shot* shots, float* seis) {
    return el_fwd_impl<float>(d, f, nshots, shots, seis);
}

extern "C" int oracle_el2d_forward_f64(const owl_ssg_desc* d, const double* const* f, int nshots,
                                       const owl_shot* shots, double* seis) {
    return el_fwd_impl<double>(d, f, nshots, shots, seis);
}

extern "C" int oracle_el2d_jvp_c128(const owl_ssg_desc* d, const double* const* f, const double* const* df,
                                    int nshots, const owl_shot* shots, double* seis, double* jvp) {
    typedef std::complex<double> C;
    const double h = 1e-30;
    const int np = aniso_nparam(d->aniso);
    if (np < 0) return -1;
    const size_t n = (size_t)d->nx * d->nz;
    std::vector<std::vector<C>> cf(np, std::vector<C>(n));
    std::vector<const C*> ptr(np);
    for (int q = 0; q < np; ++q) {
        for (size_t i = 0; i < n; ++i) cf[q][i] = C(f[q][i], h * df[q][i]);
        ptr[q] = cf[q].data();
    }
    std::vector<C> out(seis_len(d, nshots, shots));
    int rc = el_fwd_impl<C>(d, ptr.data(), nshots, shots, out.data());
    for (size_t i = 0; i < out.size(); ++i) {
        if (seis) seis[i] = out[i].real();
        jvp[i] = out[i].imag() / h;
    }
    return rc;
}

extern "C" int oracle_el2d_gradient_f64(const owl_ssg_desc* d, const double* const* f, int nshots,
                                        const owl_shot* shots, const double* data, int adj_kind, int k,
                                        double* misfit, double* grad, double* stf_grad) {
    try {
        El2d<double> m(*d, f);
        El2d<double>::Grad g;
        const int P = m.pml;
        for (Arr2<double>* a : {&g.g11, &g.g13, &g.g33, &g.g55, &g.grho}) a->init(-P, m.nx + P + 1, -P, m.nz + P + 1);
        size_t off = 0, soff = 0;
        for (int s = 0; s < nshots; ++s) {
            const owl_shot& sh = shots[s];
            const size_t n = (size_t)2 * sh.nrec * d->nt;
            std::vector<double> res(n, 0.0);
            if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
                std::vector<double> syn(n);
                m.forward_shot(sh, syn.data(), nullptr, 1 << 30);
                double mf = 0;
                for (int comp = 0; comp < 2; ++comp)
                    for (int r = 0; r < sh.nrec; ++r) {
                        if (sh.rec[r].weight == 0.f) continue;
                        for (int t = 0; t < d->nt; ++t) {
                            size_t q = ((size_t)comp * sh.nrec + r) * d->nt + t;
                            res[q] = syn[q] - data[off + q];
                            mf += (data[off + q] - syn[q]) * (data[off + q] - syn[q]);
                        }
                    }
                if (misfit) misfit[s] = mf;
            } else {
                for (size_t q = 0; q < n; ++q) res[q] = data[off + q];
                if (misfit) misfit[s] = 0;
            }
            m.adjoint_shot(sh, res.data(), k, g, stf_grad ? stf_grad + soff : nullptr);
            off += n;
            soff += (size_t)sh.nsrc * d->nt;
        }
        m.chain(g);
        const size_t nm = (size_t)d->nx * d->nz;
        for (int q = 0; q < m.np; ++q) m.fold(g.gpar[q], grad + q * nm);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

// Cij (c11, c13, c33, c55, rho) of the padded model, the M-PML ratio of one
// cell, and dt_stable: set-up pieces checked directly by the tests
extern "C" int oracle_el2d_setup(const owl_ssg_desc* d, const float* const* f, float* dt_stable) {
    try {
        El2d<float> m(*d, f);
        *dt_stable = m.dt_stable;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

// the refined mesh of a descriptor: nz_mesh, then rows -pml .. nz_mesh + pml + 1
// of z_i, z_h, dz_i, dz_h (arrays of nz_mesh + 2 pml + 2 floats, or null)
extern "C" int oracle_el2d_mesh(const owl_ssg_desc* d, int* nz_mesh, float* zi, float* zh, float* dzi, float* dzh) {
    try {
        ZMesh m = zmesh_build(*d);
        *nz_mesh = m.n;
        if (!m.refined) return 0;
        for (int j = -d->pml; j <= m.n + d->pml + 1; ++j) {
            const size_t o = (size_t)(j + d->pml);
            if (zi) zi[o] = m.zi(j);
            if (zh) zh[o] = m.zh(j);
            if (dzi) dzi[o] = m.dzi(j);
            if (dzh) dzh[o] = m.dzh(j);
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" float oracle_el2d_damp_ratio(float c11, float c13, float c33, float c55, float rho, int dir_z) {
    return damp_ratio(c11, c13, c33, c55, rho, dir_z ? 'z' : 'x');
}
