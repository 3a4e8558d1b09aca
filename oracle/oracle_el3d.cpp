// oracle_el3d.cpp -- CPU oracle for the 3D elastic (isotropic / orthorhombic)
// SSG solver.
//
// TEST INFRASTRUCTURE ONLY (see oracle_common.hpp). Restates, loop by loop:
//   model set-up (iso: Cij from vp, vs, rho; cij: the nine ORT moduli; padding,
//   pmlvp, dt_stable)            src/solver/elastic_vhtiort_3d/module_vars.f90:229-547
//   CFS-MPML damping profiles    src/solver/elastic_vhtiort_3d/module_cfspml.f90:428-625
//   update_wavefield with the inline M-PML damping
//                                src/solver/elastic_vhtiort_3d/module_wavefield.f90:52-537
//   add_source                   src/solver/elastic_vhtiort_3d/module_wavefield.f90:1095-1333
//   sampling                     src/solver/elastic_vhtiort_3d/submodule_forward_modeling.f90:82-145
//   update_wavefield_free_surface (flat free surface): zero velocities above
//   the surface, the row-1 traction condition pdzvz = -c13/c33 pdxvx - c23/c33
//   pdyvy, sigma_zz(1) = 0 and the odd stress images; on the uniform grid or
//   the depth-refined mesh (Cij interpolated linearly to the mesh planes, z
//   derivatives scaled by dz / dz_i or dz / dz_h, the z PML and the explosion
//   source on the plane's own dz_i)
//                                  module_wavefield.f90:549-1090, module_vars.f90:419-490
//   surface images before sampling submodule_forward_modeling.f90:66-82
//   sources above row 2 skipped    module_wavefield.f90:1107-1315
// plus the exact discrete adjoint and the chain rule to the model parameters.
// M-PML damping ratios of the six faces: zero -- the reference's value for the
// isotropic parameterisation (module_cfspml.f90:448-465) -- unless face arrays
// are set with oracle_el3d_set_mpml (anisotropic media: the reference's
// eigen-derivative search, module_cfspml.f90:51-421, is restated literally in
// oracle_mpml.py, which checks the library's face arrays; the tests pass those
// arrays here).
//
// Templated on T: float (forward parity), double (gradient), complex<double>
// (complex-step Jacobian-vector products).
#include <algorithm>
#include <array>
#include <cstdio>
#include <stdexcept>
#include <tuple>

#include "oracle_common.hpp"

namespace oracle {

template <typename T>
struct E3 {
    // (i, j, k), i fastest, each axis over [lo, hi]
    int i0 = 0, j0 = 0, k0 = 0, ni = 0, nj = 0, nk = 0;
    std::vector<T> a;
    void init(int lo_i, int hi_i, int lo_j, int hi_j, int lo_k, int hi_k) {
        i0 = lo_i; j0 = lo_j; k0 = lo_k;
        ni = hi_i - lo_i + 1; nj = hi_j - lo_j + 1; nk = hi_k - lo_k + 1;
        a.assign((size_t)ni * nj * nk, T(0));
    }
    inline T& operator()(int i, int j, int k) { return a[((size_t)(k - k0) * nj + (j - j0)) * ni + (i - i0)]; }
    inline const T& operator()(int i, int j, int k) const {
        return a[((size_t)(k - k0) * nj + (j - j0)) * ni + (i - i0)];
    }
};

inline int el3_nparam(int aniso) {
    return aniso == OWL_ANISO_ISO ? 3 : aniso == OWL_ANISO_THOMSEN ? 8 : (aniso == OWL_ANISO_CIJ ? 10 : -1);
}

template <typename T>
inline double el3_re(const T& v) { return std::real(v); }

// Thomsen parameters (vp, vs, eps, del, gam, the, phi, rho) to the ORT moduli:
// thomsen_to_cij3d (src/lib/module_anisotropy.f90:336-381); the tilt is
// cij_rotate_3d (:233-291) with rotation_matrix([0, -the, -phi], 'xyz') of FLIT,
// restated as R = Rz(-phi) Ry(-the), and bond_matrix (:127-170); the VHTIORT
// solver keeps the nine ORT entries of the rotated tensor (module_vars.f90:317-325).
template <typename T>
void el3_thomsen(const T* p, T* c) {
    const T vp = p[0], vs = p[1], eps = p[2], del = p[3], gam = p[4], the = p[5], phi = p[6], rho = p[7];
    const T c33 = vp * vp * rho, c44 = vs * vs * rho;
    const T c11 = c33 * (T(1) + T(2) * eps), c66 = c44 * (T(1) + T(2) * gam);
    const T c12 = c11 - T(2) * c66;
    const T tmp = T(2) * c33 * (c33 - c44) * del + (c33 - c44) * (c33 - c44);
    const T c13 = std::sqrt(el3_re(tmp) < 0 ? -tmp : tmp) - c44;
    T C[6][6] = {};
    C[0][0] = c11; C[0][1] = C[1][0] = c12; C[0][2] = C[2][0] = c13; C[1][1] = c11; C[1][2] = C[2][1] = c13;
    C[2][2] = c33; C[3][3] = c44; C[4][4] = c44; C[5][5] = c66;
    if ((el3_re(the) != 0 || el3_re(phi) != 0) && !(el3_re(eps) == 0 && el3_re(del) == 0 && el3_re(gam) == 0)) {
        const T cb = std::cos(-the), sb = std::sin(-the), cg = std::cos(-phi), sg = std::sin(-phi);
        const T Rz[3][3] = {{cg, -sg, T(0)}, {sg, cg, T(0)}, {T(0), T(0), T(1)}};
        const T Ry[3][3] = {{cb, T(0), sb}, {T(0), T(1), T(0)}, {-sb, T(0), cb}};
        T r[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                r[i][j] = T(0);
                for (int k = 0; k < 3; ++k) r[i][j] = r[i][j] + Rz[i][k] * Ry[k][j];
            }
        // Bond matrix rows as bond_matrix writes them
        const T b[6][6] = {
            {r[0][0] * r[0][0], r[0][1] * r[0][1], r[0][2] * r[0][2], T(2) * r[0][1] * r[0][2], T(2) * r[0][0] * r[0][2],
             T(2) * r[0][0] * r[0][1]},
            {r[1][0] * r[1][0], r[1][1] * r[1][1], r[1][2] * r[1][2], T(2) * r[1][1] * r[1][2], T(2) * r[1][0] * r[1][2],
             T(2) * r[1][0] * r[1][1]},
            {r[2][0] * r[2][0], r[2][1] * r[2][1], r[2][2] * r[2][2], T(2) * r[2][1] * r[2][2], T(2) * r[2][0] * r[2][2],
             T(2) * r[2][0] * r[2][1]},
            {r[1][0] * r[2][0], r[1][1] * r[2][1], r[1][2] * r[2][2], r[1][1] * r[2][2] + r[1][2] * r[2][1],
             r[1][0] * r[2][2] + r[1][2] * r[2][0], r[1][0] * r[2][1] + r[1][1] * r[2][0]},
            {r[0][0] * r[2][0], r[0][1] * r[2][1], r[0][2] * r[2][2], r[0][1] * r[2][2] + r[0][2] * r[2][1],
             r[0][0] * r[2][2] + r[0][2] * r[2][0], r[0][0] * r[2][1] + r[0][1] * r[2][0]},
            {r[0][0] * r[1][0], r[0][1] * r[1][1], r[0][2] * r[1][2], r[0][1] * r[1][2] + r[0][2] * r[1][1],
             r[0][0] * r[1][2] + r[0][2] * r[1][0], r[0][0] * r[1][1] + r[0][1] * r[1][0]}};
        T out[6][6];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) {
                T acc = T(0);
                for (int k = 0; k < 6; ++k)
                    for (int l = 0; l < 6; ++l) acc = acc + b[i][k] * C[k][l] * b[j][l];
                out[i][j] = acc;
            }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) C[i][j] = out[i][j];
    }
    c[0] = C[0][0]; c[1] = C[0][1]; c[2] = C[0][2]; c[3] = C[1][1]; c[4] = C[1][2]; c[5] = C[2][2];
    c[6] = C[3][3]; c[7] = C[4][4]; c[8] = C[5][5]; c[9] = rho;
}

// Cij of one cell, order c11 c12 c13 c22 c23 c33 c44 c55 c66 rho (module_vars.f90:278-375)
template <typename T>
void el3_cij(int aniso, const T* p, T* c) {
    if (aniso == OWL_ANISO_THOMSEN) {
        el3_thomsen(p, c);
    } else if (aniso == OWL_ANISO_ISO) {
        const T vp = p[0], vs = p[1], rho = p[2];
        const T c11 = rho * (vp * vp), c44 = rho * (vs * vs);
        const T c12 = c11 - T(2) * c44;
        c[0] = c11; c[1] = c12; c[2] = c12; c[3] = c11; c[4] = c12; c[5] = c11;
        c[6] = c44; c[7] = c44; c[8] = c44; c[9] = rho;
    } else {
        for (int q = 0; q < 10; ++q) c[q] = p[q];
    }
}

// 1D damping profile of one axis (module_cfspml.f90:517-600): d and alpha at
// integer (i) and half (h) positions over [-pml+1, n+pml]
// (zm: the per-row spacing dz_i(k) of the refined free-surface mesh,
// module_cfspml.f90:581-582 of the 3D solver)
struct Prof3 {
    Arr1<float> di, dh, ai, ah;
    void build(int n, int pml, float d, float pmlvp, float alphamax, const ZMesh* zm = nullptr) {
        di.init(-pml + 1, n + pml, 0.f); dh.init(-pml + 1, n + pml, 0.f);
        ai.init(-pml + 1, n + pml, alphamax); ah.init(-pml + 1, n + pml, alphamax);
        const float R0 = 1.0e-5f;
        for (int i = -pml + 1; i <= n + pml; ++i) {
            float nd, ndh;
            if (i <= 1) {
                nd = (float)std::abs(i - 1) * 1.0f / (float)pml;
                ndh = std::fabs((float)(i - 1) - 0.5f) * 1.0f / (float)pml;
            } else if (i >= n) {
                nd = (float)std::abs(i - n) * 1.0f / (float)pml;
                ndh = std::fabs((float)(i - n) - 0.5f) * 1.0f / (float)pml;
            } else {
                continue;
            }
            const float dd = zm && zm->refined ? zm->dzi(i) : d;
            const float c0 = std::log(1.0f / R0) * 3.0f * pmlvp / (2.0f * (float)pml * dd);
            di(i) = c0 * (nd * nd);
            dh(i) = c0 * (ndh * ndh);
            ai(i) = std::max(alphamax * (1.0f - nd), 0.25f * alphamax);
            ah(i) = std::max(alphamax * (1.0f - ndh), 0.25f * alphamax);
        }
    }
};

// damp_coef macro (module_wavefield.f90:40-43) with kappa = 1
inline void el3_ab(float dt, float d, float alpha, float& a, float& b) {
    const float adt = std::fabs(dt), bb = d + alpha;
    a = -2.0f * adt * d / (2.0f + adt * bb);
    b = (2.0f - adt * bb) / (2.0f + adt * bb);
}

template <typename T>
struct El3State {
    E3<T> f[9];   // sxx syy szz syz sxz sxy vx vy vz
    E3<T> m[18];  // memories: see the index list below
    void init(int a, int b, int c, int d, int e, int g) {
        for (auto& x : f) x.init(a, b, c, d, e, g);
        for (auto& x : m) x.init(a, b, c, d, e, g);
    }
};
enum { F_XX = 0, F_YY, F_ZZ, F_YZ, F_XZ, F_XY, F_VX, F_VY, F_VZ };
// memory order: sigma nodes dx vx, dy vy, dz vz | syz: dz vy, dy vz | sxz: dz vx, dx vz |
// sxy: dy vx, dx vy | vx: dx sxx, dy sxy, dz sxz | vy: dx sxy, dy syy, dz syz | vz: dx sxz, dy syz, dz szz
enum { M_XVX = 0, M_YVY, M_ZVZ, M_ZVY, M_YVZ, M_ZVX, M_XVZ, M_YVX, M_XVY, M_XXX, M_YXY, M_ZXZ, M_XXY, M_YYY,
       M_ZYZ, M_XXZ, M_YYZ, M_ZZZ };

// M-PML face ratios for the next oracle runs (the layout of owl_ssg_mpml_ratios);
// empty: all zero, the reference's value for the iso parameterisation
static std::vector<float> g_el3_faces;

template <typename T>
struct El3 {
    int nx, ny, nz, P, R, nt, aniso, np;
    int nzm;                  // regular (model) planes; nz: the mesh's planes
    bool fs;
    float dx, dy, dz, dt, idx, idy, idz;
    const float* c;
    ZMesh zm;
    ZLinear zl;
    E3<T> C[10];              // c11 c12 c13 c22 c23 c33 c44 c55 c66 rho, padded by pml+1, mesh planes
    E3<T> c44e, c55e, c66e;   // harmonic shear moduli at the shear-stress nodes
    std::vector<E3<T>> par;   // model parameters, regular planes
    Prof3 px, py, pz;
    int lo[3], hi[3];
    float dt_stable = 0;

    El3(const owl_ssg_desc& d, const T* const* fields) {
        nx = d.nx; ny = d.ny; nzm = d.nz; P = d.pml; R = d.fdhalf; nt = d.nt; aniso = d.aniso;
        dx = d.dx; dy = d.dy; dz = d.dz; dt = d.dt;
        fs = d.free_surface != 0;
        np = el3_nparam(aniso);
        if (np < 0) throw std::runtime_error("bad aniso");
        idx = (float)(1.0 / (double)dx); idy = (float)(1.0 / (double)dy); idz = (float)(1.0 / (double)dz);
        c = fdcoefs(R);
        zm = zmesh_build(d);
        nz = zm.n;
        if (zm.refined) zl = zlinear_build(zm, nzm, dz);
        // Cij of the regular padded planes
        E3<T> Cr[10];
        for (auto& x : Cr) x.init(-P, nx + P + 1, -P, ny + P + 1, -P, nzm + P + 1);
        par.resize(np);
        for (auto& x : par) x.init(-P, nx + P + 1, -P, ny + P + 1, -P, nzm + P + 1);
        for (int k = -P; k <= nzm + P + 1; ++k)
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i) {
                    const int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), ny),
                              kk = std::min(std::max(k, 1), nzm);
                    const size_t src = ((size_t)(ii - 1) * ny + (jj - 1)) * nzm + (kk - 1);
                    T p[10], o[10];
                    for (int q = 0; q < np; ++q) p[q] = par[q](i, j, k) = fields[q][src];
                    el3_cij(aniso, p, o);
                    for (int q = 0; q < 10; ++q) Cr[q](i, j, k) = o[q];
                }
        // the mesh's planes (map_regular_to_irregular, module_vars.f90:164-180)
        for (auto& x : C) x.init(-P, nx + P + 1, -P, ny + P + 1, -P, nz + P + 1);
        for (int k = -P; k <= nz + P + 1; ++k)
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i)
                    for (int q = 0; q < 10; ++q) {
                        if (!zm.refined) {
                            C[q](i, j, k) = Cr[q](i, j, k);
                            continue;
                        }
                        const int k0 = zl.j0(k);
                        C[q](i, j, k) = Cr[q](i, j, k0) + T(zl.w(k)) * (Cr[q](i, j, k0 + 1) - Cr[q](i, j, k0));
                    }
        c44e.init(-P + 1, nx + P, -P + 1, ny + P, -P + 1, nz + P);
        c55e.init(-P + 1, nx + P, -P + 1, ny + P, -P + 1, nz + P);
        c66e.init(-P + 1, nx + P, -P + 1, ny + P, -P + 1, nz + P);
        for (int k = -P + 1; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    const E3<T>& a44 = C[6];
                    const E3<T>& a55 = C[7];
                    const E3<T>& a66 = C[8];
                    c44e(i, j, k) = T(4) / (T(1) / a44(i, j - 1, k - 1) + T(1) / a44(i, j, k - 1) + T(1) / a44(i, j - 1, k) +
                                            T(1) / a44(i, j, k));
                    c55e(i, j, k) = T(4) / (T(1) / a55(i - 1, j, k - 1) + T(1) / a55(i, j, k - 1) + T(1) / a55(i - 1, j, k) +
                                            T(1) / a55(i, j, k));
                    c66e(i, j, k) = T(4) / (T(1) / a66(i - 1, j - 1, k) + T(1) / a66(i, j - 1, k) + T(1) / a66(i - 1, j, k) +
                                            T(1) / a66(i, j, k));
                }
        // pmlvp over the six faces of the regular model (module_vars.f90:384-406)
        // and dt_stable (:500-537; on the refined mesh the least over the
        // cells, each with its plane's smaller spacing)
        float pv = -1e30f, maxv = 0.f;
        auto rr = [&](int q, int i, int j, int k) { return (float)re(C[q](i, j, k)) / (float)re(C[9](i, j, k)); };
        for (int k = 1; k <= nzm; ++k)
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const bool face = i == 1 || i == nx || j == 1 || j == ny || k == 1 || k == nzm;
                    if (face)
                        for (int q : {0, 3, 5}) pv = std::max(pv, (float)re(Cr[q](i, j, k)) / (float)re(Cr[9](i, j, k)));
                }
        const float pmlvp = std::sqrt(pv);
        float temp = 0.f;
        for (int q = 0; q < R; ++q) temp += std::fabs(c[q]);
        if (!zm.refined) {
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i)
                        for (int q : {0, 3, 5}) maxv = std::max(maxv, std::sqrt(rr(q, i, j, k)));
            dt_stable = 1.0f / (temp * maxv * std::sqrt(1.0f / (dx * dx) + 1.0f / (dy * dy) + 1.0f / (dz * dz)));
        } else {
            float best = 3.0e38f;
            for (int k = 1; k <= nz; ++k) {
                const float h = std::min(zm.dzi(k), zm.dzh(k));
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const float mv = std::max({std::sqrt(rr(0, i, j, k)), std::sqrt(rr(3, i, j, k)),
                                                   std::sqrt(rr(5, i, j, k))});
                        best = std::min(best, 1.0f / (temp * mv * std::sqrt(1.0f / (dx * dx) + 1.0f / (dy * dy) +
                                                                             1.0f / (h * h))));
                    }
            }
            dt_stable = best;
        }
        const float alphamax = (float)(1.0 * (double)d.f0_max * 3.14159265358979323846);
        px.build(nx, P, dx, pmlvp, alphamax);
        py.build(ny, P, dy, pmlvp, alphamax);
        pz.build(nz, P, dz, pmlvp, alphamax, &zm);
        const long long fx = (long long)(ny + 2 * P) * (nz + 2 * P), fy = (long long)(nx + 2 * P) * (nz + 2 * P),
                        fz = (long long)(nx + 2 * P) * (ny + 2 * P);
        if (g_el3_faces.size() == (size_t)(2 * (fx + fy + fz))) {
            faces = g_el3_faces;
            const long long o[6] = {0, fx, 2 * fx, 2 * fx + fy, 2 * fx + 2 * fy, 2 * fx + 2 * fy + fz};
            for (int q = 0; q < 6; ++q) ofs[q] = o[q];
        }
        for (int a = 0; a < 3; ++a) lo[a] = -P - R + 1;
        hi[0] = nx + P + R; hi[1] = ny + P + R; hi[2] = nz + P + R;
    }

    // damping of the derivative along `axis` of the node (i, j, k) staggered by
    // (hx, hy, hz) (true: half position on that axis), the M-PML blocks of
    // module_wavefield.f90:101-145 (and their counterparts for the other
    // nodes): d = own profile + ratio * profile of each other axis, in the
    // reference's order, the ratio of an axis being its face's value when the
    // node lies beyond that face (index <= 0, <= 1 at a half position, or >= n + 1)
    void coef(int axis, int i, int j, int k, bool hx, bool hy, bool hz, float& a, float& b) const {
        auto beyond = [](int v, int n, bool h) { return (h ? v <= 1 : v <= 0) ? -1 : v >= n + 1 ? 1 : 0; };
        const int bx = beyond(i, nx, hx), by = beyond(j, ny, hy), bz = beyond(k, nz, hz);
        const float rx = bx < 0 ? fl(j, k) : bx > 0 ? fr(j, k) : 0.f;
        const float ry = by < 0 ? ff(i, k) : by > 0 ? fb(i, k) : 0.f;
        const float rz = bz < 0 ? ft(i, j) : bz > 0 ? fo(i, j) : 0.f;
        const float dX = hx ? px.dh(i) : px.di(i), dY = hy ? py.dh(j) : py.di(j), dZ = hz ? pz.dh(k) : pz.di(k);
        float d, al;
        if (axis == 0) { d = dX + ry * dY + rz * dZ; al = hx ? px.ah(i) : px.ai(i); }
        else if (axis == 1) { d = dY + rx * dX + rz * dZ; al = hy ? py.ah(j) : py.ai(j); }
        else { d = dZ + rx * dX + ry * dY; al = hz ? pz.ah(k) : pz.ai(k); }
        el3_ab(dt, d, al, a, b);
    }
    // face ratios over the padded ranges (-pml+1 .. n+pml): left / right (j, k),
    // front / back (i, k), top / bottom (i, j); zero unless set by oracle_el3d_set_mpml
    std::vector<float> faces;
    long long ofs[6] = {0, 0, 0, 0, 0, 0};
    float face(int f, int u, int v, int nu) const {
        if (faces.empty()) return 0.f;
        return faces[ofs[f] + (long long)(v + P - 1) * nu + (u + P - 1)];
    }
    float fl(int j, int k) const { return face(0, j, k, ny + 2 * P); }
    float fr(int j, int k) const { return face(1, j, k, ny + 2 * P); }
    float ff(int i, int k) const { return face(2, i, k, nx + 2 * P); }
    float fb(int i, int k) const { return face(3, i, k, nx + 2 * P); }
    float ft(int i, int j) const { return face(4, i, j, nx + 2 * P); }
    float fo(int i, int j) const { return face(5, i, j, nx + 2 * P); }
    // node in the PML shell: h[a] says whether the node is at a half position on axis a
    bool shell(int i, int j, int k, bool hx, bool hy, bool hz) const {
        auto out = [](int v, int n, bool h) { return h ? (v <= 1 || v >= n + 1) : (v <= 0 || v >= n + 1); };
        return out(i, nx, hx) || out(j, ny, hy) || out(k, nz, hz);
    }

    // dz scalings of the z derivatives at integer / half planes (1 on the uniform grid)
    T zsi(int k) const { return zm.refined ? T(zm.si(k)) : T(1); }
    T zsh(int k) const { return zm.refined ? T(zm.sh(k)) : T(1); }

    // stencils of pattern P (f(x+q) - f(x+1-q)) and M (f(x+q-1) - f(x-q)) along an axis
    T stP(const E3<T>& f, int i, int j, int k, int ax) const {
        T s = T(0);
        for (int q = 1; q <= R; ++q) {
            const int a = q, b = 1 - q;
            s = s + T(c[q - 1]) * (ax == 0 ? f(i + a, j, k) - f(i + b, j, k)
                                  : ax == 1 ? f(i, j + a, k) - f(i, j + b, k) : f(i, j, k + a) - f(i, j, k + b));
        }
        return s;
    }
    T stM(const E3<T>& f, int i, int j, int k, int ax) const {
        T s = T(0);
        for (int q = 1; q <= R; ++q) {
            const int a = q - 1, b = -q;
            s = s + T(c[q - 1]) * (ax == 0 ? f(i + a, j, k) - f(i + b, j, k)
                                  : ax == 1 ? f(i, j + a, k) - f(i, j + b, k) : f(i, j, k + a) - f(i, j, k + b));
        }
        return s;
    }
    // transposes: scatter e at (i,j,k) onto the field read by pattern P / M
    void scP(E3<T>& f, int i, int j, int k, int ax, T e) const {
        for (int q = 1; q <= R; ++q) {
            const int a = q, b = 1 - q;
            T v = T(c[q - 1]) * e;
            if (ax == 0) { f(i + a, j, k) = f(i + a, j, k) + v; f(i + b, j, k) = f(i + b, j, k) - v; }
            else if (ax == 1) { f(i, j + a, k) = f(i, j + a, k) + v; f(i, j + b, k) = f(i, j + b, k) - v; }
            else { f(i, j, k + a) = f(i, j, k + a) + v; f(i, j, k + b) = f(i, j, k + b) - v; }
        }
    }
    void scM(E3<T>& f, int i, int j, int k, int ax, T e) const {
        for (int q = 1; q <= R; ++q) {
            const int a = q - 1, b = -q;
            T v = T(c[q - 1]) * e;
            if (ax == 0) { f(i + a, j, k) = f(i + a, j, k) + v; f(i + b, j, k) = f(i + b, j, k) - v; }
            else if (ax == 1) { f(i, j + a, k) = f(i, j + a, k) + v; f(i, j + b, k) = f(i, j + b, k) - v; }
            else { f(i, j, k + a) = f(i, j, k + a) + v; f(i, j, k + b) = f(i, j, k + b) - v; }
        }
    }
    // forward PML of one derivative value: psi = a D + b psi; D' = D + psi
    static T pml_f(T D, float a, float b, T& psi) {
        psi = T(a) * D + T(b) * psi;
        return D + psi;
    }
    static T pml_e(T q, float a, float b, T& psih) {
        T u = q + psih;
        psih = T(b) * u;
        return q + T(a) * u;
    }

    // first z index a field is updated at: with a free surface, the nodes at
    // integer depth from row 1, those at half depth (syz, sxz, vz) from row 2
    int kmin(int f) const {
        if (!fs) return -P + 1;
        return (f == F_YZ || f == F_XZ || f == F_VZ) ? 2 : 1;
    }
    template <class Fn>
    void each(Fn fn, int k0) const {
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = k0; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) fn(i, j, k);
    }

    // forward update; S (optional, 9 planes): Dx', Dy', Dz' at sigma nodes, the
    // shear sums at syz / sxz / sxy, the velocity sums at vx / vy / vz
    void update(El3State<T>& s, E3<T>* S) const {
        if (fs) {
            // particle velocities above the free surface are zero (module_wavefield.f90:582-593)
            for (int q = 1; q <= R; ++q)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        s.f[F_VX](i, j, 1 - q) = T(0);
                        s.f[F_VY](i, j, 1 - q) = T(0);
                        s.f[F_VZ](i, j, 2 - q) = T(0);
                    }
        }
        // normal stresses (module_wavefield.f90:93-163; free surface :602-711)
        each([&](int i, int j, int k) {
            const float fdt = dt;
            T dX = T(idx) * stP(s.f[F_VX], i, j, k, 0), dY = T(idy) * stP(s.f[F_VY], i, j, k, 1), dZ;
            if (fs && k == 1) {
                if (i <= 0 || i >= nx + 1 || j <= 0 || j >= ny + 1) {
                    float ca, cb;
                    coef(0, i, j, k, false, false, false, ca, cb); dX = pml_f(dX, ca, cb, s.m[M_XVX](i, j, k));
                    coef(1, i, j, k, false, false, false, ca, cb); dY = pml_f(dY, ca, cb, s.m[M_YVY](i, j, k));
                }
                dZ = -(C[2](i, j, k) / C[5](i, j, k)) * dX - (C[4](i, j, k) / C[5](i, j, k)) * dY;
            } else {
                dZ = T(idz) * stP(s.f[F_VZ], i, j, k, 2) * zsi(k);
                if (shell(i, j, k, false, false, false)) {
                    float ca, cb;
                    coef(0, i, j, k, false, false, false, ca, cb); dX = pml_f(dX, ca, cb, s.m[M_XVX](i, j, k));
                    coef(1, i, j, k, false, false, false, ca, cb); dY = pml_f(dY, ca, cb, s.m[M_YVY](i, j, k));
                    coef(2, i, j, k, false, false, false, ca, cb); dZ = pml_f(dZ, ca, cb, s.m[M_ZVZ](i, j, k));
                }
            }
            s.f[F_XX](i, j, k) = s.f[F_XX](i, j, k) + T(fdt) * (C[0](i, j, k) * dX + C[1](i, j, k) * dY + C[2](i, j, k) * dZ);
            s.f[F_YY](i, j, k) = s.f[F_YY](i, j, k) + T(fdt) * (C[1](i, j, k) * dX + C[3](i, j, k) * dY + C[4](i, j, k) * dZ);
            s.f[F_ZZ](i, j, k) = s.f[F_ZZ](i, j, k) + T(fdt) * (C[2](i, j, k) * dX + C[4](i, j, k) * dY + C[5](i, j, k) * dZ);
            if (S) { S[0](i, j, k) = dX; S[1](i, j, k) = dY; S[2](i, j, k) = dZ; }
        }, kmin(F_XX));
        // syz at (i, j-1/2, k-1/2) (:171-221)
        each([&](int i, int n, int p) {
            T dzvy = T(idz) * stM(s.f[F_VY], i, n, p, 2) * zsh(p), dyvz = T(idy) * stM(s.f[F_VZ], i, n, p, 1);
            if (shell(i, n, p, false, true, true)) {
                float ca, cb;
                coef(1, i, n, p, false, true, true, ca, cb); dyvz = pml_f(dyvz, ca, cb, s.m[M_YVZ](i, n, p));
                coef(2, i, n, p, false, true, true, ca, cb); dzvy = pml_f(dzvy, ca, cb, s.m[M_ZVY](i, n, p));
            }
            s.f[F_YZ](i, n, p) = s.f[F_YZ](i, n, p) + T(dt) * c44e(i, n, p) * (dzvy + dyvz);
            if (S) S[3](i, n, p) = dzvy + dyvz;
        }, kmin(F_YZ));
        // sxz at (i-1/2, j, k-1/2) (:228-278)
        each([&](int m, int j, int p) {
            T dzvx = T(idz) * stM(s.f[F_VX], m, j, p, 2) * zsh(p), dxvz = T(idx) * stM(s.f[F_VZ], m, j, p, 0);
            if (shell(m, j, p, true, false, true)) {
                float ca, cb;
                coef(0, m, j, p, true, false, true, ca, cb); dxvz = pml_f(dxvz, ca, cb, s.m[M_XVZ](m, j, p));
                coef(2, m, j, p, true, false, true, ca, cb); dzvx = pml_f(dzvx, ca, cb, s.m[M_ZVX](m, j, p));
            }
            s.f[F_XZ](m, j, p) = s.f[F_XZ](m, j, p) + T(dt) * c55e(m, j, p) * (dzvx + dxvz);
            if (S) S[4](m, j, p) = dzvx + dxvz;
        }, kmin(F_XZ));
        // sxy at (i-1/2, j-1/2, k) (:285-335)
        each([&](int m, int n, int k) {
            T dyvx = T(idy) * stM(s.f[F_VX], m, n, k, 1), dxvy = T(idx) * stM(s.f[F_VY], m, n, k, 0);
            if (shell(m, n, k, true, true, false)) {
                float ca, cb;
                coef(0, m, n, k, true, true, false, ca, cb); dxvy = pml_f(dxvy, ca, cb, s.m[M_XVY](m, n, k));
                coef(1, m, n, k, true, true, false, ca, cb); dyvx = pml_f(dyvx, ca, cb, s.m[M_YVX](m, n, k));
            }
            s.f[F_XY](m, n, k) = s.f[F_XY](m, n, k) + T(dt) * c66e(m, n, k) * (dyvx + dxvy);
            if (S) S[5](m, n, k) = dyvx + dxvy;
        }, kmin(F_XY));
        if (fs) {
            // stress images (module_wavefield.f90:871-903): odd about row 1 for the
            // integer-depth stresses, sigma_zz(1) = 0, odd about row 3/2 for syz, sxz
            for (int q = 1; q <= R; ++q)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        s.f[F_ZZ](i, j, 1 - q) = -s.f[F_ZZ](i, j, 1 + q);
                        s.f[F_ZZ](i, j, 1) = T(0);
                        s.f[F_XX](i, j, 1 - q) = -s.f[F_XX](i, j, 1 + q);
                        s.f[F_YY](i, j, 1 - q) = -s.f[F_YY](i, j, 1 + q);
                        s.f[F_XY](i, j, 1 - q) = -s.f[F_XY](i, j, 1 + q);
                        s.f[F_YZ](i, j, 2 - q) = -s.f[F_YZ](i, j, 1 + q);
                        s.f[F_XZ](i, j, 2 - q) = -s.f[F_XZ](i, j, 1 + q);
                    }
        }
        // vx at (i-1/2, j, k) (:350-410)
        each([&](int m, int j, int k) {
            T hx = T(idx) * stM(s.f[F_XX], m, j, k, 0), hy = T(idy) * stP(s.f[F_XY], m, j, k, 1),
              hz = T(idz) * stP(s.f[F_XZ], m, j, k, 2) * zsi(k);
            if (shell(m, j, k, true, false, false)) {
                float ca, cb;
                coef(0, m, j, k, true, false, false, ca, cb); hx = pml_f(hx, ca, cb, s.m[M_XXX](m, j, k));
                coef(1, m, j, k, true, false, false, ca, cb); hy = pml_f(hy, ca, cb, s.m[M_YXY](m, j, k));
                coef(2, m, j, k, true, false, false, ca, cb); hz = pml_f(hz, ca, cb, s.m[M_ZXZ](m, j, k));
            }
            const T re = T(0.5f) * (C[9](m - 1, j, k) + C[9](m, j, k));
            s.f[F_VX](m, j, k) = s.f[F_VX](m, j, k) + T(dt) / re * (hx + hy + hz);
            if (S) S[6](m, j, k) = hx + hy + hz;
        }, kmin(F_VX));
        // vy at (i, j-1/2, k) (:416-476)
        each([&](int i, int n, int k) {
            T hx = T(idx) * stP(s.f[F_XY], i, n, k, 0), hy = T(idy) * stM(s.f[F_YY], i, n, k, 1),
              hz = T(idz) * stP(s.f[F_YZ], i, n, k, 2) * zsi(k);
            if (shell(i, n, k, false, true, false)) {
                float ca, cb;
                coef(0, i, n, k, false, true, false, ca, cb); hx = pml_f(hx, ca, cb, s.m[M_XXY](i, n, k));
                coef(1, i, n, k, false, true, false, ca, cb); hy = pml_f(hy, ca, cb, s.m[M_YYY](i, n, k));
                coef(2, i, n, k, false, true, false, ca, cb); hz = pml_f(hz, ca, cb, s.m[M_ZYZ](i, n, k));
            }
            const T re = T(0.5f) * (C[9](i, n - 1, k) + C[9](i, n, k));
            s.f[F_VY](i, n, k) = s.f[F_VY](i, n, k) + T(dt) / re * (hx + hy + hz);
            if (S) S[7](i, n, k) = hx + hy + hz;
        }, kmin(F_VY));
        // vz at (i, j, k-1/2) (:482-542)
        each([&](int i, int j, int p) {
            T hx = T(idx) * stP(s.f[F_XZ], i, j, p, 0), hy = T(idy) * stP(s.f[F_YZ], i, j, p, 1),
              hz = T(idz) * stM(s.f[F_ZZ], i, j, p, 2) * zsh(p);
            if (shell(i, j, p, false, false, true)) {
                float ca, cb;
                coef(0, i, j, p, false, false, true, ca, cb); hx = pml_f(hx, ca, cb, s.m[M_XXZ](i, j, p));
                coef(1, i, j, p, false, false, true, ca, cb); hy = pml_f(hy, ca, cb, s.m[M_YYZ](i, j, p));
                coef(2, i, j, p, false, false, true, ca, cb); hz = pml_f(hz, ca, cb, s.m[M_ZZZ](i, j, p));
            }
            const T re = T(0.5f) * (C[9](i, j, p - 1) + C[9](i, j, p));
            s.f[F_VZ](i, j, p) = s.f[F_VZ](i, j, p) + T(dt) / re * (hx + hy + hz);
            if (S) S[8](i, j, p) = hx + hy + hz;
        }, kmin(F_VZ));
    }

    // source taps of one source: (field, i, j, k, weight without the STF amplitude)
    void src_taps(const owl_source& q, std::vector<std::tuple<int, int, int, int, T>>& out, int& rho_cell_used) const {
        out.clear();
        rho_cell_used = 0;
        const float* ix = q.interp_ix; const float* iy = q.interp_iy; const float* iz = q.interp_iz;
        const float* hx = q.interp_hx; const float* hy = q.interp_hy; const float* hz = q.interp_hz;
        for (int irz = -4; irz <= 4; ++irz)
            for (int iry = -4; iry <= 4; ++iry)
                for (int irx = -4; irx <= 4; ++irx) {
                    const int a = irx + 4, b = iry + 4, cc = irz + 4;
                    if (q.mechanism == OWL_SRC_FORCE) {
                        const T r = C[9](q.gx, q.gy, q.gz);
                        rho_cell_used = 1;
                        out.emplace_back(F_VX, q.hx + irx, q.gy + iry, q.gz + irz,
                                         T(std::sin(q.polar) * std::cos(q.azimuth)) / r * T(hx[a]) * T(iy[b]) * T(iz[cc]));
                        out.emplace_back(F_VY, q.gx + irx, q.hy + iry, q.gz + irz,
                                         T(std::sin(q.polar) * std::sin(q.azimuth)) / r * T(ix[a]) * T(hy[b]) * T(iz[cc]));
                        out.emplace_back(F_VZ, q.gx + irx, q.gy + iry, q.hz + irz,
                                         T(std::cos(q.polar)) / r * T(ix[a]) * T(iy[b]) * T(hz[cc]));
                    } else {
                        const bool mt = q.mechanism == OWL_SRC_MT;
                        // dz_s: the local spacing dz_i(gz) on the refined mesh (module_wavefield.f90:1107-1111)
                        const T inv = T(1) / (T(dx) * T(dy) * T(zm.refined ? zm.dzi(q.gz) : dz));
                        const T w = T(ix[a]) * T(iy[b]) * T(iz[cc]);
                        out.emplace_back(F_XX, q.gx + irx, q.gy + iry, q.gz + irz, -inv * T(mt ? q.mt[0] : 1.f) * w);
                        out.emplace_back(F_YY, q.gx + irx, q.gy + iry, q.gz + irz, -inv * T(mt ? q.mt[1] : 1.f) * w);
                        out.emplace_back(F_ZZ, q.gx + irx, q.gy + iry, q.gz + irz, -inv * T(mt ? q.mt[2] : 1.f) * w);
                        if (mt) {
                            out.emplace_back(F_XY, q.hx + irx, q.hy + iry, q.gz + irz, -inv * T(q.mt[3]) * T(hx[a]) * T(hy[b]) * T(iz[cc]));
                            out.emplace_back(F_XZ, q.hx + irx, q.gy + iry, q.hz + irz, -inv * T(q.mt[4]) * T(hx[a]) * T(iy[b]) * T(hz[cc]));
                            out.emplace_back(F_YZ, q.gx + irx, q.hy + iry, q.hz + irz, -inv * T(q.mt[5]) * T(ix[a]) * T(hy[b]) * T(hz[cc]));
                        }
                    }
                }
        // with a free surface, no source tap above row 2 (module_wavefield.f90:1147-1315)
        if (fs)
            out.erase(std::remove_if(out.begin(), out.end(), [](const std::tuple<int, int, int, int, T>& tp) {
                          return std::get<3>(tp) < 2;
                      }), out.end());
    }

    // surface images of the velocities before sampling (submodule_forward_modeling.f90:66-82),
    // over the interpolation half-width nkw = 4 (module_source_receiver.f90:146)
    void images(El3State<T>& s) const {
        for (int q = 1; q <= 4; ++q)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    s.f[F_VX](i, j, 1 - q) = s.f[F_VX](i, j, 1 + q);
                    s.f[F_VY](i, j, 1 - q) = s.f[F_VY](i, j, 1 + q);
                    s.f[F_VZ](i, j, 2 - q) = s.f[F_VZ](i, j, 1 + q);
                }
    }

    void add_source(int t, const owl_shot& sh, El3State<T>& s) const {
        std::vector<std::tuple<int, int, int, int, T>> taps;
        int ru;
        for (int kk = 0; kk < sh.nsrc; ++kk) {
            const owl_source& q = sh.src[kk];
            if (t < q.nbeg || t > q.nbeg + q.nt_stf - 1) continue;
            const T amp = T(q.stf[t - q.nbeg]) * T(q.amp) * T(dt);
            src_taps(q, taps, ru);
            for (auto& tp : taps) {
                E3<T>& f = s.f[std::get<0>(tp)];
                T& v = f(std::get<1>(tp), std::get<2>(tp), std::get<3>(tp));
                v = v + amp * std::get<4>(tp);
            }
        }
    }

    // sampling of step t: out[(comp * nrec + r) * nt + t - 1], comps vx, vy, vz
    void sample(int t, const owl_shot& sh, const El3State<T>& s, T* out) const {
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T a0 = T(0), a1 = T(0), a2 = T(0);
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx) {
                        const int a = irx + 4, b = iry + 4, cc = irz + 4;
                        a0 = a0 + s.f[F_VX](q.hx + irx, q.gy + iry, q.gz + irz) * T(q.interp_hx[a]) * T(q.interp_iy[b]) * T(q.interp_iz[cc]) * T(q.weight);
                        a1 = a1 + s.f[F_VY](q.gx + irx, q.hy + iry, q.gz + irz) * T(q.interp_ix[a]) * T(q.interp_hy[b]) * T(q.interp_iz[cc]) * T(q.weight);
                        a2 = a2 + s.f[F_VZ](q.gx + irx, q.gy + iry, q.hz + irz) * T(q.interp_ix[a]) * T(q.interp_iy[b]) * T(q.interp_hz[cc]) * T(q.weight);
                    }
            out[(size_t)r * nt + (t - 1)] = a0;
            out[((size_t)sh.nrec + r) * nt + (t - 1)] = a1;
            out[((size_t)2 * sh.nrec + r) * nt + (t - 1)] = a2;
        }
    }

    void new_state(El3State<T>& s) const { s.init(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]); }

    void forward_shot(const owl_shot& sh, T* seis, std::vector<El3State<T>>* ckpt, int k) const {
        El3State<T> s;
        new_state(s);
        std::fill(seis, seis + (size_t)3 * sh.nrec * nt, T(0));
        for (int t = 1; t <= nt; ++t) {
            if (ckpt && (t - 1) % k == 0) ckpt->push_back(s);
            if (fs) images(s);
            sample(t, sh, s, seis);
            update(s, nullptr);
            add_source(t, sh, s);
        }
    }

    // ---------------- exact adjoint ----------------
    struct Grad {
        E3<T> g[10];  // d J / d (c11 c12 c13 c22 c23 c33 c44 c55 c66 rho), padded grid
        std::vector<E3<T>> gpar;
    };

    void adjoint_step(int t, const owl_shot& sh, El3State<T>& a, E3<T>* S, const T* res, Grad& g, T* stf_grad) const {
        // add_source(t): STF and force-point rho gradients
        std::vector<std::tuple<int, int, int, int, T>> taps;
        int ru;
        for (int kk = 0; kk < sh.nsrc; ++kk) {
            const owl_source& q = sh.src[kk];
            if (t < q.nbeg || t > q.nbeg + q.nt_stf - 1) continue;
            const T amp = T(q.stf[t - q.nbeg]) * T(q.amp) * T(dt);
            src_taps(q, taps, ru);
            T acc = T(0);
            for (auto& tp : taps)
                acc = acc + a.f[std::get<0>(tp)](std::get<1>(tp), std::get<2>(tp), std::get<3>(tp)) * std::get<4>(tp);
            if (stf_grad) stf_grad[(size_t)kk * nt + (t - 1)] = stf_grad[(size_t)kk * nt + (t - 1)] + acc * T(q.amp) * T(dt);
            if (ru) {
                // force weights carry 1 / rho(gx, gy, gz)
                const T r = C[9](q.gx, q.gy, q.gz);
                g.g[9](q.gx, q.gy, q.gz) = g.g[9](q.gx, q.gy, q.gz) - amp * acc / r;
            }
        }
        // reverse vz, vy, vx (independent of each other)
        auto vrev = [&](int fv, int i, int j, int k, int di, int dj, int dk, int si, E3<T>* Sv, bool hxh, bool hyh, bool hzh,
                        int mx, int my, int mz) {
            const T rhoe = T(0.5f) * (C[9](i - di, j - dj, k - dk) + C[9](i, j, k));
            const T vh = a.f[fv](i, j, k);
            const T gr = -vh * Sv[si](i, j, k) * T(dt) * T(0.5f) / (rhoe * rhoe);
            g.g[9](i - di, j - dj, k - dk) = g.g[9](i - di, j - dj, k - dk) + gr;
            g.g[9](i, j, k) = g.g[9](i, j, k) + gr;
            const T q = T(dt) / rhoe * vh;
            T ex = q, ey = q, ez = q;
            if (shell(i, j, k, hxh, hyh, hzh)) {
                float ca, cb;
                coef(0, i, j, k, hxh, hyh, hzh, ca, cb); ex = pml_e(q, ca, cb, a.m[mx](i, j, k));
                coef(1, i, j, k, hxh, hyh, hzh, ca, cb); ey = pml_e(q, ca, cb, a.m[my](i, j, k));
                coef(2, i, j, k, hxh, hyh, hzh, ca, cb); ez = pml_e(q, ca, cb, a.m[mz](i, j, k));
            }
            return std::array<T, 3>{T(idx) * ex, T(idy) * ey, T(idz) * (hzh ? zsh(k) : zsi(k)) * ez};
        };
        for (int k = kmin(F_VX); k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    std::array<T, 3> e;
                    if (k >= kmin(F_VZ)) {
                        // vz (i, j, k-1/2): reads sxz (P,x), syz (P,y), szz (M,z)
                        e = vrev(F_VZ, i, j, k, 0, 0, 1, 8, S, false, false, true, M_XXZ, M_YYZ, M_ZZZ);
                        scP(a.f[F_XZ], i, j, k, 0, e[0]);
                        scP(a.f[F_YZ], i, j, k, 1, e[1]);
                        scM(a.f[F_ZZ], i, j, k, 2, e[2]);
                    }
                    // vy (i, j-1/2, k): sxy (P,x), syy (M,y), syz (P,z)
                    e = vrev(F_VY, i, j, k, 0, 1, 0, 7, S, false, true, false, M_XXY, M_YYY, M_ZYZ);
                    scP(a.f[F_XY], i, j, k, 0, e[0]);
                    scM(a.f[F_YY], i, j, k, 1, e[1]);
                    scP(a.f[F_YZ], i, j, k, 2, e[2]);
                    // vx (i-1/2, j, k): sxx (M,x), sxy (P,y), sxz (P,z)
                    e = vrev(F_VX, i, j, k, 1, 0, 0, 6, S, true, false, false, M_XXX, M_YXY, M_ZXZ);
                    scM(a.f[F_XX], i, j, k, 0, e[0]);
                    scP(a.f[F_XY], i, j, k, 1, e[1]);
                    scP(a.f[F_XZ], i, j, k, 2, e[2]);
                }
        if (fs) {
            // reverse the stress images and sigma_zz(1) = 0: an image's adjoint
            // folds onto the row it copies, with the image's sign
            for (int q = R; q >= 1; --q)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        for (int f : {F_YZ, F_XZ}) {
                            a.f[f](i, j, 1 + q) = a.f[f](i, j, 1 + q) - a.f[f](i, j, 2 - q);
                            a.f[f](i, j, 2 - q) = T(0);
                        }
                        a.f[F_ZZ](i, j, 1) = T(0);
                        for (int f : {F_ZZ, F_XX, F_YY, F_XY}) {
                            a.f[f](i, j, 1 + q) = a.f[f](i, j, 1 + q) - a.f[f](i, j, 1 - q);
                            a.f[f](i, j, 1 - q) = T(0);
                        }
                    }
        }
        // reverse the shear updates; c_e = 4 / sum(1 / c) over the 4 cells
        auto shear = [&](int fs, E3<T>& ce, int cq, int i, int j, int k, int si, const int (&cells)[4][3], int ax1, int ax2,
                         bool h1, bool h2, int m1, int m2, int fa, int fb) {
            // sigma = sigma + dt ce (D_ax1 fa + D_ax2 fb): D along ax1 of field fa, along ax2 of field fb
            const T sh_ = a.f[fs](i, j, k);
            const T gce = T(dt) * sh_ * S[si](i, j, k);
            if (re(ce(i, j, k)) != 0)
                for (int q = 0; q < 4; ++q) {
                    const T cc = C[cq](cells[q][0], cells[q][1], cells[q][2]);
                    g.g[cq](cells[q][0], cells[q][1], cells[q][2]) =
                        g.g[cq](cells[q][0], cells[q][1], cells[q][2]) + gce * ce(i, j, k) * ce(i, j, k) / (T(4) * cc * cc);
                }
            const T q = T(dt) * ce(i, j, k) * sh_;
            T e1 = q, e2 = q;
            const int pos[3] = {i, j, k};
            bool hh[3] = {false, false, false};
            hh[ax1] = h1; hh[ax2] = h2;
            if (shell(i, j, k, hh[0], hh[1], hh[2])) {
                float ca, cb;
                coef(ax1, i, j, k, hh[0], hh[1], hh[2], ca, cb); e1 = pml_e(q, ca, cb, a.m[m1](i, j, k));
                coef(ax2, i, j, k, hh[0], hh[1], hh[2], ca, cb); e2 = pml_e(q, ca, cb, a.m[m2](i, j, k));
            }
            // (the z derivatives of the shear nodes sit at half planes)
            const T id[3] = {T(idx), T(idy), T(idz) * zsh(k)};
            scM(a.f[fa], i, j, k, ax1, id[ax1] * e1);
            scM(a.f[fb], i, j, k, ax2, id[ax2] * e2);
        };
        for (int k = kmin(F_XY); k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    if (k >= kmin(F_YZ)) {
                    // syz (i, n, p): dt c44e (Dz vy + Dy vz)
                    { const int cl[4][3] = {{i, j - 1, k - 1}, {i, j, k - 1}, {i, j - 1, k}, {i, j, k}};
                      shear(F_YZ, const_cast<E3<T>&>(c44e), 6, i, j, k, 3, cl, 2, 1, true, true, M_ZVY, M_YVZ, F_VY, F_VZ); }
                    // sxz (m, j, p): dt c55e (Dz vx + Dx vz)
                    { const int cl[4][3] = {{i - 1, j, k - 1}, {i, j, k - 1}, {i - 1, j, k}, {i, j, k}};
                      shear(F_XZ, const_cast<E3<T>&>(c55e), 7, i, j, k, 4, cl, 2, 0, true, true, M_ZVX, M_XVZ, F_VX, F_VZ); }
                    }
                    // sxy (m, n, k): dt c66e (Dy vx + Dx vy)
                    { const int cl[4][3] = {{i - 1, j - 1, k}, {i, j - 1, k}, {i - 1, j, k}, {i, j, k}};
                      shear(F_XY, const_cast<E3<T>&>(c66e), 8, i, j, k, 5, cl, 1, 0, true, true, M_YVX, M_XVY, F_VX, F_VY); }
                }
        // reverse the normal-stress update
        for (int k = kmin(F_XX); k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    const T xh = a.f[F_XX](i, j, k), yh = a.f[F_YY](i, j, k), zh = a.f[F_ZZ](i, j, k);
                    const T dX = S[0](i, j, k), dY = S[1](i, j, k), dZ = S[2](i, j, k);
                    const T tt = T(dt);
                    if (fs && k == 1) {
                        // row 1: dZ = -(c13 dX + c23 dY) / c33 and sigma_zz(1) overwritten by 0
                        const T r13 = C[2](i, j, k) / C[5](i, j, k), r23 = C[4](i, j, k) / C[5](i, j, k);
                        g.g[0](i, j, k) = g.g[0](i, j, k) + tt * xh * dX;
                        g.g[1](i, j, k) = g.g[1](i, j, k) + tt * (xh * dY + yh * dX);
                        g.g[2](i, j, k) = g.g[2](i, j, k) + tt * (xh * (dZ - r13 * dX) - yh * r23 * dX);
                        g.g[3](i, j, k) = g.g[3](i, j, k) + tt * yh * dY;
                        g.g[4](i, j, k) = g.g[4](i, j, k) + tt * (yh * (dZ - r23 * dY) - xh * r13 * dY);
                        g.g[5](i, j, k) = g.g[5](i, j, k) - tt * (xh * r13 + yh * r23) * dZ;
                        const T w = tt * (C[2](i, j, k) * xh + C[4](i, j, k) * yh);
                        T qx = tt * (C[0](i, j, k) * xh + C[1](i, j, k) * yh) - r13 * w;
                        T qy = tt * (C[1](i, j, k) * xh + C[3](i, j, k) * yh) - r23 * w;
                        if (i <= 0 || i >= nx + 1 || j <= 0 || j >= ny + 1) {
                            float ca, cb;
                            coef(0, i, j, k, false, false, false, ca, cb); qx = pml_e(qx, ca, cb, a.m[M_XVX](i, j, k));
                            coef(1, i, j, k, false, false, false, ca, cb); qy = pml_e(qy, ca, cb, a.m[M_YVY](i, j, k));
                        }
                        scP(a.f[F_VX], i, j, k, 0, T(idx) * qx);
                        scP(a.f[F_VY], i, j, k, 1, T(idy) * qy);
                        continue;
                    }
                    g.g[0](i, j, k) = g.g[0](i, j, k) + tt * xh * dX;
                    g.g[1](i, j, k) = g.g[1](i, j, k) + tt * (xh * dY + yh * dX);
                    g.g[2](i, j, k) = g.g[2](i, j, k) + tt * (xh * dZ + zh * dX);
                    g.g[3](i, j, k) = g.g[3](i, j, k) + tt * yh * dY;
                    g.g[4](i, j, k) = g.g[4](i, j, k) + tt * (yh * dZ + zh * dY);
                    g.g[5](i, j, k) = g.g[5](i, j, k) + tt * zh * dZ;
                    T qx = tt * (C[0](i, j, k) * xh + C[1](i, j, k) * yh + C[2](i, j, k) * zh);
                    T qy = tt * (C[1](i, j, k) * xh + C[3](i, j, k) * yh + C[4](i, j, k) * zh);
                    T qz = tt * (C[2](i, j, k) * xh + C[4](i, j, k) * yh + C[5](i, j, k) * zh);
                    if (shell(i, j, k, false, false, false)) {
                        float ca, cb;
                        coef(0, i, j, k, false, false, false, ca, cb); qx = pml_e(qx, ca, cb, a.m[M_XVX](i, j, k));
                        coef(1, i, j, k, false, false, false, ca, cb); qy = pml_e(qy, ca, cb, a.m[M_YVY](i, j, k));
                        coef(2, i, j, k, false, false, false, ca, cb); qz = pml_e(qz, ca, cb, a.m[M_ZVZ](i, j, k));
                    }
                    scP(a.f[F_VX], i, j, k, 0, T(idx) * qx);
                    scP(a.f[F_VY], i, j, k, 1, T(idy) * qy);
                    scP(a.f[F_VZ], i, j, k, 2, T(idz) * zsi(k) * qz);
                }
        clear_outside(a);
        // sampling of step t
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            const T r0 = res[(size_t)r * nt + (t - 1)], r1 = res[((size_t)sh.nrec + r) * nt + (t - 1)],
                    r2 = res[((size_t)2 * sh.nrec + r) * nt + (t - 1)];
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx) {
                        const int a0 = irx + 4, b0 = iry + 4, c0 = irz + 4;
                        T& v0 = a.f[F_VX](q.hx + irx, q.gy + iry, q.gz + irz);
                        v0 = v0 + r0 * T(q.interp_hx[a0]) * T(q.interp_iy[b0]) * T(q.interp_iz[c0]) * T(q.weight);
                        T& v1 = a.f[F_VY](q.gx + irx, q.hy + iry, q.gz + irz);
                        v1 = v1 + r1 * T(q.interp_ix[a0]) * T(q.interp_hy[b0]) * T(q.interp_iz[c0]) * T(q.weight);
                        T& v2 = a.f[F_VZ](q.gx + irx, q.gy + iry, q.hz + irz);
                        v2 = v2 + r2 * T(q.interp_ix[a0]) * T(q.interp_iy[b0]) * T(q.interp_hz[c0]) * T(q.weight);
                    }
        }
        if (fs) {
            // the sampled images fold onto the rows they copy
            for (int q = 4; q >= 1; --q)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        a.f[F_VX](i, j, 1 + q) = a.f[F_VX](i, j, 1 + q) + a.f[F_VX](i, j, 1 - q);
                        a.f[F_VX](i, j, 1 - q) = T(0);
                        a.f[F_VY](i, j, 1 + q) = a.f[F_VY](i, j, 1 + q) + a.f[F_VY](i, j, 1 - q);
                        a.f[F_VY](i, j, 1 - q) = T(0);
                        a.f[F_VZ](i, j, 1 + q) = a.f[F_VZ](i, j, 1 + q) + a.f[F_VZ](i, j, 2 - q);
                        a.f[F_VZ](i, j, 2 - q) = T(0);
                    }
        }
        clear_outside(a);
    }

    void clear_outside(El3State<T>& a) const {
        for (int q = 0; q < 9; ++q) {
            E3<T>& f = a.f[q];
            for (int k = lo[2]; k <= hi[2]; ++k)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        const bool in = i >= -P + 1 && i <= nx + P && j >= -P + 1 && j <= ny + P && k >= kmin(q) &&
                                        k <= nz + P;
                        if (!in) f(i, j, k) = T(0);
                    }
        }
    }

    void adjoint_shot(const owl_shot& sh, const T* res, int k, Grad& g, T* stf_grad) const {
        std::vector<El3State<T>> ck;
        std::vector<T> dummy((size_t)3 * sh.nrec * nt);
        forward_shot(sh, dummy.data(), &ck, k);
        El3State<T> a;
        new_state(a);
        std::vector<std::array<E3<T>, 9>> Sbuf((size_t)k);
        for (auto& s9 : Sbuf)
            for (auto& arr : s9) arr.init(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
        for (int sg = (int)ck.size() - 1; sg >= 0; --sg) {
            const int n0 = sg * k, n1 = std::min(nt, n0 + k);
            El3State<T> s = ck[sg];
            for (int t = n0 + 1; t <= n1; ++t) {
                if (fs) images(s);
                update(s, Sbuf[t - n0 - 1].data());
                add_source(t, sh, s);
            }
            for (int t = n1; t >= n0 + 1; --t) adjoint_step(t, sh, a, Sbuf[t - n0 - 1].data(), res, g, stf_grad);
        }
    }

    // (on the refined mesh first the transpose of the depth interpolation, from
    // the mesh planes to the regular planes)
    void chain(Grad& g) const {
        typedef std::complex<double> Cx;
        std::vector<E3<T>> rg;
        const E3<T>* src[10];
        for (int r = 0; r < 10; ++r) src[r] = &g.g[r];
        if (zm.refined) {
            rg.resize(10);
            for (auto& x : rg) x.init(-P, nx + P + 1, -P, ny + P + 1, -P, nzm + P + 1);
            for (int f = -P; f <= nz + P + 1; ++f) {
                const int k0 = zl.j0(f);
                const T w = T(zl.w(f));
                for (int r = 0; r < 10; ++r)
                    for (int j = -P; j <= ny + P + 1; ++j)
                        for (int i = -P; i <= nx + P + 1; ++i) {
                            const T v = g.g[r](i, j, f);
                            rg[r](i, j, k0) = rg[r](i, j, k0) + (T(1) - w) * v;
                            rg[r](i, j, k0 + 1) = rg[r](i, j, k0 + 1) + w * v;
                        }
            }
            for (int r = 0; r < 10; ++r) src[r] = &rg[r];
        }
        g.gpar.assign(np, E3<T>());
        for (auto& x : g.gpar) x.init(-P, nx + P + 1, -P, ny + P + 1, -P, nzm + P + 1);
        for (int k = -P; k <= nzm + P + 1; ++k)
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i)
                    for (int q = 0; q < np; ++q) {
                        Cx p[10], o[10];
                        for (int r = 0; r < np; ++r) p[r] = Cx(re(par[r](i, j, k)), r == q ? 1e-30 : 0.0);
                        el3_cij(aniso, p, o);
                        T acc = T(0);
                        for (int r = 0; r < 10; ++r) acc = acc + (*src[r])(i, j, k) * T(o[r].imag() / 1e-30);
                        g.gpar[q](i, j, k) = acc;
                    }
    }

    void fold(const E3<T>& gp, T* out) const {
        std::fill(out, out + (size_t)nx * ny * nzm, T(0));
        for (int k = -P; k <= nzm + P + 1; ++k)
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i) {
                    const int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), ny),
                              kk = std::min(std::max(k, 1), nzm);
                    out[((size_t)(ii - 1) * ny + (jj - 1)) * nzm + (kk - 1)] += gp(i, j, k);
                }
    }
};

}  // namespace oracle

using namespace oracle;

template <typename T>
static int el3_fwd_impl(const owl_ssg_desc* d, const T* const* f, int nshots, const owl_shot* shots, T* seis) {
    try {
        El3<T> m(*d, f);
        size_t off = 0;
        for (int s = 0; s < nshots; ++s) {
            m.forward_shot(shots[s], seis + off, nullptr, 1 << 30);
            off += (size_t)3 * shots[s].nrec * d->nt;
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" int oracle_el3d_forward_f32(const owl_ssg_desc* d, const float* const* f, int nshots,
                                       const owl_shot* shots, float* seis) {
    return el3_fwd_impl<float>(d, f, nshots, shots, seis);
}

extern "C" int oracle_el3d_forward_f64(const owl_ssg_desc* d, const double* const* f, int nshots,
                                       const owl_shot* shots, double* seis) {
    return el3_fwd_impl<double>(d, f, nshots, shots, seis);
}

extern "C" int oracle_el3d_jvp_c128(const owl_ssg_desc* d, const double* const* f, const double* const* df,
                                    int nshots, const owl_shot* shots, double* seis, double* jvp) {
    typedef std::complex<double> Cx;
    const double h = 1e-30;
    const int np = el3_nparam(d->aniso);
    if (np < 0) return -1;
    const size_t n = (size_t)d->nx * d->ny * d->nz;
    std::vector<std::vector<Cx>> cf(np, std::vector<Cx>(n));
    std::vector<const Cx*> ptr(np);
    for (int q = 0; q < np; ++q) {
        for (size_t i = 0; i < n; ++i) cf[q][i] = Cx(f[q][i], h * df[q][i]);
        ptr[q] = cf[q].data();
    }
    size_t ns = 0;
    for (int s = 0; s < nshots; ++s) ns += (size_t)3 * shots[s].nrec * d->nt;
    std::vector<Cx> out(ns);
    const int rc = el3_fwd_impl<Cx>(d, ptr.data(), nshots, shots, out.data());
    for (size_t i = 0; i < ns; ++i) {
        if (seis) seis[i] = out[i].real();
        jvp[i] = out[i].imag() / h;
    }
    return rc;
}

extern "C" int oracle_el3d_gradient_f64(const owl_ssg_desc* d, const double* const* f, int nshots,
                                        const owl_shot* shots, const double* data, int adj_kind, int k,
                                        double* misfit, double* grad, double* stf_grad) {
    try {
        El3<double> m(*d, f);
        El3<double>::Grad g;
        for (auto& x : g.g) x.init(-m.P, m.nx + m.P + 1, -m.P, m.ny + m.P + 1, -m.P, m.nz + m.P + 1);
        size_t off = 0, soff = 0;
        for (int s = 0; s < nshots; ++s) {
            const owl_shot& sh = shots[s];
            const size_t n = (size_t)3 * sh.nrec * d->nt;
            std::vector<double> res(n, 0.0);
            if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
                std::vector<double> syn(n);
                m.forward_shot(sh, syn.data(), nullptr, 1 << 30);
                double mf = 0;
                for (int comp = 0; comp < 3; ++comp)
                    for (int r = 0; r < sh.nrec; ++r) {
                        if (sh.rec[r].weight == 0.f) continue;
                        for (int t = 0; t < d->nt; ++t) {
                            const size_t q = ((size_t)comp * sh.nrec + r) * d->nt + t;
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
        const size_t nm = (size_t)d->nx * d->ny * d->nz;
        for (int q = 0; q < m.np; ++q) m.fold(g.gpar[q], grad + q * nm);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" void oracle_el3d_set_mpml(const float* faces, long long n) {
    if (faces && n > 0) g_el3_faces.assign(faces, faces + n);
    else g_el3_faces.clear();
}

extern "C" int oracle_el3d_setup(const owl_ssg_desc* d, const float* const* f, float* dt_stable) {
    try {
        El3<float> m(*d, f);
        *dt_stable = m.dt_stable;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}
