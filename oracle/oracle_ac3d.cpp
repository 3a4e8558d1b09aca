// oracle_ac3d.cpp -- CPU oracle for the 3D isotropic acoustic SSG solver.
//
// TEST INFRASTRUCTURE ONLY (see oracle_common.hpp). Restates, single rank:
//   prepare_modeling     src/solver/acoustic_iso_3d/module_vars.f90:108-261
//   CFS-PML coefficients src/solver/acoustic_iso_3d/module_cfspml.f90
//   update_wavefield     src/solver/acoustic_iso_3d/module_wavefield.f90:40-172
//                        (free-surface variant :177-317: p from k = 2, mirror
//                        p(i,j,1-k) = -p(i,j,1+k), no top PML)
//   add_source           module_wavefield.f90:322-444
//   sampling             src/solver/acoustic_iso_3d/submodule_forward_modeling.f90
// plus the exact discrete adjoint of that loop (FP64 gradient oracle).
#include <algorithm>
#include <array>
#include <cstdio>
#include <stdexcept>

#include "oracle_common.hpp"

namespace oracle {

template <typename T>
struct Arr3 {
    int i0, j0, k0, ni, nj, nk;
    std::vector<T> a;
    void init(int lo, int hix, int hiy, int hiz) {
        i0 = j0 = k0 = lo;
        ni = hix - lo + 1; nj = hiy - lo + 1; nk = hiz - lo + 1;
        a.assign((size_t)ni * nj * nk, T(0));
    }
    inline T& operator()(int i, int j, int k) { return a[((size_t)(k - k0) * nj + (j - j0)) * ni + (i - i0)]; }
    inline const T& operator()(int i, int j, int k) const { return a[((size_t)(k - k0) * nj + (j - j0)) * ni + (i - i0)]; }
};

template <typename T>
struct Ac3dState {
    Arr3<T> p, vx, vy, vz, mxv, myv, mzv, mxp, myp, mzp;  // memory of d(vx)/dx ... and of dp/dx ...
    void init(int lo, int hx, int hy, int hz) {
        for (Arr3<T>* q : {&p, &vx, &vy, &vz, &mxv, &myv, &mzv, &mxp, &myp, &mzp}) q->init(lo, hx, hy, hz);
    }
};

template <typename T>
struct Ac3d {
    int nx, ny, nz, pml, R, nt;
    float dx, dy, dz, dt, idx, idy, idz;
    bool fs;
    const float* c;
    Arr3<T> vp, rho, bk;
    Pml1D px, py, pz;
    int lo, hx, hy, hz;

    Ac3d(const owl_ssg_desc& d, const T* vp_in, const T* rho_in) {
        nx = d.nx; ny = d.ny; nz = d.nz; pml = d.pml; R = d.fdhalf; nt = d.nt;
        dx = d.dx; dy = d.dy; dz = d.dz; dt = d.dt; fs = d.free_surface != 0;
        idx = (float)(1.0 / (double)dx); idy = (float)(1.0 / (double)dy); idz = (float)(1.0 / (double)dz);
        c = fdcoefs(R);
        vp.init(-pml, nx + pml + 1, ny + pml + 1, nz + pml + 1);
        rho.init(-pml, nx + pml + 1, ny + pml + 1, nz + pml + 1);
        bk.init(-pml, nx + pml + 1, ny + pml + 1, nz + pml + 1);
        for (int k = -pml; k <= nz + pml + 1; ++k)
            for (int j = -pml; j <= ny + pml + 1; ++j)
                for (int i = -pml; i <= nx + pml + 1; ++i) {
                    int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), ny), kk = std::min(std::max(k, 1), nz);
                    size_t src = ((size_t)(ii - 1) * ny + (jj - 1)) * nz + (kk - 1);
                    vp(i, j, k) = vp_in[src];
                    rho(i, j, k) = rho_in[src];
                    bk(i, j, k) = rho(i, j, k) * vp(i, j, k) * vp(i, j, k);
                }
        float pmlvp = -1e30f;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j) pmlvp = std::max({pmlvp, (float)re(vp(1, j, k)), (float)re(vp(nx, j, k))});
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, (float)re(vp(i, 1, k)), (float)re(vp(i, ny, k))});
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, (float)re(vp(i, j, 1)), (float)re(vp(i, j, nz))});
        float alphamax = (float)(1.0 * (double)d.f0_max * 3.14159265358979323846);
        px.build(nx, pml, dx, dt, pmlvp, alphamax);
        py.build(ny, pml, dy, dt, pmlvp, alphamax);
        pz.build(nz, pml, dz, dt, pmlvp, alphamax);
        lo = -pml - R + 1; hx = nx + pml + R; hy = ny + pml + R; hz = nz + pml + R;
    }

    bool zpml_i(int k) const { return (!fs && k <= 0) || k >= nz + 1; }
    bool zpml_h(int k) const { return (!fs && k <= 1) || k >= nz + 1; }

    // S[0] = p-update stencil term, S[1..3] = vx, vy, vz update terms
    void update(Ac3dState<T>& s, Arr3<T>* S) const {
        const int P = pml, k0 = fs ? 2 : -P + 1;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = k0; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    T sx = T(0), sy = T(0), sz = T(0);
                    for (int q = 1; q <= R; ++q) sx = sx + T(c[q - 1]) * (s.vx(i + q, j, k) - s.vx(i - q + 1, j, k));
                    for (int q = 1; q <= R; ++q) sy = sy + T(c[q - 1]) * (s.vy(i, j + q, k) - s.vy(i, j - q + 1, k));
                    for (int q = 1; q <= R; ++q) sz = sz + T(c[q - 1]) * (s.vz(i, j, k + q) - s.vz(i, j, k - q + 1));
                    T gx = T(idx) * sx, gy = T(idy) * sy, gz = T(idz) * sz;
                    if (i <= 0 || i >= nx + 1) {
                        s.mxv(i, j, k) = T(px.ai(i)) * gx + T(px.bi(i)) * s.mxv(i, j, k);
                        gx = (gx + s.mxv(i, j, k)) / T(px.ki(i));
                    }
                    if (j <= 0 || j >= ny + 1) {
                        s.myv(i, j, k) = T(py.ai(j)) * gy + T(py.bi(j)) * s.myv(i, j, k);
                        gy = (gy + s.myv(i, j, k)) / T(py.ki(j));
                    }
                    if (zpml_i(k)) {
                        s.mzv(i, j, k) = T(pz.ai(k)) * gz + T(pz.bi(k)) * s.mzv(i, j, k);
                        gz = (gz + s.mzv(i, j, k)) / T(pz.ki(k));
                    }
                    s.p(i, j, k) = s.p(i, j, k) - T(dt) * bk(i, j, k) * (gx + gy + gz);
                    if (S) S[0](i, j, k) = gx + gy + gz;
                }
        if (fs) {
            for (int k = -P + 1; k <= 0; ++k)
                for (int j = -P + 1; j <= ny + P; ++j)
                    for (int i = -P + 1; i <= nx + P; ++i) s.p(i, j, k) = -s.p(i, j, 2 - k);
        }
        const int kv = fs ? 1 : -P + 1;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = kv; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int m = -P + 1; m <= nx + P; ++m) {
                    // vx(m) = vx(i+1) with i = m-1 (module_wavefield.f90:106-123), same for vy
                    T h = T(0), hy = T(0);
                    for (int q = 1; q <= R; ++q) h = h + T(c[q - 1]) * (s.p(m + q - 1, j, k) - s.p(m - q, j, k));
                    for (int q = 1; q <= R; ++q) hy = hy + T(c[q - 1]) * (s.p(m, j + q - 1, k) - s.p(m, j - q, k));
                    h = T(idx) * h;
                    hy = T(idy) * hy;
                    if (m <= 1 || m >= nx + 1) {
                        s.mxp(m, j, k) = T(px.ah(m)) * h + T(px.bh(m)) * s.mxp(m, j, k);
                        h = (h + s.mxp(m, j, k)) / T(px.kh(m));
                    }
                    if (j <= 1 || j >= ny + 1) {
                        s.myp(m, j, k) = T(py.ah(j)) * hy + T(py.bh(j)) * s.myp(m, j, k);
                        hy = (hy + s.myp(m, j, k)) / T(py.kh(j));
                    }
                    T rx = T(0.5f) * (rho(m, j, k) + rho(m - 1, j, k));
                    T ry = T(0.5f) * (rho(m, j, k) + rho(m, j - 1, k));
                    s.vx(m, j, k) = s.vx(m, j, k) - T(dt) / rx * h;
                    s.vy(m, j, k) = s.vy(m, j, k) - T(dt) / ry * hy;
                    if (S) { S[1](m, j, k) = h; S[2](m, j, k) = hy; }
                }
        const int kz0 = fs ? 2 : -P + 1;
#pragma omp parallel for collapse(2) schedule(static)
        for (int m = kz0; m <= nz + P; ++m)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    T h = T(0);
                    for (int q = 1; q <= R; ++q) h = h + T(c[q - 1]) * (s.p(i, j, m + q - 1) - s.p(i, j, m - q));
                    h = T(idz) * h;
                    if (zpml_h(m)) {
                        s.mzp(i, j, m) = T(pz.ah(m)) * h + T(pz.bh(m)) * s.mzp(i, j, m);
                        h = (h + s.mzp(i, j, m)) / T(pz.kh(m));
                    }
                    T rz = T(0.5f) * (rho(i, j, m) + rho(i, j, m - 1));
                    s.vz(i, j, m) = s.vz(i, j, m) - T(dt) / rz * h;
                    if (S) S[3](i, j, m) = h;
                }
    }

    T taps3(const float* a, const float* b, const float* cc, int x, int y, int z) const {
        return T(a[x + 4]) * T(b[y + 4]) * T(cc[z + 4]);
    }

    void add_source(int t, const owl_shot& sh, Ac3dState<T>& s) const {
        for (int q = 0; q < sh.nsrc; ++q) {
            const owl_source& sr = sh.src[q];
            if (t < sr.nbeg || t > sr.nbeg + sr.nt_stf - 1) continue;
            T amp = T(sr.stf[t - sr.nbeg]) * T(sr.amp) * T(dt);
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx) {
                        if (sr.mechanism == OWL_SRC_FORCE) {
                            T a2 = amp / rho(sr.gx, sr.gy, sr.gz);
                            if (!fs || sr.gz + irz >= 2)
                                s.vx(sr.hx + irx, sr.gy + iry, sr.gz + irz) += T(std::sin(sr.polar) * std::cos(sr.azimuth)) * a2 *
                                    taps3(sr.interp_hx, sr.interp_iy, sr.interp_iz, irx, iry, irz);
                            if (!fs || sr.gz + irz >= 2)
                                s.vy(sr.gx + irx, sr.hy + iry, sr.gz + irz) += T(std::sin(sr.polar) * std::sin(sr.azimuth)) * a2 *
                                    taps3(sr.interp_ix, sr.interp_hy, sr.interp_iz, irx, iry, irz);
                            if (!fs || sr.hz + irz >= 2)
                                s.vz(sr.gx + irx, sr.gy + iry, sr.hz + irz) += T(std::cos(sr.polar)) * a2 *
                                    taps3(sr.interp_ix, sr.interp_iy, sr.interp_hz, irx, iry, irz);
                        } else if (!fs || sr.gz + irz >= 2) {
                            s.p(sr.gx + irx, sr.gy + iry, sr.gz + irz) +=
                                amp * taps3(sr.interp_ix, sr.interp_iy, sr.interp_iz, irx, iry, irz);
                        }
                    }
        }
    }

    void sample(int t, const owl_shot& sh, const Ac3dState<T>& s, T* out) const {
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T acc = T(0);
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx)
                        acc = acc + s.p(q.gx + irx, q.gy + iry, q.gz + irz) *
                                        taps3(q.interp_ix, q.interp_iy, q.interp_iz, irx, iry, irz) * T(q.weight);
            out[(size_t)r * nt + (t - 1)] = acc;
        }
    }

    void forward_shot(const owl_shot& sh, T* seis, std::vector<Ac3dState<T>>* ck, int k) const {
        Ac3dState<T> s;
        s.init(lo, hx, hy, hz);
        std::fill(seis, seis + (size_t)sh.nrec * nt, T(0));
        for (int t = 1; t <= nt; ++t) {
            if (ck && (t - 1) % k == 0) ck->push_back(s);
            sample(t, sh, s, seis);
            update(s, nullptr);
            add_source(t, sh, s);
        }
    }

    // adjoint of one step (no force sources in the 3D gradient oracle)
    void adjoint_step(int t, const owl_shot& sh, Ac3dState<T>& a, Arr3<T>* S, const T* res, Arr3<T>& gv, Arr3<T>& gr) const {
        const int P = pml;
        // reverse vz update
        const int kz0 = fs ? 2 : -P + 1;
        for (int m = kz0; m <= nz + P; ++m)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    T rz = T(0.5f) * (rho(i, j, m) + rho(i, j, m - 1));
                    T zh = a.vz(i, j, m);
                    T g = zh * S[3](i, j, m) * T(dt) * T(0.5f) / (rz * rz);
                    gr(i, j, m) += g; gr(i, j, m - 1) += g;
                    T q = -T(dt) / rz * zh, e = q;
                    if (zpml_h(m)) {
                        T u = q / T(pz.kh(m)) + a.mzp(i, j, m);
                        a.mzp(i, j, m) = T(pz.bh(m)) * u;
                        e = q / T(pz.kh(m)) + T(pz.ah(m)) * u;
                    }
                    e = T(idz) * e;
                    for (int qq = 1; qq <= R; ++qq) {
                        a.p(i, j, m + qq - 1) += T(c[qq - 1]) * e;
                        a.p(i, j, m - qq) -= T(c[qq - 1]) * e;
                    }
                }
        // reverse vx, vy updates
        const int kv = fs ? 1 : -P + 1;
        for (int k = kv; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int m = -P + 1; m <= nx + P; ++m) {
                    T rx = T(0.5f) * (rho(m, j, k) + rho(m - 1, j, k));
                    T ry = T(0.5f) * (rho(m, j, k) + rho(m, j - 1, k));
                    T xh = a.vx(m, j, k), yh = a.vy(m, j, k);
                    T g1 = xh * S[1](m, j, k) * T(dt) * T(0.5f) / (rx * rx);
                    gr(m, j, k) += g1; gr(m - 1, j, k) += g1;
                    T g2 = yh * S[2](m, j, k) * T(dt) * T(0.5f) / (ry * ry);
                    gr(m, j, k) += g2; gr(m, j - 1, k) += g2;
                    T q = -T(dt) / rx * xh, e = q;
                    if (m <= 1 || m >= nx + 1) {
                        T u = q / T(px.kh(m)) + a.mxp(m, j, k);
                        a.mxp(m, j, k) = T(px.bh(m)) * u;
                        e = q / T(px.kh(m)) + T(px.ah(m)) * u;
                    }
                    e = T(idx) * e;
                    for (int qq = 1; qq <= R; ++qq) {
                        a.p(m + qq - 1, j, k) += T(c[qq - 1]) * e;
                        a.p(m - qq, j, k) -= T(c[qq - 1]) * e;
                    }
                    T qy = -T(dt) / ry * yh, ey = qy;
                    if (j <= 1 || j >= ny + 1) {
                        T u = qy / T(py.kh(j)) + a.myp(m, j, k);
                        a.myp(m, j, k) = T(py.bh(j)) * u;
                        ey = qy / T(py.kh(j)) + T(py.ah(j)) * u;
                    }
                    ey = T(idy) * ey;
                    for (int qq = 1; qq <= R; ++qq) {
                        a.p(m, j + qq - 1, k) += T(c[qq - 1]) * ey;
                        a.p(m, j - qq, k) -= T(c[qq - 1]) * ey;
                    }
                }
        if (fs) {
            for (int k = 0; k >= -P + 1; --k)
                for (int j = -P + 1; j <= ny + P; ++j)
                    for (int i = -P + 1; i <= nx + P; ++i) {
                        a.p(i, j, 2 - k) -= a.p(i, j, k);
                        a.p(i, j, k) = T(0);
                    }
        }
        // reverse p update
        const int k0 = fs ? 2 : -P + 1;
        for (int k = k0; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    T ph = a.p(i, j, k);
                    T gbk = -T(dt) * ph * S[0](i, j, k);
                    gv(i, j, k) += gbk * T(2.0) * rho(i, j, k) * vp(i, j, k);
                    gr(i, j, k) += gbk * vp(i, j, k) * vp(i, j, k);
                    T q = -T(dt) * bk(i, j, k) * ph, ex = q, ey = q, ez = q;
                    if (i <= 0 || i >= nx + 1) {
                        T u = q / T(px.ki(i)) + a.mxv(i, j, k);
                        a.mxv(i, j, k) = T(px.bi(i)) * u;
                        ex = q / T(px.ki(i)) + T(px.ai(i)) * u;
                    }
                    if (j <= 0 || j >= ny + 1) {
                        T u = q / T(py.ki(j)) + a.myv(i, j, k);
                        a.myv(i, j, k) = T(py.bi(j)) * u;
                        ey = q / T(py.ki(j)) + T(py.ai(j)) * u;
                    }
                    if (zpml_i(k)) {
                        T u = q / T(pz.ki(k)) + a.mzv(i, j, k);
                        a.mzv(i, j, k) = T(pz.bi(k)) * u;
                        ez = q / T(pz.ki(k)) + T(pz.ai(k)) * u;
                    }
                    ex = T(idx) * ex; ey = T(idy) * ey; ez = T(idz) * ez;
                    for (int qq = 1; qq <= R; ++qq) {
                        a.vx(i + qq, j, k) += T(c[qq - 1]) * ex;
                        a.vx(i - qq + 1, j, k) -= T(c[qq - 1]) * ex;
                        a.vy(i, j + qq, k) += T(c[qq - 1]) * ey;
                        a.vy(i, j - qq + 1, k) -= T(c[qq - 1]) * ey;
                        a.vz(i, j, k + qq) += T(c[qq - 1]) * ez;
                        a.vz(i, j, k - qq + 1) -= T(c[qq - 1]) * ez;
                    }
                }
        // clear entries outside each field's update range
        const int pz0 = fs ? 2 : -P + 1, vx0 = fs ? 1 : -P + 1, vz0 = fs ? 2 : -P + 1;
        for (int k = lo; k <= hz; ++k)
            for (int j = lo; j <= hy; ++j)
                for (int i = lo; i <= hx; ++i) {
                    bool in = i >= -P + 1 && i <= nx + P && j >= -P + 1 && j <= ny + P && k <= nz + P;
                    if (!(in && k >= pz0)) a.p(i, j, k) = T(0);
                    if (!(in && k >= vx0)) { a.vx(i, j, k) = T(0); a.vy(i, j, k) = T(0); }
                    if (!(in && k >= vz0)) a.vz(i, j, k) = T(0);
                }
        // adjoint of the sampling of step t
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T rv = res[(size_t)r * nt + (t - 1)];
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx) {
                        int kk = q.gz + irz;
                        T w = rv * taps3(q.interp_ix, q.interp_iy, q.interp_iz, irx, iry, irz) * T(q.weight);
                        if (fs && kk <= 0) a.p(q.gx + irx, q.gy + iry, 2 - kk) -= w;
                        else if (!fs || kk >= 2) a.p(q.gx + irx, q.gy + iry, kk) += w;
                    }
        }
    }
};

}  // namespace oracle

using namespace oracle;

template <typename T>
static int fwd3(const owl_ssg_desc* d, const T* vp, const T* rho, int nshots, const owl_shot* shots, T* seis) {
    try {
        Ac3d<T> m(*d, vp, rho);
        size_t off = 0;
        for (int s = 0; s < nshots; ++s) {
            m.forward_shot(shots[s], seis + off, nullptr, 1 << 30);
            off += (size_t)shots[s].nrec * d->nt;
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" int oracle_ac3d_forward_f32(const owl_ssg_desc* d, const float* vp, const float* rho, int nshots,
                                       const owl_shot* shots, float* seis) {
    return fwd3<float>(d, vp, rho, nshots, shots, seis);
}
extern "C" int oracle_ac3d_forward_f64(const owl_ssg_desc* d, const double* vp, const double* rho, int nshots,
                                       const owl_shot* shots, double* seis) {
    return fwd3<double>(d, vp, rho, nshots, shots, seis);
}
extern "C" int oracle_ac3d_jvp_c128(const owl_ssg_desc* d, const double* vp, const double* rho, const double* dvp,
                                    const double* drho, int nshots, const owl_shot* shots, double* seis_jvp) {
    typedef std::complex<double> C;
    const double h = 1e-30;
    size_t n = (size_t)d->nx * d->ny * d->nz;
    std::vector<C> cv(n), cr(n);
    for (size_t i = 0; i < n; ++i) { cv[i] = C(vp[i], h * dvp[i]); cr[i] = C(rho[i], h * drho[i]); }
    size_t ns = 0;
    for (int s = 0; s < nshots; ++s) ns += (size_t)shots[s].nrec * d->nt;
    std::vector<C> out(ns);
    int rc = fwd3<C>(d, cv.data(), cr.data(), nshots, shots, out.data());
    for (size_t i = 0; i < ns; ++i) seis_jvp[i] = out[i].imag() / h;
    return rc;
}

// exact gradient in FP64 of J = 0.5 sum (syn - obs)^2 (adj_kind 0) or of <syn, data> (adj_kind 1)
extern "C" int oracle_ac3d_gradient_f64(const owl_ssg_desc* d, const double* vp, const double* rho, int nshots,
                                        const owl_shot* shots, const double* data, int adj_kind, int k,
                                        double* misfit, double* grad) {
    try {
        Ac3d<double> m(*d, vp, rho);
        const int P = m.pml;
        Arr3<double> gv, gr;
        gv.init(-P, d->nx + P + 1, d->ny + P + 1, d->nz + P + 1);
        gr.init(-P, d->nx + P + 1, d->ny + P + 1, d->nz + P + 1);
        size_t off = 0;
        for (int s = 0; s < nshots; ++s) {
            const owl_shot& sh = shots[s];
            size_t n = (size_t)sh.nrec * d->nt;
            std::vector<double> res(n, 0.0), syn(n);
            std::vector<Ac3dState<double>> ck;
            m.forward_shot(sh, syn.data(), &ck, k);
            double mf = 0;
            for (int r = 0; r < sh.nrec; ++r) {
                if (sh.rec[r].weight == 0.f) continue;
                for (int t = 0; t < d->nt; ++t) {
                    size_t q = (size_t)r * d->nt + t;
                    if (adj_kind == 0) {
                        res[q] = syn[q] - data[off + q];
                        mf += res[q] * res[q];
                    } else {
                        res[q] = data[off + q];
                    }
                }
            }
            if (misfit) misfit[s] = mf;
            Ac3dState<double> a;
            a.init(m.lo, m.hx, m.hy, m.hz);
            std::vector<std::array<Arr3<double>, 4>> Sb(k);
            for (auto& s4 : Sb)
                for (auto& q : s4) q.init(m.lo, m.hx, m.hy, m.hz);
            for (int sg = (int)ck.size() - 1; sg >= 0; --sg) {
                int n0 = sg * k, n1 = std::min(d->nt, n0 + k);
                Ac3dState<double> st = ck[sg];
                for (int t = n0 + 1; t <= n1; ++t) {
                    m.update(st, Sb[t - n0 - 1].data());
                    m.add_source(t, sh, st);
                }
                for (int t = n1; t >= n0 + 1; --t) m.adjoint_step(t, sh, a, Sb[t - n0 - 1].data(), res.data(), gv, gr);
            }
            off += n;
        }
        size_t nm = (size_t)d->nx * d->ny * d->nz;
        std::fill(grad, grad + 2 * nm, 0.0);
        for (int kk = -P; kk <= d->nz + P + 1; ++kk)
            for (int j = -P; j <= d->ny + P + 1; ++j)
                for (int i = -P; i <= d->nx + P + 1; ++i) {
                    int ii = std::min(std::max(i, 1), d->nx), jj = std::min(std::max(j, 1), d->ny),
                        zz = std::min(std::max(kk, 1), d->nz);
                    size_t o = ((size_t)(ii - 1) * d->ny + (jj - 1)) * d->nz + (zz - 1);
                    grad[o] += gv(i, j, kk);
                    grad[nm + o] += gr(i, j, kk);
                }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}
