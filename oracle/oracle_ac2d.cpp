// oracle_ac2d.cpp -- CPU oracle for the 2D isotropic acoustic SSG solver.
//
// TEST INFRASTRUCTURE ONLY (see oracle_common.hpp). Restates, loop by loop:
//   prepare_modeling           src/solver/acoustic_iso_2d/module_vars.f90:90-134
//   CFS-PML coefficients       src/solver/acoustic_iso_2d/module_cfspml.f90:37-133
//   update_wavefield           src/solver/acoustic_iso_2d/module_wavefield.f90:40-107
//   update_wavefield_free_surface                      module_wavefield.f90:112-187
//   add_source                 src/solver/acoustic_iso_2d/module_wavefield.f90:192-263
//   time loop + sampling       src/solver/acoustic_iso_2d/submodule_forward_modeling.f90:48-117
//   L2 misfit / adjoint source src/inverse/module_inversion_adjoint_source.f90:371-383
// and adds the exact discrete adjoint of that forward loop (the reference's own
// gradient, submodule_fwi_gradient.f90:31-269, back-propagates with -dt and is
// not the transpose; it is restated separately in ref_gradient below).
//
// Templated on T: float (forward parity oracle), double (FP64 gradient oracle),
// std::complex<double> (complex-step Jacobian-vector products).
#include <algorithm>
#include <array>
#include <cstdio>
#include <stdexcept>

#include "oracle_common.hpp"

namespace oracle {

template <typename T>
struct Ac2dState {
    Arr2<T> p, vx, vz, mpdxvx, mpdzvz, mpdxp, mpdzp;
    void init(int lo_x, int hi_x, int lo_z, int hi_z) {
        for (Arr2<T>* a : {&p, &vx, &vz, &mpdxvx, &mpdzvz, &mpdxp, &mpdzp}) a->init(lo_x, hi_x, lo_z, hi_z);
    }
};

template <typename T>
struct Ac2d {
    int nx, nz, pml, R, nt;
    float dx, dz, dt, idx, idz;
    bool fs;
    const float* c;
    Arr2<T> vp, rho, bk;  // padded by pml+1 (pad_array, module_vars.f90:113-115)
    Pml1D px, pz;
    int lo_x, hi_x, lo_z, hi_z;  // wavefield bounds: pad = pml + fdhalf

    Ac2d(const owl_ssg_desc& d, const T* vp_in, const T* rho_in) {
        nx = d.nx; nz = d.nz; pml = d.pml; R = d.fdhalf; nt = d.nt;
        dx = d.dx; dz = d.dz; dt = d.dt; fs = d.free_surface != 0;
        idx = (float)(1.0 / (double)dx);
        idz = (float)(1.0 / (double)dz);
        c = fdcoefs(R);
        // transpose (nz,nx) z-fastest -> (i,j) x-fastest, then edge-replicate pad
        vp.init(-pml, nx + pml + 1, -pml, nz + pml + 1);
        rho.init(-pml, nx + pml + 1, -pml, nz + pml + 1);
        bk.init(-pml, nx + pml + 1, -pml, nz + pml + 1);
        for (int j = -pml; j <= nz + pml + 1; ++j)
            for (int i = -pml; i <= nx + pml + 1; ++i) {
                int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nz);
                size_t src = (size_t)(ii - 1) * nz + (jj - 1);
                vp(i, j) = vp_in[src];
                rho(i, j) = rho_in[src];
                bk(i, j) = rho(i, j) * vp(i, j) * vp(i, j);
            }
        // pmlvp = max of vp on the four model edges (module_cfspml.f90:93)
        float pmlvp = -1e30f;
        for (int j = 1; j <= nz; ++j) pmlvp = std::max({pmlvp, (float)re(vp(1, j)), (float)re(vp(nx, j))});
        for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, (float)re(vp(i, 1)), (float)re(vp(i, nz))});
        float alphamax = (float)(1.0 * (double)d.f0_max * 3.14159265358979323846);
        px.build(nx, pml, dx, dt, pmlvp, alphamax);
        pz.build(nz, pml, dz, dt, pmlvp, alphamax);
        lo_x = -pml - R + 1; hi_x = nx + pml + R;
        lo_z = -pml - R + 1; hi_z = nz + pml + R;
    }

    // forward update. If S != nullptr, store the stencil terms that multiply the
    // material coefficients (needed by the exact gradient): S[0] = pdxvx + pdzvz
    // at cells, S[1] = pdxp at vx nodes, S[2] = pdzp at vz nodes.
    void update(float dtt, Ac2dState<T>& s, Arr2<T>* S) const {
        const int P = pml;
        const int jbeg = fs ? 2 : -P + 1;
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = jbeg; j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T sx = T(0), sz = T(0);
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.vx(i + k, j) - s.vx(i - k + 1, j));
                for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.vz(i, j + k) - s.vz(i, j - k + 1));
                T pdxvx = T(idx) * sx, pdzvz = T(idz) * sz;
                if (i <= 0 || i >= nx + 1) {
                    s.mpdxvx(i, j) = T(px.ai(i)) * pdxvx + T(px.bi(i)) * s.mpdxvx(i, j);
                    pdxvx = (pdxvx + s.mpdxvx(i, j)) / T(px.ki(i));
                }
                if ((!fs && j <= 0) || j >= nz + 1) {
                    s.mpdzvz(i, j) = T(pz.ai(j)) * pdzvz + T(pz.bi(j)) * s.mpdzvz(i, j);
                    pdzvz = (pdzvz + s.mpdzvz(i, j)) / T(pz.ki(j));
                }
                s.p(i, j) = s.p(i, j) - T(dtt) * bk(i, j) * (pdxvx + pdzvz);
                if (S) S[0](i, j) = pdxvx + pdzvz;
            }
        if (fs) {
#pragma omp parallel for collapse(2) schedule(static)
            for (int j = -P + 1; j <= 0; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) s.p(i, j) = -s.p(i, 2 - j);
        }
        const int jbeg_x = fs ? 1 : -P + 1;
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = jbeg_x; j <= nz + P; ++j)
            for (int i = -P; i <= nx + P - 1; ++i) {
                T sx = T(0);
                for (int k = 1; k <= R; ++k) sx = sx + T(c[k - 1]) * (s.p(i + k, j) - s.p(i - k + 1, j));
                T pdxp = T(idx) * sx;
                if (i + 1 <= 1 || i + 1 >= nx + 1) {
                    s.mpdxp(i + 1, j) = T(px.ah(i + 1)) * pdxp + T(px.bh(i + 1)) * s.mpdxp(i + 1, j);
                    pdxp = (pdxp + s.mpdxp(i + 1, j)) / T(px.kh(i + 1));
                }
                T rho_eff = T(0.5f) * (rho(i + 1, j) + rho(i, j));
                s.vx(i + 1, j) = s.vx(i + 1, j) - T(dtt) / rho_eff * pdxp;
                if (S) S[1](i + 1, j) = pdxp;
            }
        const int jbeg_z = fs ? 1 : -P;
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = jbeg_z; j <= nz + P - 1; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T sz = T(0);
                for (int k = 1; k <= R; ++k) sz = sz + T(c[k - 1]) * (s.p(i, j + k) - s.p(i, j - k + 1));
                T pdzp = T(idz) * sz;
                if ((!fs && j + 1 <= 1) || j + 1 >= nz + 1) {
                    s.mpdzp(i, j + 1) = T(pz.ah(j + 1)) * pdzp + T(pz.bh(j + 1)) * s.mpdzp(i, j + 1);
                    pdzp = (pdzp + s.mpdzp(i, j + 1)) / T(pz.kh(j + 1));
                }
                T rho_eff = T(0.5f) * (rho(i, j + 1) + rho(i, j));
                s.vz(i, j + 1) = s.vz(i, j + 1) - T(dtt) / rho_eff * pdzp;
                if (S) S[2](i, j + 1) = pdzp;
            }
    }

    // add_source(t) (module_wavefield.f90:192-263). stf_scale multiplies every
    // STF sample (1 for modelling; used to build linear-in-source tests).
    void add_source(int t, const owl_shot& sh, Ac2dState<T>& s) const {
        for (int k = 0; k < sh.nsrc; ++k) {
            const owl_source& q = sh.src[k];
            int nbeg = q.nbeg, nend = nbeg + q.nt_stf - 1;
            if (t < nbeg || t > nend) continue;
            T amp = T(q.stf[t - nbeg]) * T(q.amp) * T(dt);
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
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx)
                        if (!fs || q.gz + irz >= 2)
                            s.p(q.gx + irx, q.gz + irz) = s.p(q.gx + irx, q.gz + irz) +
                                amp * T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]);
            }
        }
    }

    // receiver sampling at step t (submodule_forward_modeling.f90:58-79) into
    // out[r*nt + (t-1)].
    void sample(int t, const owl_shot& sh, const Ac2dState<T>& s, T* out) const {
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T acc = out[(size_t)r * nt + (t - 1)];
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx)
                    acc = acc + s.p(q.gx + irx, q.gz + irz) * T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]) * T(q.weight);
            out[(size_t)r * nt + (t - 1)] = acc;
        }
    }

    void forward_shot(const owl_shot& sh, T* seis, std::vector<Ac2dState<T>>* ckpt, int k) const {
        Ac2dState<T> s;
        s.init(lo_x, hi_x, lo_z, hi_z);
        std::fill(seis, seis + (size_t)sh.nrec * nt, T(0));
        for (int t = 1; t <= nt; ++t) {
            if (ckpt && (t - 1) % k == 0) ckpt->push_back(s);
            sample(t, sh, s, seis);
            update(dt, s, nullptr);
            add_source(t, sh, s);
        }
    }

    // ---------------- exact discrete adjoint -----------------------------------
    struct Grad {
        Arr2<T> gvp, grho;  // on the padded model grid [-pml, n+pml+1]
    };

    // adjoint of one forward step t. a = adjoint state (p^, vx^, vz^, memory^),
    // S = stored stencil terms of step t, s_fwd_rho for force-source rho terms.
    void adjoint_step(int t, const owl_shot& sh, Ac2dState<T>& a, Arr2<T>* S, const T* res,
                      Grad& g, T* stf_grad) const {
        const int P = pml;
        // source injection: gradient w.r.t. stf samples and rho at force points
        for (int kk = 0; kk < sh.nsrc; ++kk) {
            const owl_source& q = sh.src[kk];
            int nbeg = q.nbeg, nend = nbeg + q.nt_stf - 1;
            if (t < nbeg || t > nend) continue;
            T amp = T(q.stf[t - nbeg]) * T(q.amp) * T(dt);
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
                T ap = T(0);
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx)
                        if (!fs || q.gz + irz >= 2)
                            ap = ap + a.p(q.gx + irx, q.gz + irz) * T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]);
                dstf = ap * T(q.amp) * T(dt);
            }
            if (stf_grad) stf_grad[(size_t)kk * nt + (t - 1)] = stf_grad[(size_t)kk * nt + (t - 1)] + dstf;
        }
        // reverse the vz update (module_wavefield.f90:90-105)
        const int jbeg_z = fs ? 1 : -P;
        for (int j = jbeg_z; j <= nz + P - 1; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T rho_eff = T(0.5f) * (rho(i, j + 1) + rho(i, j));
                T coef = T(dt) / rho_eff;
                T zhat = a.vz(i, j + 1);
                // gradient: d vz / d rho = pdzp_out * dt * 0.5 / rho_eff^2 for both rho
                T gr = zhat * S[2](i, j + 1) * T(dt) * T(0.5f) / (rho_eff * rho_eff);
                g.grho(i, j + 1) = g.grho(i, j + 1) + gr;
                g.grho(i, j) = g.grho(i, j) + gr;
                T q = -coef * zhat;
                T e = q;
                if ((!fs && j + 1 <= 1) || j + 1 >= nz + 1) {
                    T kk = T(pz.kh(j + 1));
                    T u = q / kk + a.mpdzp(i, j + 1);
                    a.mpdzp(i, j + 1) = T(pz.bh(j + 1)) * u;
                    e = q / kk + T(pz.ah(j + 1)) * u;
                }
                e = T(idz) * e;
                for (int k = 1; k <= R; ++k) {
                    a.p(i, j + k) = a.p(i, j + k) + T(c[k - 1]) * e;
                    a.p(i, j - k + 1) = a.p(i, j - k + 1) - T(c[k - 1]) * e;
                }
            }
        // reverse the vx update (module_wavefield.f90:73-88)
        const int jbeg_x = fs ? 1 : -P + 1;
        for (int j = jbeg_x; j <= nz + P; ++j)
            for (int i = -P; i <= nx + P - 1; ++i) {
                T rho_eff = T(0.5f) * (rho(i + 1, j) + rho(i, j));
                T coef = T(dt) / rho_eff;
                T xhat = a.vx(i + 1, j);
                T gr = xhat * S[1](i + 1, j) * T(dt) * T(0.5f) / (rho_eff * rho_eff);
                g.grho(i + 1, j) = g.grho(i + 1, j) + gr;
                g.grho(i, j) = g.grho(i, j) + gr;
                T q = -coef * xhat;
                T e = q;
                if (i + 1 <= 1 || i + 1 >= nx + 1) {
                    T kk = T(px.kh(i + 1));
                    T u = q / kk + a.mpdxp(i + 1, j);
                    a.mpdxp(i + 1, j) = T(px.bh(i + 1)) * u;
                    e = q / kk + T(px.ah(i + 1)) * u;
                }
                e = T(idx) * e;
                for (int k = 1; k <= R; ++k) {
                    a.p(i + k, j) = a.p(i + k, j) + T(c[k - 1]) * e;
                    a.p(i - k + 1, j) = a.p(i - k + 1, j) - T(c[k - 1]) * e;
                }
            }
        // reverse the free-surface mirror p(i,j) = -p(i,2-j), j <= 0
        if (fs) {
            for (int j = 0; j >= -P + 1; --j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    a.p(i, 2 - j) = a.p(i, 2 - j) - a.p(i, j);
                    a.p(i, j) = T(0);
                }
        }
        // reverse the p update (module_wavefield.f90:51-71)
        const int jbeg = fs ? 2 : -P + 1;
        for (int j = jbeg; j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                T phat = a.p(i, j);
                // d p / d bk = -dt * S0 ; bk = rho vp^2
                T gbk = -T(dt) * phat * S[0](i, j);
                g.gvp(i, j) = g.gvp(i, j) + gbk * T(2.0) * rho(i, j) * vp(i, j);
                g.grho(i, j) = g.grho(i, j) + gbk * vp(i, j) * vp(i, j);
                T q = -T(dt) * bk(i, j) * phat;
                T ex = q, ez = q;
                if (i <= 0 || i >= nx + 1) {
                    T kk = T(px.ki(i));
                    T u = q / kk + a.mpdxvx(i, j);
                    a.mpdxvx(i, j) = T(px.bi(i)) * u;
                    ex = q / kk + T(px.ai(i)) * u;
                }
                if ((!fs && j <= 0) || j >= nz + 1) {
                    T kk = T(pz.ki(j));
                    T u = q / kk + a.mpdzvz(i, j);
                    a.mpdzvz(i, j) = T(pz.bi(j)) * u;
                    ez = q / kk + T(pz.ai(j)) * u;
                }
                ex = T(idx) * ex;
                ez = T(idz) * ez;
                for (int k = 1; k <= R; ++k) {
                    a.vx(i + k, j) = a.vx(i + k, j) + T(c[k - 1]) * ex;
                    a.vx(i - k + 1, j) = a.vx(i - k + 1, j) - T(c[k - 1]) * ex;
                    a.vz(i, j + k) = a.vz(i, j + k) + T(c[k - 1]) * ez;
                    a.vz(i, j - k + 1) = a.vz(i, j - k + 1) - T(c[k - 1]) * ez;
                }
            }
        // entries of the adjoint state outside each field's update range belong
        // to constants (halo, rows above a free surface); clear them
        const int pz0 = fs ? 2 : -P + 1, vx0 = fs ? 1 : -P + 1, vz0 = fs ? 2 : -P + 1;
        for (int j = lo_z; j <= hi_z; ++j)
            for (int i = lo_x; i <= hi_x; ++i) {
                bool inx = i >= -P + 1 && i <= nx + P, inz = j <= nz + P;
                if (!(inx && inz && j >= pz0)) a.p(i, j) = T(0);
                if (!(inx && inz && j >= vx0)) a.vx(i, j) = T(0);
                if (!(inx && inz && j >= vz0)) a.vz(i, j) = T(0);
            }
        // adjoint of the sampling at step t: p^ += res * taps * weight
        for (int r = 0; r < sh.nrec; ++r) {
            const owl_receiver& q = sh.rec[r];
            if (q.weight == 0.f) continue;
            T rv = res[(size_t)r * nt + (t - 1)];
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx)
                    a.p(q.gx + irx, q.gz + irz) = a.p(q.gx + irx, q.gz + irz) +
                        rv * T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]) * T(q.weight);
        }
    }

    // gradient of J = 0.5 sum res^2 given the adjoint source res (nrec x nt) of one shot
    void adjoint_shot(const owl_shot& sh, const T* res, int k, Grad& g, T* stf_grad) const {
        std::vector<Ac2dState<T>> ck;
        std::vector<T> dummy((size_t)sh.nrec * nt);
        forward_shot(sh, dummy.data(), &ck, k);
        Ac2dState<T> a;
        a.init(lo_x, hi_x, lo_z, hi_z);
        int nseg = (int)ck.size();
        std::vector<std::array<Arr2<T>, 3>> Sbuf((size_t)k);
        for (auto& s3 : Sbuf)
            for (auto& arr : s3) arr.init(lo_x, hi_x, lo_z, hi_z);
        for (int sg = nseg - 1; sg >= 0; --sg) {
            int n0 = sg * k, n1 = std::min(nt, n0 + k);
            Ac2dState<T> s = ck[sg];
            for (int t = n0 + 1; t <= n1; ++t) {
                update(dt, s, Sbuf[t - n0 - 1].data());
                add_source(t, sh, s);
            }
            for (int t = n1; t >= n0 + 1; --t) adjoint_step(t, sh, a, Sbuf[t - n0 - 1].data(), res, g, stf_grad);
        }
    }

    // ---------------- the reference's own gradient ------------------------------
    // Restates compute_forward with yn_reconstruct (boundary rings of vx / vz
    // saved before every step, final wavefield saved at the top of step nt,
    // module_boundary_saving.f90:52-153) and compute_adjoint
    // (submodule_fwi_gradient.f90:31-199): source-wavefield reconstruction and
    // adjoint propagation both by update_wavefield(-dt), adjoint-source
    // injection, and the imaging condition of compute_gradient (:201-269) every
    // cc steps, for t = nt down to hnt. Rings are kept in memory instead of a
    // direct-access file. Output: grad_vp, grad_rho on the model cells.
    void ref_gradient_shot(const owl_shot& sh, const T* adj, int hnt, int cc, T* gvp, T* grho) const {
        const int P = pml;
        Ac2dState<T> s;
        s.init(lo_x, hi_x, lo_z, hi_z);
        // ring extents (prepare_boundary_saving)
        const int xb1 = 1 - R + 1, xb2 = 1, xe1 = nx + 1, xe2 = nx + R, xz0 = 1 - R, xz1 = nz + R;
        const int zx0 = 1 - R, zx1 = nx + R, zb1 = 1 - R + 1, zb2 = 1, ze1 = nz + 1, ze2 = nz + R;
        auto save = [&](std::vector<T>& r) {
            r.clear();
            for (int j = xz0; j <= xz1; ++j) for (int i = xb1; i <= xb2; ++i) r.push_back(s.vx(i, j));
            for (int j = xz0; j <= xz1; ++j) for (int i = xe1; i <= xe2; ++i) r.push_back(s.vx(i, j));
            for (int j = zb1; j <= zb2; ++j) for (int i = zx0; i <= zx1; ++i) r.push_back(s.vz(i, j));
            for (int j = ze1; j <= ze2; ++j) for (int i = zx0; i <= zx1; ++i) r.push_back(s.vz(i, j));
        };
        auto inject = [&](const std::vector<T>& r, Ac2dState<T>& d) {
            size_t q = 0;
            for (int j = xz0; j <= xz1; ++j) for (int i = xb1; i <= xb2; ++i) d.vx(i, j) = r[q++];
            for (int j = xz0; j <= xz1; ++j) for (int i = xe1; i <= xe2; ++i) d.vx(i, j) = r[q++];
            for (int j = zb1; j <= zb2; ++j) for (int i = zx0; i <= zx1; ++i) d.vz(i, j) = r[q++];
            for (int j = ze1; j <= ze2; ++j) for (int i = zx0; i <= zx1; ++i) d.vz(i, j) = r[q++];
        };
        std::vector<std::vector<T>> rings(nt + 1);
        Ac2dState<T> fin;
        std::vector<T> seis((size_t)sh.nrec * nt, T(0));
        for (int t = 1; t <= nt; ++t) {
            save(rings[t]);
            if (t == nt) fin = s;
            sample(t, sh, s, seis.data());
            update(dt, s, nullptr);
            add_source(t, sh, s);
        }
        // adjoint
        Ac2dState<T> f, a;
        f.init(lo_x, hi_x, lo_z, hi_z);
        a.init(lo_x, hi_x, lo_z, hi_z);
        Arr2<T> pp(lo_x, hi_x, lo_z, hi_z), pvx(lo_x, hi_x, lo_z, hi_z), pvz(lo_x, hi_x, lo_z, hi_z);
        Arr2<T> gv(1, nx, 1, nz), gr(1, nx, 1, nz);
        for (int t = nt; t >= hnt; --t) {
            pp = f.p; pvx = f.vx; pvz = f.vz;
            if (t == nt) { f.p = fin.p; f.vx = fin.vx; f.vz = fin.vz; }
            inject(rings[t], f);
            update(-dt, f, nullptr);
            update(-dt, a, nullptr);
            for (int r = 0; r < sh.nrec; ++r) {
                const owl_receiver& q = sh.rec[r];
                if (q.weight == 0.f) continue;
                T rv = adj[(size_t)r * nt + (t - 1)];
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx)
                        a.p(q.gx + irx, q.gz + irz) = a.p(q.gx + irx, q.gz + irz) +
                            rv * T(q.interp_ix[irx + 4]) * T(q.interp_iz[irz + 4]) * T(q.weight);
            }
            if (t % cc == 0) {
#pragma omp parallel for collapse(2) schedule(static)
                for (int j = 1; j <= nz; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        T sp = f.p(i, j) - pp(i, j);
                        gv(i, j) = gv(i, j) - sp * a.p(i, j) / (rho(i, j) * vp(i, j) * vp(i, j) * vp(i, j));
                        T sx = (f.vx(i, j) + f.vx(i + 1, j)) - (pvx(i, j) + pvx(i + 1, j));
                        T rx = a.vx(i, j) + a.vx(i + 1, j);
                        T sz = (f.vz(i, j) + f.vz(i, j + 1)) - (pvz(i, j) + pvz(i, j + 1));
                        T rz = a.vz(i, j) + a.vz(i, j + 1);
                        gr(i, j) = gr(i, j) + sx * rx + sz * rz;
                    }
            }
        }
        for (int i = 1; i <= nx; ++i)
            for (int j = 1; j <= nz; ++j) {
                gvp[(size_t)(i - 1) * nz + (j - 1)] += gv(i, j);
                grho[(size_t)(i - 1) * nz + (j - 1)] += gr(i, j);
            }
    }

    // fold the padded-grid gradient onto the model cells (adjoint of pad_array's
    // edge replication) and write (nz,nx) z-fastest.
    void fold(const Arr2<T>& gp, T* out) const {
        std::fill(out, out + (size_t)nx * nz, T(0));
        for (int j = gp.j0; j <= gp.j1; ++j)
            for (int i = gp.i0; i <= gp.i1; ++i) {
                int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nz);
                out[(size_t)(ii - 1) * nz + (jj - 1)] += gp(i, j);
            }
    }
};

}  // namespace oracle

// ---------------------------------------------------------------------------
// C entry points used by the Python test harness (ctypes)
// ---------------------------------------------------------------------------
using namespace oracle;

template <typename T>
static int fwd_impl(const owl_ssg_desc* d, const T* vp, const T* rho, int nshots, const owl_shot* shots, T* seis) {
    try {
        Ac2d<T> m(*d, vp, rho);
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

extern "C" int oracle_ac2d_forward_f32(const owl_ssg_desc* d, const float* vp, const float* rho, int nshots,
                                       const owl_shot* shots, float* seis) {
    return fwd_impl<float>(d, vp, rho, nshots, shots, seis);
}

extern "C" int oracle_ac2d_forward_f64(const owl_ssg_desc* d, const double* vp, const double* rho, int nshots,
                                       const owl_shot* shots, double* seis) {
    return fwd_impl<double>(d, vp, rho, nshots, shots, seis);
}

// complex-step Jacobian-vector product: seis_jvp = d seis / d m . (dvp, drho),
// computed as Im F(m + i h dm) / h with h = 1e-30.
extern "C" int oracle_ac2d_jvp_c128(const owl_ssg_desc* d, const double* vp, const double* rho, const double* dvp,
                                    const double* drho, int nshots, const owl_shot* shots, double* seis,
                                    double* seis_jvp) {
    typedef std::complex<double> C;
    const double h = 1e-30;
    size_t n = (size_t)d->nx * d->nz;
    std::vector<C> cvp(n), crho(n);
    for (size_t i = 0; i < n; ++i) {
        cvp[i] = C(vp[i], h * dvp[i]);
        crho[i] = C(rho[i], h * drho[i]);
    }
    size_t ns = 0;
    for (int s = 0; s < nshots; ++s) ns += (size_t)shots[s].nrec * d->nt;
    std::vector<C> out(ns);
    int rc = fwd_impl<C>(d, cvp.data(), crho.data(), nshots, shots, out.data());
    for (size_t i = 0; i < ns; ++i) {
        if (seis) seis[i] = out[i].real();
        seis_jvp[i] = out[i].imag() / h;
    }
    return rc;
}

// exact gradient (T = double or float). adj_kind as in owl_ssg_gradient.
template <typename T>
static int grad_impl(const owl_ssg_desc* d, const T* vp, const T* rho, int nshots, const owl_shot* shots,
                     const T* data, int adj_kind, int k, double* misfit, T* grad, T* stf_grad) {
    try {
        Ac2d<T> m(*d, vp, rho);
        typename Ac2d<T>::Grad g;
        g.gvp.init(-m.pml, m.nx + m.pml + 1, -m.pml, m.nz + m.pml + 1);
        g.grho.init(-m.pml, m.nx + m.pml + 1, -m.pml, m.nz + m.pml + 1);
        size_t off = 0, soff = 0;
        for (int s = 0; s < nshots; ++s) {
            const owl_shot& sh = shots[s];
            size_t n = (size_t)sh.nrec * d->nt;
            std::vector<T> res(n, T(0));
            if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
                std::vector<T> syn(n);
                m.forward_shot(sh, syn.data(), nullptr, 1 << 30);
                double mf = 0;
                for (int r = 0; r < sh.nrec; ++r) {
                    if (sh.rec[r].weight == 0.f) continue;
                    for (int t = 0; t < d->nt; ++t) {
                        size_t q = (size_t)r * d->nt + t;
                        res[q] = syn[q] - data[off + q];
                        double dd = re(data[off + q]) - re(syn[q]);
                        mf += dd * dd;
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
        size_t nm = (size_t)d->nx * d->nz;
        m.fold(g.gvp, grad);
        m.fold(g.grho, grad + nm);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}

extern "C" int oracle_ac2d_gradient_f64(const owl_ssg_desc* d, const double* vp, const double* rho, int nshots,
                                        const owl_shot* shots, const double* data, int adj_kind, int k,
                                        double* misfit, double* grad, double* stf_grad) {
    return grad_impl<double>(d, vp, rho, nshots, shots, data, adj_kind, k, misfit, grad, stf_grad);
}

extern "C" int oracle_ac2d_gradient_f32(const owl_ssg_desc* d, const float* vp, const float* rho, int nshots,
                                        const owl_shot* shots, const float* data, int adj_kind, int k,
                                        double* misfit, float* grad, float* stf_grad) {
    return grad_impl<float>(d, vp, rho, nshots, shots, data, adj_kind, k, misfit, grad, stf_grad);
}

// the reference's own gradient (time-reversed -dt propagation), summed over shots.
// hnt: per shot, the last reverse step (prepare_stf's hnt of the shot's first source);
// cc: cc_step_interval. adj: adjoint sources, same layout as seismograms.
extern "C" int oracle_ac2d_ref_gradient_f32(const owl_ssg_desc* d, const float* vp, const float* rho, int nshots,
                                            const owl_shot* shots, const float* adj, const int* hnt, int cc,
                                            float* grad) {
    try {
        Ac2d<float> m(*d, vp, rho);
        size_t nm = (size_t)d->nx * d->nz, off = 0;
        std::fill(grad, grad + 2 * nm, 0.f);
        for (int s = 0; s < nshots; ++s) {
            m.ref_gradient_shot(shots[s], adj + off, hnt[s], cc, grad, grad + nm);
            off += (size_t)shots[s].nrec * d->nt;
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
}
