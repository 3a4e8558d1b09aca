// ac2d.cu -- 2D isotropic acoustic SSG solver for B200 (sm_100a).
//
// Forward (replaces update_wavefield / add_source / receiver sampling,
// src/solver/acoustic_iso_2d/module_wavefield.f90:40-263 and
// submodule_forward_modeling.f90:48-117) and the exact discrete adjoint with
// every-k-step checkpoints (replaces compute_adjoint / compute_gradient,
// submodule_fwi_gradient.f90:31-269, whose -dt back-propagation is not the
// transpose of the forward).
//
// Layout in HBM. A field is a (NZs x pitch) float32 plane, x fastest (the
// reference transposes to x fastest too, module_vars.f90:109); storage
// x = i + pml + R - 1 for the reference's i in [-pml-R+1, nx+pml+R], same for z.
// Forward state per shot: p, vx, vz and the four CFS-PML memory planes (touched
// only inside the PML), shot-major. Material coefficients shared by all shots:
// dtbk = dt*rho*vp^2, dtbx = dt/rho_eff_x, dtbz = dt/rho_eff_z.
//
// One time step is three launches over all shots of a batch:
//   k_ac2d_fwd_p : p -= dtbk * (dx vx + dz vz), CFS-PML memory fused
//   k_ac2d_fwd_v : vx -= dtbx * dx p ; vz -= dtbz * dz p, CFS-PML memory fused
//   point kernel : add_source(t), receivers of step t+1, step counter (ssg_base.cu)
#include <algorithm>
#include <cmath>

#include "ssg_base.cuh"

namespace owl {

__constant__ float c_fd2[8];

struct Ac2dDev {
    int nx, nz, P, R, pr, pitch;
    long long fs, sst, sad;  // field size (S buffer / G stride), state / adjoint shot strides
    int x0, x1, z1, zp0, zvx0, zvz0, fsurf;
    float idx, idz;
    int nshots, spt;
    const float *dtbk, *dtbx, *dtbz;
    const float *axi, *bxi, *axh, *bxh, *azi, *bzi, *azh, *bzh;
    float *p, *vx, *vz, *m1, *m2, *m3, *m4;
    float *Sp, *Svx, *Svz;
    long long sslot;
    int k;
    int* d_step;
    float *ap, *avx, *avz, *am1, *am2, *am3, *am4;
    float *aex, *aez, *aepx, *aepz;
    float *Gbk, *Gbx, *Gbz, *Cbk, *Cbx, *Cbz;
};

__device__ __forceinline__ bool pml_int(int x, int pr, int n) { return x < pr || x >= pr + n; }
__device__ __forceinline__ bool pml_half(int x, int pr, int n) { return x <= pr || x >= pr + n; }

// ------------------------------- forward ------------------------------------
template <int R, bool STORE>
__global__ void __launch_bounds__(512) k_ac2d_fwd_p(Ac2dDev a) {
    pdl_prologue();
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = a.zp0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const float dtbk = a.dtbk[o];
    const bool px = pml_int(x, a.pr, a.nx);
    const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const float ax = px ? a.axi[x] : 0.f, bx = px ? a.bxi[x] : 0.f;
    const float az = pz ? a.azi[z] : 0.f, bz = pz ? a.bzi[z] : 0.f;
    const bool mirror = a.fsurf && z <= a.pr + a.P;
    const long long omir = (long long)(2 * a.pr - z) * a.pitch + x;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int pt = a.pitch;
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst + o;
        const float* vx = a.vx + so;
        const float* vz = a.vz + so;
        // the cell's own values are read ahead of its stores: the arrays share
        // one allocation, so no plain read could move above a store; the
        // neighbours' fields, which this launch does not write, are read
        // through the read-only path
        const float p0 = a.p[so], m1 = px ? a.m1[so] : 0.f, m2 = pz ? a.m2[so] : 0.f;
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (__ldg(vx + k) - __ldg(vx + 1 - k));
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fd2[k - 1] * (__ldg(vz + k * pt) - __ldg(vz + (1 - k) * pt));
        float gx = a.idx * sx, gz = a.idz * sz;
        if (px) {
            float m = ax * gx + bx * m1;
            a.m1[so] = m;
            gx = gx + m;
        }
        if (pz) {
            float m = az * gz + bz * m2;
            a.m2[so] = m;
            gz = gz + m;
        }
        const float g = gx + gz;
        const float pn = p0 - dtbk * g;
        a.p[so] = pn;
        if (mirror) a.p[s * a.sst + omir] = -pn;
        if (STORE) a.Sp[slot + s * a.fs + o] = g;
    }
}

template <int R, bool STORE>
__global__ void __launch_bounds__(512) k_ac2d_fwd_v(Ac2dDev a) {
    pdl_prologue();
    const int zr0 = min(a.zvx0, a.zvz0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
    const float bxc = a.dtbx[o], bzc = a.dtbz[o];
    const bool px = pml_half(x, a.pr, a.nx);
    const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float ax = px ? a.axh[x] : 0.f, bx = px ? a.bxh[x] : 0.f;
    const float az = pz ? a.azh[z] : 0.f, bz = pz ? a.bzh[z] : 0.f;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int pt = a.pitch;
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst + o;
        const float* p = a.p + so;
        // the cell's own values are read ahead of its stores (see k_ac2d_fwd_p)
        const float vx0 = dox ? a.vx[so] : 0.f, m3 = dox && px ? a.m3[so] : 0.f;
        const float vz0 = doz ? a.vz[so] : 0.f, m4 = doz && pz ? a.m4[so] : 0.f;
        if (dox) {
            float sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (__ldg(p + k - 1) - __ldg(p - k));
            float h = a.idx * sx;
            if (px) {
                float m = ax * h + bx * m3;
                a.m3[so] = m;
                h = h + m;
            }
            a.vx[so] = vx0 - bxc * h;
            if (STORE) a.Svx[slot + s * a.fs + o] = h;
        }
        if (doz) {
            float sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fd2[k - 1] * (__ldg(p + (k - 1) * pt) - __ldg(p - k * pt));
            float h = a.idz * sz;
            if (pz) {
                float m = az * h + bz * m4;
                a.m4[so] = m;
                h = h + m;
            }
            a.vz[so] = vz0 - bzc * h;
            if (STORE) a.Svz[slot + s * a.fs + o] = h;
        }
    }
}

// ------------------------------- adjoint ------------------------------------
// The exact adjoint of step t in two stencil launches that mirror the forward:
//
//   k_ac2d_adj_p : reverse of the vx / vz updates, p^ += Dx^T e_x + Dz^T e_z,
//                  where e_x, e_z are the adjoint PML terms of the vx / vz nodes
//                  (written by k_ac2d_adj_v of the step after); then, per cell,
//                  the reverse of the p update's PML: q = -dtbk p^,
//                  e_p = q + a_i (q + psi^), psi^ <- b_i (q + psi^), stored as
//                  e_px, e_pz; Kahan sums of v^ . S_v and p^ . S_p for the
//                  coefficient gradients.
//   k_ac2d_adj_v : reverse of the p update, vx^ += Dx^T e_px, vz^ += Dz^T e_pz;
//                  then, per node, the adjoint PML terms e_x, e_z of step t-1.
//
// Every node's e is computed once by its owner and read by its neighbours in
// the next launch: no double buffering, no halo recomputation. Entries of e
// outside a field's update range stay zero.
template <int R>
__global__ void __launch_bounds__(512) k_ac2d_adj_p(Ac2dDev a) {
    pdl_prologue();
    const int zr0 = min(min(a.zvx0, a.zvz0), a.zp0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const long long o = (long long)z * a.pitch + x;
    const bool dop = z >= a.zp0, ownx = z >= a.zvx0, ownz = z >= a.zvz0;
    const bool px = pml_int(x, a.pr, a.nx);
    const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const float bk = a.dtbk[o];
    const float axi = px ? a.axi[x] : 0.f, bxi = px ? a.bxi[x] : 0.f;
    const float azi = pz ? a.azi[z] : 0.f, bzi = pz ? a.bzi[z] : 0.f;
    const bool mirror = a.fsurf && z <= a.pr + a.P;
    const long long om = (long long)(2 * a.pr - z) * a.pitch + x;
    const int pt = a.pitch;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    float gbk = 0.f, gbx = 0.f, gbz = 0.f;
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad + o, ss = slot + s * a.fs + o;
        // every read of the shot's cell is issued ahead of its stores: the
        // arrays share one allocation, so no plain read could move above a
        // store and each would cost its own round trip. Arrays that no thread
        // of this launch writes (the e terms of the neighbours, the stored
        // stencil terms) are read through the read-only path, which the
        // compiler may schedule freely.
        const float vx = ownx ? a.avx[sa] : 0.f, svx = ownx ? __ldg(a.Svx + ss) : 0.f;
        const float vz = ownz ? a.avz[sa] : 0.f, svz = ownz ? __ldg(a.Svz + ss) : 0.f;
        const float p0 = dop ? a.ap[sa] : 0.f, sp = dop ? __ldg(a.Sp + ss) : 0.f;
        const float m1 = dop && px ? a.am1[sa] : 0.f, m2 = dop && pz ? a.am2[sa] : 0.f;
        if (ownx) gbx += vx * svx;
        if (ownz) gbz += vz * svz;
        if (!dop) continue;
        const float* ex = a.aex + sa;
        const float* ez = a.aez + sa;
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (__ldg(ex + 1 - k) - __ldg(ex + k));
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fd2[k - 1] * (__ldg(ez + (1 - k) * pt) - __ldg(ez + k * pt));
        float dP = a.idx * sx + a.idz * sz;
        if (mirror) {
            // p(i, 2-j) = -p(i, j), j <= 0: the adjoint landing on the mirror row folds back with a minus
            const float* em = a.aez + s * a.sad + om;
            float sm = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sm = sm + c_fd2[k - 1] * (__ldg(em + (1 - k) * pt) - __ldg(em + k * pt));
            dP = dP - a.idz * sm;
        }
        const float ph = p0 + dP;
        a.ap[sa] = ph;
        gbk += ph * sp;
        const float q = -bk * ph;
        float epx = q, epz = q;
        if (px) {
            float u = q + m1;
            a.am1[sa] = bxi * u;
            epx = q + axi * u;
        }
        if (pz) {
            float u = q + m2;
            a.am2[sa] = bzi * u;
            epz = q + azi * u;
        }
        a.aepx[sa] = epx;
        a.aepz[sa] = epz;
    }
    const long long go = (long long)blockIdx.z * a.fs + o;
    float sm, c;
    if (dop) { sm = a.Gbk[go]; c = a.Cbk[go]; kahan_add(sm, c, gbk); a.Gbk[go] = sm; a.Cbk[go] = c; }
    if (ownx) { sm = a.Gbx[go]; c = a.Cbx[go]; kahan_add(sm, c, gbx); a.Gbx[go] = sm; a.Cbx[go] = c; }
    if (ownz) { sm = a.Gbz[go]; c = a.Cbz[go]; kahan_add(sm, c, gbz); a.Gbz[go] = sm; a.Cbz[go] = c; }
}

template <int R>
__global__ void __launch_bounds__(512) k_ac2d_adj_v(Ac2dDev a) {
    pdl_prologue();
    const int zr0 = min(a.zvx0, a.zvz0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
    const bool px = pml_half(x, a.pr, a.nx);
    const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float bxc = a.dtbx[o], bzc = a.dtbz[o];
    const float axh = px ? a.axh[x] : 0.f, bxh = px ? a.bxh[x] : 0.f;
    const float azh = pz ? a.azh[z] : 0.f, bzh = pz ? a.bzh[z] : 0.f;
    const int pt = a.pitch;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad + o;
        // the shot's cell values are read ahead of its stores (see k_ac2d_adj_p)
        const float vx = dox ? a.avx[sa] : 0.f, m3 = dox && px ? a.am3[sa] : 0.f;
        const float vz = doz ? a.avz[sa] : 0.f, m4 = doz && pz ? a.am4[sa] : 0.f;
        if (dox) {
            const float* ep = a.aepx + sa;
            float sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (__ldg(ep - k) - __ldg(ep + k - 1));
            const float xh = vx + a.idx * sx;
            a.avx[sa] = xh;
            const float q = -bxc * xh;
            float e = q;
            if (px) {
                float u = q + m3;
                a.am3[sa] = bxh * u;
                e = q + axh * u;
            }
            a.aex[sa] = e;
        }
        if (doz) {
            const float* ep = a.aepz + sa;
            float sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fd2[k - 1] * (__ldg(ep - k * pt) - __ldg(ep + (k - 1) * pt));
            const float zh = vz + a.idz * sz;
            a.avz[sa] = zh;
            const float q = -bzc * zh;
            float e = q;
            if (pz) {
                float u = q + m4;
                a.am4[sa] = bzh * u;
                e = q + azh * u;
            }
            a.aez[sa] = e;
        }
    }
}

// ------------------------- FP64 chain rule ---------------------------------
// Gradient w.r.t. vp and rho on the padded model grid [-P, n+P+1] from the
// time-summed coefficient gradients G = sum v^ . S (Kahan: value = G - C):
//   p' = p - dtbk S_p, dtbk = dt rho vp^2
//   v' = v - dtb S_v, dtb = dt / (0.5 (rho[m] + rho[m-1]))
__global__ void k_ac2d_chain(Ac2dDev a, int ngroups, const float* __restrict__ vpp, const float* __restrict__ rhop,
                             double dt, double* __restrict__ gvp, double* __restrict__ grho, int nxq, int nzq) {
    int ix = blockIdx.x * blockDim.x + threadIdx.x, iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= nxq || iz >= nzq) return;
    int x = a.R - 1 + ix, z = a.R - 1 + iz;
    const long long o = (long long)z * a.pitch + x;
    auto sumG = [&](const float* G, const float* C, long long oo) {
        double v = 0;
        for (int g = 0; g < ngroups; ++g) v += (double)G[g * a.fs + oo] - (double)C[g * a.fs + oo];
        return v;
    };
    double vp = vpp[o], rho = rhop[o];
    double dv = 0, dr = 0;
    if (x >= a.x0 && x < a.x1 && z >= a.zp0 && z < a.z1) {
        double gbk = sumG(a.Gbk, a.Cbk, o);
        dv += -gbk * dt * 2.0 * rho * vp;
        dr += -gbk * dt * vp * vp;
    }
    for (int d = 0; d <= 1; ++d) {
        int m = x + d;
        if (m >= a.x0 && m < a.x1 && z >= a.zvx0 && z < a.z1) {
            long long om = (long long)z * a.pitch + m;
            double re = 0.5 * ((double)rhop[om] + (double)rhop[om - 1]);
            dr += sumG(a.Gbx, a.Cbx, om) * 0.5 * dt / (re * re);
        }
        int mz = z + d;
        if (x >= a.x0 && x < a.x1 && mz >= a.zvz0 && mz < a.z1) {
            long long om = (long long)mz * a.pitch + x;
            double re = 0.5 * ((double)rhop[om] + (double)rhop[om - a.pitch]);
            dr += sumG(a.Gbz, a.Cbz, om) * 0.5 * dt / (re * re);
        }
    }
    gvp[(size_t)iz * nxq + ix] += dv;
    grho[(size_t)iz * nxq + ix] += dr;
}

// ============================================================================
// host engine
// ============================================================================
struct Ac2dEngine : SsgBase {
    float idx, idz;
    DevBuf<float> dtbk, dtbx, dtbz, vpp, rhop, pml_x, pml_z;

    explicit Ac2dEngine(const owl_ssg_desc& d) : SsgBase(d, 2) {
        idx = (float)(1.0 / (double)d.dx);
        idz = (float)(1.0 / (double)d.dz);
        OWL_CUDA(cudaMemcpyToSymbol(c_fd2, fd_coefs(R), sizeof(float) * R));
        sst = 7 * fs;   // p, vx, vz, psi(dx vx), psi(dz vz), psi(dx p), psi(dz p)
        sad = 11 * fs;  // p^, vx^, vz^, 4 memory adjoints, e_x, e_z, e_px, e_pz
        nS = 3;
        ngrad = 3;
        nparam = 2;
        ncomp = 1;
        for (int f = 0; f < 7; ++f) st_segments.push_back({f * fs, fs});
    }

    float* st_field(int f) const override { return f < 3 ? st.p + f * fs : nullptr; }
    float* ad_field(int f) const override { return f < 3 ? ad.p + f * fs : nullptr; }
    int rho_param() const override { return 1; }

    void set_model(int nparam_, const float* const* f) override {
        OWL_CHECK(nparam_ == 2 && f && f[0] && f[1], OWL_ERR_INVALID, "acoustic model needs vp and rho");
        const float* vp = f[0];
        const float* rho = f[1];
        std::vector<float> hvp(fs, 0.f), hrho(fs, 0.f), hbk(fs, 0.f), hbx(fs, 0.f), hbz(fs, 0.f);
        float maxv = -1e30f;
        for (int j = -P; j <= nz + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nz);
                float v = vp[(size_t)(ii - 1) * nz + (jj - 1)], r = rho[(size_t)(ii - 1) * nz + (jj - 1)];
                OWL_CHECK(std::isfinite(v) && std::isfinite(r) && v > 0 && r > 0, OWL_ERR_INVALID,
                          "vp and rho must be finite and positive");
                long long o = soff(i, 1, j);
                hvp[o] = v; hrho[o] = r;
                hbk[o] = dt * (r * v * v);
                maxv = std::max(maxv, v);
            }
        for (int j = -P + 1; j <= nz + P; ++j)
            for (int m = -P + 1; m <= nx + P; ++m) {
                float re = 0.5f * (hrho[soff(m, 1, j)] + hrho[soff(m - 1, 1, j)]);
                hbx[soff(m, 1, j)] = dt / re;
                float rz = 0.5f * (hrho[soff(m, 1, j)] + hrho[soff(m, 1, j - 1)]);
                hbz[soff(m, 1, j)] = dt / rz;
            }
        // stability (module_vars.f90:121-125)
        const float* c = fd_coefs(R);
        float temp = 0.f;
        for (int k = 0; k < R; ++k) temp += std::fabs(c[k]);
        dt_stable_ = 1.0f / (temp * maxv * std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (desc.dz * desc.dz)));
        if (dt > dt_stable_ && !desc.allow_dt_adjust)
            throw OwlError(OWL_ERR_UNSTABLE, "dt = " + std::to_string(dt) + " exceeds the stable dt " +
                                                 std::to_string(dt_stable_));
        // CFS-PML (module_cfspml.f90:68-93)
        float pmlvp = -1e30f;
        for (int j = 1; j <= nz; ++j) pmlvp = std::max({pmlvp, hvp[soff(1, 1, j)], hvp[soff(nx, 1, j)]});
        for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, hvp[soff(i, 1, 1)], hvp[soff(i, 1, nz)]});
        float alphamax = (float)(1.0 * (double)desc.f0_max * 3.14159265358979323846);
        Pml1DHost hx = build_pml_1d(nx, P, R, pitch, desc.dx, dt, pmlvp, alphamax);
        Pml1DHost hz = build_pml_1d(nz, P, R, NZs, desc.dz, dt, pmlvp, alphamax);
        std::vector<float> px(4 * pitch), pz(4 * NZs);
        for (int q = 0; q < 4; ++q) {
            const std::vector<float>& a = q == 0 ? hx.ai : q == 1 ? hx.bi : q == 2 ? hx.ah : hx.bh;
            const std::vector<float>& b = q == 0 ? hz.ai : q == 1 ? hz.bi : q == 2 ? hz.ah : hz.bh;
            std::copy(a.begin(), a.end(), px.begin() + q * pitch);
            std::copy(b.begin(), b.end(), pz.begin() + q * NZs);
        }
        dtbk.upload(hbk.data(), fs, stream);
        dtbx.upload(hbx.data(), fs, stream);
        dtbz.upload(hbz.data(), fs, stream);
        vpp.upload(hvp.data(), fs, stream);
        rhop.upload(hrho.data(), fs, stream);
        pml_x.upload(px.data(), px.size(), stream);
        pml_z.upload(pz.data(), pz.size(), stream);
        OWL_CUDA(cudaStreamSynchronize(stream));
        h_rhop = std::move(hrho);
        model_set = true;
        invalidate_graphs();
    }

    // ---- sources / receivers (module_wavefield.f90:192-263, submodule_forward_modeling.f90:58-79)
    int src_ncomp(const owl_source& q) const override {
        OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION || q.mechanism == OWL_SRC_FORCE, OWL_ERR_UNSUPPORTED,
                  "acoustic media support explosion and force sources");
        return q.mechanism == OWL_SRC_FORCE ? 2 : 1;
    }
    void src_taps(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rc, float& rv) const override {
        const bool fsf = desc.free_surface != 0;
        if (q.mechanism == OWL_SRC_FORCE) {
            const int ci = comp == 0 ? q.hx : q.gx, ck = comp == 0 ? q.gz : q.hz;
            OWL_CHECK(in_wavefield(ci, 1, ck), OWL_ERR_INVALID, "force source outside the grid");
            rv = h_rhop[soff(ci, 1, ck)];
            rc = pad_index(ci, 1, ck);
        }
        for (int irz = -4; irz <= 4; ++irz)
            for (int irx = -4; irx <= 4; ++irx) {
                TapPt t;
                if (q.mechanism == OWL_SRC_EXPLOSION) {
                    t = TapPt{0, q.gx + irx, 1, q.gz + irz, q.interp_ix[irx + 4] * q.interp_iz[irz + 4]};
                } else if (comp == 0) {
                    t = TapPt{1, q.hx + irx, 1, q.gz + irz,
                              std::sin(q.polar) / rv * q.interp_hx[irx + 4] * q.interp_iz[irz + 4]};
                } else {
                    t = TapPt{2, q.gx + irx, 1, q.hz + irz,
                              std::cos(q.polar) / rv * q.interp_ix[irx + 4] * q.interp_hz[irz + 4]};
                }
                if (fsf && t.k < 2) continue;
                taps.push_back(t);
            }
    }
    void rec_taps(const owl_receiver& q, int, std::vector<TapPt>& taps) const override {
        for (int irz = -4; irz <= 4; ++irz)
            for (int irx = -4; irx <= 4; ++irx)
                taps.push_back(TapPt{0, q.gx + irx, 1, q.gz + irz, q.interp_ix[irx + 4] * q.interp_iz[irz + 4] * q.weight});
    }
    // with a free surface, p(i, 2-j) = -p(i, j) for j <= 0 and p(i, 1) = 0
    void scatter_map(const TapPt& t, std::vector<TapPt>& out) const override {
        if (!desc.free_surface) { out.push_back(t); return; }
        if (t.k <= 0) out.push_back(TapPt{t.field, t.i, t.j, 2 - t.k, -t.w});
        else if (t.k >= 2) out.push_back(t);
    }

    Ac2dDev dev(int S) const {
        Ac2dDev a{};
        a.nx = nx; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch;
        a.fs = fs; a.sst = sst; a.sad = sad;
        a.x0 = R; a.x1 = R + NXp; a.z1 = R + NZp;
        a.fsurf = desc.free_surface != 0;
        a.zp0 = a.fsurf ? pr + 1 : R;
        a.zvx0 = a.fsurf ? pr : R;
        a.zvz0 = a.fsurf ? pr + 1 : R;
        a.idx = idx; a.idz = idz;
        a.nshots = S;
        a.dtbk = dtbk.p; a.dtbx = dtbx.p; a.dtbz = dtbz.p;
        a.axi = pml_x.p; a.bxi = pml_x.p + pitch; a.axh = pml_x.p + 2 * pitch; a.bxh = pml_x.p + 3 * pitch;
        a.azi = pml_z.p; a.bzi = pml_z.p + NZs; a.azh = pml_z.p + 2 * NZs; a.bzh = pml_z.p + 3 * NZs;
        a.p = st.p; a.vx = st.p + fs; a.vz = st.p + 2 * fs;
        a.m1 = st.p + 3 * fs; a.m2 = st.p + 4 * fs; a.m3 = st.p + 5 * fs; a.m4 = st.p + 6 * fs;
        a.k = std::max(1, cur_k);
        a.d_step = ctr.p;
        const long long F = (long long)S * fs;
        if (Sbuf.p && Sbuf.n >= (size_t)3 * a.k * F) {
            a.sslot = F;
            a.Sp = Sbuf.p; a.Svx = Sbuf.p + (long long)a.k * F; a.Svz = Sbuf.p + 2LL * a.k * F;
        }
        if (ad.p && ad.n >= (size_t)sad * S) {
            a.ap = ad.p; a.avx = ad.p + fs; a.avz = ad.p + 2 * fs;
            a.am1 = ad.p + 3 * fs; a.am2 = ad.p + 4 * fs; a.am3 = ad.p + 5 * fs; a.am4 = ad.p + 6 * fs;
            a.aex = ad.p + 7 * fs; a.aez = ad.p + 8 * fs; a.aepx = ad.p + 9 * fs; a.aepz = ad.p + 10 * fs;
        }
        if (G.p) {
            const long long gg = (long long)((S + spt_a - 1) / spt_a) * fs;
            a.Gbk = G.p; a.Gbx = G.p + gg; a.Gbz = G.p + 2 * gg;
            a.Cbk = G.p + 3 * gg; a.Cbx = G.p + 4 * gg; a.Cbz = G.p + 5 * gg;
        }
        return a;
    }

    template <int RR>
    void launch_r(int id, int S, bool store) {
        Ac2dDev a = dev(S);
        const int rows_p = a.z1 - a.zp0, rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        const int rows_a = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
        if (id == OWL_K_FWD_P || id == OWL_K_FWD_V) {
            a.spt = spt_f;
            dim3 b(tile_x, tz_f);
            if (id == OWL_K_FWD_P) {
                if (store) launch_pdl(k_ac2d_fwd_p<RR, true>, grid_for(rows_p, S, spt_f, tz_f), b, 0, stream, a);
                else launch_pdl(k_ac2d_fwd_p<RR, false>, grid_for(rows_p, S, spt_f, tz_f), b, 0, stream, a);
            } else {
                if (store) launch_pdl(k_ac2d_fwd_v<RR, true>, grid_for(rows_v, S, spt_f, tz_f), b, 0, stream, a);
                else launch_pdl(k_ac2d_fwd_v<RR, false>, grid_for(rows_v, S, spt_f, tz_f), b, 0, stream, a);
            }
        } else {
            a.spt = spt_a;
            dim3 b(tile_x, tz_a);
            if (id == OWL_K_ADJ_P) launch_pdl(k_ac2d_adj_p<RR>, grid_for(rows_a, S, spt_a, tz_a), b, 0, stream, a);
            else launch_pdl(k_ac2d_adj_v<RR>, grid_for(rows_v, S, spt_a, tz_a), b, 0, stream, a);
        }
    }
    void launch_kernel(int id, int S, bool store) override {
        if (R == 4) launch_r<4>(id, S, store);
        else launch_r<8>(id, S, store);
    }

    // compulsory bytes of one launch (each state field read / written once per
    // shot, materials once per launch, PML memory only inside the PML, gradient
    // accumulators once per shot group)
    double alg_bytes(int id, int S, int groups) const override {
        const double cells = (double)NXp * NZp;
        double npx_i = 0, npz_i = 0, npx_h = 0, npz_h = 0;
        const bool fsf = desc.free_surface != 0;
        for (int x = R; x < R + NXp; ++x) {
            npx_i += (x < pr || x >= pr + nx) ? NZp : 0;
            npx_h += (x <= pr || x >= pr + nx) ? NZp : 0;
        }
        for (int z = R; z < R + NZp; ++z) {
            npz_i += ((!fsf && z < pr) || z >= pr + nz) ? NXp : 0;
            npz_h += ((!fsf && z <= pr) || z >= pr + nz) ? NXp : 0;
        }
        switch (id) {
            case OWL_K_FWD_P: return S * (cells * 16.0 + (npx_i + npz_i) * 8.0) + cells * 4.0;
            case OWL_K_FWD_V: return S * (cells * 20.0 + (npx_h + npz_h) * 8.0) + cells * 8.0;
            case OWL_K_ADJ_P: return S * (cells * 44.0 + (npx_i + npz_i) * 8.0) + cells * 4.0 + groups * cells * 48.0;
            case OWL_K_ADJ_V: return S * (cells * 32.0 + (npx_h + npz_h) * 8.0) + cells * 8.0;
        }
        return 0;
    }

    void chain_rule(int S, int groups) override {
        Ac2dDev a = dev(S);
        dim3 b(32, 8), g((nxq() + 31) / 32, (nzq() + 7) / 8);
        k_ac2d_chain<<<g, b, 0, stream>>>(a, groups, vpp.p, rhop.p, (double)dt, gpad.p, gpad.p + npad(), nxq(), nzq());
        OWL_LAUNCH_CHECK();
        launches++;
    }
};

Engine* make_ac2d_engine(const owl_ssg_desc& d) { return new Ac2dEngine(d); }

}  // namespace owl
