// ac2d.cu -- 2D isotropic acoustic SSG solver for B200 (sm_100a).
//
// Forward (replaces update_wavefield / add_source / receiver sampling,
// src/solver/acoustic_iso_2d/module_wavefield.f90:40-263 and
// submodule_forward_modeling.f90:48-117) and the exact discrete adjoint with
// every-k-step checkpoints (replaces compute_adjoint / compute_gradient,
// submodule_fwi_gradient.f90:31-269, whose -dt back-propagation is not the
// transpose of the forward).
//
// Layout in HBM. Every field of one shot is a (NZs x pitch) float32 plane,
// x fastest (the reference transposes to x fastest too, module_vars.f90:109):
//   storage x = i + pml + R - 1 for the reference's index i in
//   [-pml-R+1, nx+pml+R]; same for z. pitch = NXs rounded up to 32 floats.
// Shots of a batch are stacked: field[s][z][x]. The material coefficients
// dtbk = dt*rho*vp^2, dtbx = dt/rho_eff_x, dtbz = dt/rho_eff_z are shared by
// all shots. PML memory variables are full planes touched only inside the PML.
//
// One time step t is three launches (all shots of a batch in each):
//   k_fwd_p   : p -= dtbk * (dx vx + dz vz), CFS-PML memory fused
//   k_fwd_v   : vx -= dtbx * dx p ; vz -= dtbz * dz p, CFS-PML memory fused
//   k_point_fwd: add_source(t) then sample receivers for step t+1, one CTA per
//                shot; its last CTA advances the device step counter so the
//                same captured CUDA graph serves every segment of k steps.
#include <algorithm>
#include <cmath>
#include <array>
#include <map>

#include "engine.cuh"

namespace owl {

__constant__ float c_fd[8];

struct Ac2dDev {
    int nx, nz, P, R, pr, pitch;
    long long fs;
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
        const long long so = s * a.fs + o;
        const float* vx = a.vx + so;
        const float* vz = a.vz + so;
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fd[k - 1] * (vx[k] - vx[1 - k]);
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fd[k - 1] * (vz[k * pt] - vz[(1 - k) * pt]);
        float gx = a.idx * sx, gz = a.idz * sz;
        if (px) {
            float m = ax * gx + bx * a.m1[so];
            a.m1[so] = m;
            gx = gx + m;
        }
        if (pz) {
            float m = az * gz + bz * a.m2[so];
            a.m2[so] = m;
            gz = gz + m;
        }
        const float g = gx + gz;
        const float pn = a.p[so] - dtbk * g;
        a.p[so] = pn;
        if (mirror) a.p[s * a.fs + omir] = -pn;
        if (STORE) a.Sp[slot + so] = g;
    }
}

template <int R, bool STORE>
__global__ void __launch_bounds__(512) k_ac2d_fwd_v(Ac2dDev a) {
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
        const long long so = s * a.fs + o;
        const float* p = a.p + so;
        if (dox) {
            float sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fd[k - 1] * (p[k - 1] - p[-k]);
            float h = a.idx * sx;
            if (px) {
                float m = ax * h + bx * a.m3[so];
                a.m3[so] = m;
                h = h + m;
            }
            a.vx[so] = a.vx[so] - bxc * h;
            if (STORE) a.Svx[slot + so] = h;
        }
        if (doz) {
            float sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fd[k - 1] * (p[(k - 1) * pt] - p[-k * pt]);
            float h = a.idz * sz;
            if (pz) {
                float m = az * h + bz * a.m4[so];
                a.m4[so] = m;
                h = h + m;
            }
            a.vz[so] = a.vz[so] - bzc * h;
            if (STORE) a.Svz[slot + so] = h;
        }
    }
}

// ------------------------------- adjoint ------------------------------------
// The exact adjoint of step t, in two stencil launches that mirror the forward:
//
//   k_ac2d_adj_p : reverse of the vx / vz updates, p^ += Dx^T e_x + Dz^T e_z,
//                  where e_x, e_z are the adjoint PML terms of the vx / vz nodes
//                  (arrays written by k_ac2d_adj_v of the step after); then, per
//                  cell, the reverse of the p update's PML: q = -dtbk p^,
//                  e_p = q + a_i (q + psi^), psi^ <- b_i (q + psi^), written as
//                  the arrays e_px, e_pz; Kahan sums of v^ . S_v and p^ . S_p
//                  for the coefficient gradients.
//   k_ac2d_adj_v : reverse of the p update, vx^ += Dx^T e_px, vz^ += Dz^T e_pz;
//                  then, per node, the adjoint PML terms e_x, e_z of step t-1.
//
// Every node's e is computed once by its owner and read by its neighbours in
// the next launch, so no double buffering and no halo recomputation is needed.
// Entries of e outside a field's update range stay zero.
template <int R>
__global__ void __launch_bounds__(512) k_ac2d_adj_p(Ac2dDev a) {
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
        const long long so = s * a.fs + o;
        if (ownx) gbx += a.avx[so] * a.Svx[slot + so];
        if (ownz) gbz += a.avz[so] * a.Svz[slot + so];
        if (!dop) continue;
        const float* ex = a.aex + so;
        const float* ez = a.aez + so;
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fd[k - 1] * (ex[1 - k] - ex[k]);
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fd[k - 1] * (ez[(1 - k) * pt] - ez[k * pt]);
        float dP = a.idx * sx + a.idz * sz;
        if (mirror) {
            // p(i, 2-j) = -p(i, j), j <= 0: the adjoint landing on the mirror row folds back with a minus
            const float* em = a.aez + s * a.fs + om;
            float sm = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sm = sm + c_fd[k - 1] * (em[(1 - k) * pt] - em[k * pt]);
            dP = dP - a.idz * sm;
        }
        const float ph = a.ap[so] + dP;
        a.ap[so] = ph;
        gbk += ph * a.Sp[slot + so];
        const float q = -bk * ph;
        float epx = q, epz = q;
        if (px) {
            float u = q + a.am1[so];
            a.am1[so] = bxi * u;
            epx = q + axi * u;
        }
        if (pz) {
            float u = q + a.am2[so];
            a.am2[so] = bzi * u;
            epz = q + azi * u;
        }
        a.aepx[so] = epx;
        a.aepz[so] = epz;
    }
    const long long go = (long long)blockIdx.z * a.fs + o;
    float sm, c;
    if (dop) { sm = a.Gbk[go]; c = a.Cbk[go]; kahan_add(sm, c, gbk); a.Gbk[go] = sm; a.Cbk[go] = c; }
    if (ownx) { sm = a.Gbx[go]; c = a.Cbx[go]; kahan_add(sm, c, gbx); a.Gbx[go] = sm; a.Cbx[go] = c; }
    if (ownz) { sm = a.Gbz[go]; c = a.Cbz[go]; kahan_add(sm, c, gbz); a.Gbz[go] = sm; a.Cbz[go] = c; }
}

template <int R>
__global__ void __launch_bounds__(512) k_ac2d_adj_v(Ac2dDev a) {
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
        const long long so = s * a.fs + o;
        if (dox) {
            const float* ep = a.aepx + so;
            float sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fd[k - 1] * (ep[-k] - ep[k - 1]);
            const float xh = a.avx[so] + a.idx * sx;
            a.avx[so] = xh;
            const float q = -bxc * xh;
            float e = q;
            if (px) {
                float u = q + a.am3[so];
                a.am3[so] = bxh * u;
                e = q + axh * u;
            }
            a.aex[so] = e;
        }
        if (doz) {
            const float* ep = a.aepz + so;
            float sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fd[k - 1] * (ep[-k * pt] - ep[(k - 1) * pt]);
            const float zh = a.avz[so] + a.idz * sz;
            a.avz[so] = zh;
            const float q = -bzc * zh;
            float e = q;
            if (pz) {
                float u = q + a.am4[so];
                a.am4[so] = bzh * u;
                e = q + azh * u;
            }
            a.aez[so] = e;
        }
    }
}

// ------------------------------ point operators ----------------------------
struct PointDev {
    float* fld[3];
    long long fs;
    int nt, rtot;
    CSRView inj;
    const int* inj_shot_ptr;
    const float* amp;
    CSRView smp;
    const int* rec_shot_ptr;
    float* rec;
    CSRView sct;
    const int* sct_shot_ptr;
    const float* res;
    float* src_adj;
    int* d_step;
    int* d_done;
};

enum { PT_INJECT = 1, PT_SAMPLE = 2, PT_TICK = 4 };

__global__ void k_point_fwd(PointDev a, int mode) {
    const int s = blockIdx.x;
    const int cur = *a.d_step;
    const int t = cur + 1;
    if (mode & PT_INJECT) {
        for (int it = a.inj_shot_ptr[s]; it < a.inj_shot_ptr[s + 1]; ++it) {
            const float A = a.amp[(size_t)it * a.nt + (t - 1)];
            if (A != 0.f) {
                for (int j = a.inj.ptr[it] + threadIdx.x; j < a.inj.ptr[it + 1]; j += blockDim.x) {
                    float* f = a.fld[a.inj.field[j]] + s * a.fs + a.inj.off[j];
                    *f = *f + A * a.inj.w[j];
                }
            }
            __syncthreads();
        }
    }
    if (mode & PT_SAMPLE) {
        const int tr = (mode & PT_INJECT) ? t + 1 : t;
        if (tr <= a.nt) {
            for (int r = a.rec_shot_ptr[s] + threadIdx.x; r < a.rec_shot_ptr[s + 1]; r += blockDim.x) {
                float acc = 0.f;
                for (int j = a.smp.ptr[r]; j < a.smp.ptr[r + 1]; ++j)
                    acc = acc + a.fld[a.smp.field[j]][s * a.fs + a.smp.off[j]] * a.smp.w[j];
                a.rec[(size_t)(tr - 1) * a.rtot + r] = acc;
            }
        }
    }
    if (mode & PT_TICK) tick_last_block(a.d_step, a.d_done, 1);
}

__global__ void k_point_adj(PointDev a) {
    const int s = blockIdx.x;
    const int t = *a.d_step;
    // adjoint of the sampling of step t (which read p_{t-1})
    for (int it = a.sct_shot_ptr[s] + threadIdx.x; it < a.sct_shot_ptr[s + 1]; it += blockDim.x) {
        float acc = 0.f;
        const int j0 = a.sct.ptr[it], j1 = a.sct.ptr[it + 1];
        for (int j = j0; j < j1; ++j) acc = acc + a.res[(size_t)(t - 1) * a.rtot + a.sct.item[j]] * a.sct.w[j];
        float* f = a.fld[a.sct.field[j0]] + s * a.fs + a.sct.off[j0];
        *f = *f + acc;
    }
    __syncthreads();
    // source-side adjoint at step t-1: taps . lambda_{t-1}
    if (a.src_adj && t - 1 >= 1) {
        for (int it = a.inj_shot_ptr[s] + threadIdx.x; it < a.inj_shot_ptr[s + 1]; it += blockDim.x) {
            float acc = 0.f;
            for (int j = a.inj.ptr[it]; j < a.inj.ptr[it + 1]; ++j)
                acc = acc + a.fld[a.inj.field[j]][s * a.fs + a.inj.off[j]] * a.inj.w[j];
            a.src_adj[(size_t)it * a.nt + (t - 2)] = acc;
        }
    }
    tick_last_block(a.d_step, a.d_done, -1);
}

// ------------------------- FP64 chain rule + fold ---------------------------
// Gradient w.r.t. vp and rho on the padded model grid from the time-summed
// coefficient gradients, then folded onto the model cells (adjoint of the edge
// replication of pad_array, module_vars.f90:113-115).
__global__ void k_ac2d_chain(Ac2dDev a, int ngroups, const float* __restrict__ vpp, const float* __restrict__ rhop,
                             double dt, double* __restrict__ gvp, double* __restrict__ grho, int nxq, int nzq) {
    // padded grid [-P, n+P+1] -> storage [R-1, R+NXp]
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
    // vx nodes m = x (uses rho[x], rho[x-1]) and m = x+1 (uses rho[x+1], rho[x])
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

__global__ void k_add_points_f64(double* g, const int* idx, const double* val, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[idx[i]] += val[i];  // sequential per index list (host merges duplicates)
}

__global__ void k_fold2d(const double* __restrict__ gp, int nxq, int nzq, int P, int nx, int nz, float* __restrict__ out) {
    // out (nz, nx) z fastest: out[(ix-1)*nz + (iz-1)]
    int iz = blockIdx.x * blockDim.x + threadIdx.x + 1, ix = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (ix > nx || iz > nz) return;
    int xa = (ix == 1) ? -P : ix, xb = (ix == nx) ? nx + P + 1 : ix;
    int za = (iz == 1) ? -P : iz, zb = (iz == nz) ? nz + P + 1 : iz;
    double acc = 0;
    for (int j = za; j <= zb; ++j)
        for (int i = xa; i <= xb; ++i) acc += gp[(size_t)(j + P) * nxq + (i + P)];
    out[(size_t)(ix - 1) * nz + (iz - 1)] = (float)acc;
}

// ============================================================================
// host engine
// ============================================================================
struct Ac2dEngine : Engine {
    int nx, nz, P, R, pr, NXp, NZp, NXs, NZs, pitch;
    long long fs;
    float dt, idx, idz;
    // materials (storage layout, fp32)
    DevBuf<float> dtbk, dtbx, dtbz, vpp, rhop;
    DevBuf<float> pml_x, pml_z;  // ai, bi, ah, bh each of length pitch / NZs
    std::vector<float> h_rhop;   // padded rho (storage layout) for force-source weights
    // batch state
    int cap = 0;        // shots of allocated state
    int cap_groups = 0; // gradient accumulator groups
    DevBuf<float> st;   // 7 fields [f][S][fs]
    DevBuf<float> ad;   // adjoint: p, vx, vz [3][S][fs] + 4 memory x 2 buffers [8][S][fs]
    DevBuf<float> G;    // [6][groups][fs]
    DevBuf<float> Sbuf; // [3][k][S][fs]
    DevBuf<float> ckpt; // [nseg][7][S][fs]
    DevBuf<int> ctr;    // d_step, d_done, nonfinite flag
    DevBuf<float> rec, res, obs_t, src_adj;
    DevBuf<double> gpad, misfit_d;
    DevCSR inj, smp, sct;
    DevBuf<int> inj_shot_ptr, rec_shot_ptr, sct_shot_ptr;
    DevBuf<float> amp;
    DevBuf<unsigned char> live;
    DevBuf<float> seis_tmp;
    DevBuf<int> pt_idx;
    DevBuf<double> pt_val;
    GraphCache g_fwd, g_rec, g_adj;
    long long launches = 0;
    int cur_k = 0, cur_S = 0, tile_x = 32;

    explicit Ac2dEngine(const owl_ssg_desc& d) {
        desc = d;
        OWL_CHECK(d.nx >= 8 && d.nz >= 8, OWL_ERR_INVALID, "nx, nz must be >= 8");
        OWL_CHECK(d.fdhalf == 4 || d.fdhalf == 8, OWL_ERR_INVALID, "fdhalf must be 4 or 8");
        OWL_CHECK(d.pml >= 1, OWL_ERR_INVALID, "pml must be >= 1");
        OWL_CHECK(d.dx > 0 && d.dz > 0 && d.dt > 0 && d.nt >= 1, OWL_ERR_INVALID, "dx, dz, dt, nt must be positive");
        nx = d.nx; nz = d.nz; P = d.pml; R = d.fdhalf; pr = P + R;
        NXp = nx + 2 * P; NZp = nz + 2 * P; NXs = NXp + 2 * R; NZs = NZp + 2 * R;
        pitch = (NXs + 31) / 32 * 32;
        fs = (long long)pitch * NZs;
        dt = d.dt;
        idx = (float)(1.0 / (double)d.dx);
        idz = (float)(1.0 / (double)d.dz);
        OWL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        OWL_CUDA(cudaMemcpyToSymbol(c_fd, fd_coefs(R), sizeof(float) * R));
        ctr.reserve(4);
    }
    ~Ac2dEngine() override {
        g_fwd.reset(); g_rec.reset(); g_adj.reset();
        if (stream) cudaStreamDestroy(stream);
    }

    long long soff(int i, int j) const { return (long long)(j + pr - 1) * pitch + (i + pr - 1); }

    void set_model(int nparam, const float* const* f) override {
        OWL_CHECK(nparam == 2 && f && f[0] && f[1], OWL_ERR_INVALID, "acoustic model needs vp and rho");
        const float* vp = f[0];
        const float* rho = f[1];
        std::vector<float> hvp(fs, 0.f), hrho(fs, 0.f), hbk(fs, 0.f), hbx(fs, 0.f), hbz(fs, 0.f);
        float maxv = -1e30f, minv = 1e30f;
        for (int j = -P; j <= nz + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nz);
                float v = vp[(size_t)(ii - 1) * nz + (jj - 1)], r = rho[(size_t)(ii - 1) * nz + (jj - 1)];
                OWL_CHECK(std::isfinite(v) && std::isfinite(r) && v > 0 && r > 0, OWL_ERR_INVALID,
                          "vp and rho must be finite and positive");
                long long o = soff(i, j);
                hvp[o] = v; hrho[o] = r;
                hbk[o] = dt * (r * v * v);
                maxv = std::max(maxv, v); minv = std::min(minv, v);
            }
        // dtbx at vx node (i+1,j) = dt / (0.5*(rho(i+1,j)+rho(i,j))), same for z
        for (int j = -P + 1; j <= nz + P; ++j)
            for (int m = -P + 1; m <= nx + P; ++m) {
                float re = 0.5f * (hrho[soff(m, j)] + hrho[soff(m - 1, j)]);
                hbx[soff(m, j)] = dt / re;
                float rz = 0.5f * (hrho[soff(m, j)] + hrho[soff(m, j - 1)]);
                hbz[soff(m, j)] = dt / rz;
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
        for (int j = 1; j <= nz; ++j) pmlvp = std::max({pmlvp, hvp[soff(1, j)], hvp[soff(nx, j)]});
        for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, hvp[soff(i, 1)], hvp[soff(i, nz)]});
        float alphamax = (float)(1.0 * (double)desc.f0_max * 3.14159265358979323846);
        Pml1DHost hx = build_pml_1d(nx, P, R, pitch, desc.dx, dt, pmlvp, alphamax);
        Pml1DHost hz = build_pml_1d(nz, P, R, NZs, desc.dz, dt, pmlvp, alphamax);
        std::vector<float> px(4 * pitch), pz(4 * NZs);
        std::copy(hx.ai.begin(), hx.ai.end(), px.begin());
        std::copy(hx.bi.begin(), hx.bi.end(), px.begin() + pitch);
        std::copy(hx.ah.begin(), hx.ah.end(), px.begin() + 2 * pitch);
        std::copy(hx.bh.begin(), hx.bh.end(), px.begin() + 3 * pitch);
        std::copy(hz.ai.begin(), hz.ai.end(), pz.begin());
        std::copy(hz.bi.begin(), hz.bi.end(), pz.begin() + NZs);
        std::copy(hz.ah.begin(), hz.ah.end(), pz.begin() + 2 * NZs);
        std::copy(hz.bh.begin(), hz.bh.end(), pz.begin() + 3 * NZs);
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

    void invalidate_graphs() { g_fwd.reset(); g_rec.reset(); g_adj.reset(); }

    // ---------------- tables ----------------
    int rtot = 0;
    std::vector<int> h_rec_shot_ptr, h_inj_shot_ptr;
    std::vector<int> item_src;     // injection item -> (shot-local source index)
    std::vector<int> item_comp;    // 0: p / vx part, 1: vz part
    std::vector<int> item_shot;
    std::vector<long long> item_rho_cell;  // padded-grid index of rho used by a force component, -1 otherwise
    std::vector<float> item_rho;

    void check_cell(int i, int j, const char* what) const {
        if (i < -P - R + 1 || i > nx + P + R || j < -P - R + 1 || j > nz + P + R)
            throw OwlError(OWL_ERR_INVALID, std::string(what) + " tap outside the padded grid");
    }
    int first_row_p() const { return desc.free_surface ? 2 : -P + 1; }

    void build_tables(int S, const owl_shot* shots, bool need_sct) {
        HostCSR hinj, hsmp, hsct;
        h_inj_shot_ptr.assign(1, 0);
        h_rec_shot_ptr.assign(1, 0);
        std::vector<int> hsct_ptr(1, 0);
        std::vector<float> hamp;
        std::vector<unsigned char> hlive;
        item_src.clear(); item_comp.clear(); item_shot.clear(); item_rho_cell.clear(); item_rho.clear();
        const bool fsf = desc.free_surface != 0;
        const int nt = desc.nt;
        rtot = 0;
        for (int s = 0; s < S; ++s) {
            const owl_shot& sh = shots[s];
            OWL_CHECK(sh.nsrc >= 0 && sh.nrec >= 0 && (sh.nsrc == 0 || sh.src) && (sh.nrec == 0 || sh.rec),
                      OWL_ERR_INVALID, "bad shot arrays");
            for (int k = 0; k < sh.nsrc; ++k) {
                const owl_source& q = sh.src[k];
                OWL_CHECK(q.nt_stf >= 0 && (q.nt_stf == 0 || q.stf), OWL_ERR_INVALID, "bad source STF");
                OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION || q.mechanism == OWL_SRC_FORCE, OWL_ERR_UNSUPPORTED,
                          "acoustic media support explosion and force sources");
                int ncomp = q.mechanism == OWL_SRC_FORCE ? 2 : 1;
                for (int comp = 0; comp < ncomp; ++comp) {
                    long long rc = -1;
                    float rv = 0.f;
                    for (int irz = -4; irz <= 4; ++irz)
                        for (int irx = -4; irx <= 4; ++irx) {
                            int i, j, fld;
                            float w;
                            if (q.mechanism == OWL_SRC_EXPLOSION) {
                                i = q.gx + irx; j = q.gz + irz; fld = 0;
                                w = q.interp_ix[irx + 4] * q.interp_iz[irz + 4];
                                if (fsf && j < 2) continue;
                            } else if (comp == 0) {
                                check_cell(q.hx, q.gz, "force source");
                                float r = h_rhop[soff(q.hx, q.gz)];
                                rc = (long long)(q.gz + P) * (NXp + 2) + (q.hx + P); rv = r;
                                i = q.hx + irx; j = q.gz + irz; fld = 1;
                                w = std::sin(q.polar) / r * q.interp_hx[irx + 4] * q.interp_iz[irz + 4];
                                if (fsf && j < 2) continue;
                            } else {
                                check_cell(q.gx, q.hz, "force source");
                                float r = h_rhop[soff(q.gx, q.hz)];
                                rc = (long long)(q.hz + P) * (NXp + 2) + (q.gx + P); rv = r;
                                i = q.gx + irx; j = q.hz + irz; fld = 2;
                                w = std::cos(q.polar) / r * q.interp_ix[irx + 4] * q.interp_hz[irz + 4];
                                if (fsf && j < 2) continue;
                            }
                            if (w == 0.f) continue;
                            check_cell(i, j, "source");
                            hinj.push(Tap{fld, s, soff(i, j), w, 0});
                        }
                    hinj.close_item();
                    item_src.push_back(k); item_comp.push_back(comp); item_shot.push_back(s);
                    item_rho_cell.push_back(rc); item_rho.push_back(rv);
                    size_t base = hamp.size();
                    hamp.resize(base + nt, 0.f);
                    for (int t = q.nbeg; t <= q.nbeg + q.nt_stf - 1 && t <= nt; ++t)
                        if (t >= 1) hamp[base + t - 1] = q.stf[t - q.nbeg] * q.amp * dt;
                }
            }
            h_inj_shot_ptr.push_back(hinj.nitems());
            // receivers
            std::map<long long, std::vector<std::pair<int, float>>> cells;
            for (int r = 0; r < sh.nrec; ++r) {
                const owl_receiver& q = sh.rec[r];
                int rg = rtot + r;
                hlive.push_back(q.weight != 0.f);
                if (q.weight != 0.f) {
                    for (int irz = -4; irz <= 4; ++irz)
                        for (int irx = -4; irx <= 4; ++irx) {
                            float w = q.interp_ix[irx + 4] * q.interp_iz[irz + 4] * q.weight;
                            if (w == 0.f) continue;
                            int i = q.gx + irx, j = q.gz + irz;
                            check_cell(i, j, "receiver");
                            hsmp.push(Tap{0, s, soff(i, j), w, rg});
                            if (need_sct) {
                                // the adjoint routes mirror-row taps through p(i,2-j) = -p(i,j)
                                int jj = j;
                                float ww = w;
                                if (fsf && j <= 0) { jj = 2 - j; ww = -w; }
                                if (fsf && jj < 2) continue;
                                cells[soff(i, jj)].push_back({rg, ww});
                            }
                        }
                }
                hsmp.close_item();
            }
            for (auto& kv : cells) {
                for (auto& pr_ : kv.second) hsct.push(Tap{0, s, kv.first, pr_.second, pr_.first});
                hsct.close_item();
            }
            rtot += sh.nrec;
            h_rec_shot_ptr.push_back(rtot);
            hsct_ptr.push_back(hsct.nitems());
        }
        inj.upload(hinj, stream);
        smp.upload(hsmp, stream);
        sct.upload(hsct, stream);
        inj_shot_ptr.upload(h_inj_shot_ptr.data(), h_inj_shot_ptr.size(), stream);
        rec_shot_ptr.upload(h_rec_shot_ptr.data(), h_rec_shot_ptr.size(), stream);
        sct_shot_ptr.upload(hsct_ptr.data(), hsct_ptr.size(), stream);
        amp.upload(hamp.data(), hamp.size(), stream);
        live.upload(hlive.data(), hlive.size(), stream);
    }

    // ---------------- state ----------------
    void ensure_state(int S, int groups, int k, bool grad) {
        st.reserve((size_t)7 * S * fs);
        if (grad) {
            ad.reserve((size_t)11 * S * fs);
            G.reserve((size_t)6 * groups * fs);
            Sbuf.reserve((size_t)3 * k * S * fs);
        }
    }

    Ac2dDev dev(int S, int k) {
        Ac2dDev a{};
        a.nx = nx; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch; a.fs = fs;
        a.x0 = R; a.x1 = R + NXp; a.z1 = R + NZp;
        a.fsurf = desc.free_surface != 0;
        a.zp0 = a.fsurf ? pr + 1 : R;
        a.zvx0 = a.fsurf ? pr : R;
        a.zvz0 = a.fsurf ? pr + 1 : R;
        a.idx = idx; a.idz = idz;
        a.nshots = S; a.spt = spt_f;
        a.dtbk = dtbk.p; a.dtbx = dtbx.p; a.dtbz = dtbz.p;
        a.axi = pml_x.p; a.bxi = pml_x.p + pitch; a.axh = pml_x.p + 2 * pitch; a.bxh = pml_x.p + 3 * pitch;
        a.azi = pml_z.p; a.bzi = pml_z.p + NZs; a.azh = pml_z.p + 2 * NZs; a.bzh = pml_z.p + 3 * NZs;
        long long F = (long long)S * fs;
        a.p = st.p; a.vx = st.p + F; a.vz = st.p + 2 * F;
        a.m1 = st.p + 3 * F; a.m2 = st.p + 4 * F; a.m3 = st.p + 5 * F; a.m4 = st.p + 6 * F;
        a.k = k;
        a.d_step = ctr.p;
        if (Sbuf.p && Sbuf.n >= (size_t)3 * k * F) {
            a.sslot = F;
            a.Sp = Sbuf.p; a.Svx = Sbuf.p + (long long)k * F; a.Svz = Sbuf.p + 2LL * k * F;
        }
        if (ad.p && ad.n >= (size_t)11 * F) {
            a.ap = ad.p; a.avx = ad.p + F; a.avz = ad.p + 2 * F;
            a.am1 = ad.p + 3 * F; a.am2 = ad.p + 4 * F; a.am3 = ad.p + 5 * F; a.am4 = ad.p + 6 * F;
            a.aex = ad.p + 7 * F; a.aez = ad.p + 8 * F; a.aepx = ad.p + 9 * F; a.aepz = ad.p + 10 * F;
        }
        if (G.p) {
            long long gg = (long long)((S + spt_a - 1) / spt_a) * fs;
            a.Gbk = G.p; a.Gbx = G.p + gg; a.Gbz = G.p + 2 * gg;
            a.Cbk = G.p + 3 * gg; a.Cbx = G.p + 4 * gg; a.Cbz = G.p + 5 * gg;
        }
        return a;
    }

    PointDev pdev(int S, bool adjoint, bool want_src_adj) {
        PointDev q{};
        long long F = (long long)S * fs;
        if (!adjoint) {
            q.fld[0] = st.p; q.fld[1] = st.p + F; q.fld[2] = st.p + 2 * F;
        } else {
            q.fld[0] = ad.p; q.fld[1] = ad.p + F; q.fld[2] = ad.p + 2 * F;
        }
        q.fs = fs; q.nt = desc.nt; q.rtot = rtot;
        q.inj = view(inj); q.inj_shot_ptr = inj_shot_ptr.p; q.amp = amp.p;
        q.smp = view(smp); q.rec_shot_ptr = rec_shot_ptr.p; q.rec = rec.p;
        q.sct = view(sct); q.sct_shot_ptr = sct_shot_ptr.p; q.res = res.p;
        q.src_adj = want_src_adj ? src_adj.p : nullptr;
        q.d_step = ctr.p; q.d_done = ctr.p + 1;
        return q;
    }

    dim3 grid_for(int rows, int S, int spt, int tz) const {
        return dim3((NXp + tile_x - 1) / tile_x, (rows + tz - 1) / tz, (S + spt - 1) / spt);
    }

    // forward kernels: block tile_x x tz_f, spt_f shots per thread
    template <int RR, bool STORE>
    void launch_fwd(int which, const Ac2dDev& a, int S) {
        dim3 b(tile_x, tz_f);
        if (which == 0) {
            k_ac2d_fwd_p<RR, STORE><<<grid_for(a.z1 - a.zp0, S, spt_f, tz_f), b, 0, stream>>>(a);
        } else {
            k_ac2d_fwd_v<RR, STORE><<<grid_for(a.z1 - std::min(a.zvx0, a.zvz0), S, spt_f, tz_f), b, 0, stream>>>(a);
        }
    }

    // adjoint kernels: block tile_x x tz_a, spt_a shots per thread (one gradient
    // accumulator group per spt_a shots)
    template <int RR>
    void launch_adj(int which, const Ac2dDev& a0, int S) {
        Ac2dDev a = a0;
        a.spt = spt_a;
        dim3 b(tile_x, tz_a);
        if (which == 0) {
            const int rows = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
            k_ac2d_adj_p<RR><<<grid_for(rows, S, spt_a, tz_a), b, 0, stream>>>(a);
        } else {
            const int rows = a.z1 - std::min(a.zvx0, a.zvz0);
            k_ac2d_adj_v<RR><<<grid_for(rows, S, spt_a, tz_a), b, 0, stream>>>(a);
        }
    }

    void launch_kernel(int id, const Ac2dDev& a, int S, bool store = false) {
        if (R == 4) {
            if (id == OWL_K_FWD_P) store ? launch_fwd<4, true>(0, a, S) : launch_fwd<4, false>(0, a, S);
            if (id == OWL_K_FWD_V) store ? launch_fwd<4, true>(1, a, S) : launch_fwd<4, false>(1, a, S);
            if (id == OWL_K_ADJ_P) launch_adj<4>(0, a, S);
            if (id == OWL_K_ADJ_V) launch_adj<4>(1, a, S);
        } else {
            if (id == OWL_K_FWD_P) store ? launch_fwd<8, true>(0, a, S) : launch_fwd<8, false>(0, a, S);
            if (id == OWL_K_FWD_V) store ? launch_fwd<8, true>(1, a, S) : launch_fwd<8, false>(1, a, S);
            if (id == OWL_K_ADJ_P) launch_adj<8>(0, a, S);
            if (id == OWL_K_ADJ_V) launch_adj<8>(1, a, S);
        }
    }

    void launch_step(int kind, const Ac2dDev& a, const PointDev& q, int S) {
        if (kind == 0 || kind == 1) {
            launch_kernel(OWL_K_FWD_P, a, S, kind == 1);
            launch_kernel(OWL_K_FWD_V, a, S, kind == 1);
            k_point_fwd<<<S, 256, 0, stream>>>(q, kind == 0 ? (PT_INJECT | PT_SAMPLE | PT_TICK) : (PT_INJECT | PT_TICK));
        } else {
            launch_kernel(OWL_K_ADJ_P, a, S);
            launch_kernel(OWL_K_ADJ_V, a, S);
            k_point_adj<<<S, 256, 0, stream>>>(q);
        }
        launches += 3;
    }

    void launch_step_any(int kind, const Ac2dDev& a, const PointDev& q, int S) { launch_step(kind, a, q, S); }

    // run n steps of a kind (0 forward, 1 recompute storing S, 2 adjoint)
    void run_steps(int kind, int n, const Ac2dDev& a, const PointDev& q, int S, bool graph) {
        if (n <= 0) return;
        if (!graph) {
            for (int i = 0; i < n; ++i) launch_step_any(kind, a, q, S);
            OWL_LAUNCH_CHECK();
            return;
        }
        GraphCache& gc = kind == 0 ? g_fwd : (kind == 1 ? g_rec : g_adj);
        std::vector<uintptr_t> sig = {(uintptr_t)n, (uintptr_t)S, (uintptr_t)spt_f, (uintptr_t)spt_a,
                                      (uintptr_t)tz_f, (uintptr_t)tz_a, (uintptr_t)a.k,
                                      (uintptr_t)st.p, (uintptr_t)ad.p, (uintptr_t)Sbuf.p, (uintptr_t)G.p,
                                      (uintptr_t)rec.p, (uintptr_t)res.p, (uintptr_t)src_adj.p,
                                      (uintptr_t)q.src_adj, (uintptr_t)inj.ptr.p, (uintptr_t)inj.w.p,
                                      (uintptr_t)smp.ptr.p, (uintptr_t)smp.w.p, (uintptr_t)sct.ptr.p,
                                      (uintptr_t)sct.w.p, (uintptr_t)amp.p, (uintptr_t)inj_shot_ptr.p,
                                      (uintptr_t)rec_shot_ptr.p, (uintptr_t)sct_shot_ptr.p, (uintptr_t)q.rtot,
                                      (uintptr_t)tile_x, (uintptr_t)dtbk.p};
        if (!gc.exec || gc.sig != sig) {
            gc.reset();
            cudaGraph_t g;
            OWL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            long long l0 = launches;
            for (int i = 0; i < n; ++i) launch_step_any(kind, a, q, S);
            cudaError_t e1 = cudaGetLastError();
            cudaError_t e2 = cudaStreamEndCapture(stream, &g);
            OWL_CUDA(e1);
            OWL_CUDA(e2);
            launches = l0;
            cudaError_t e3 = cudaGraphInstantiate(&gc.exec, g, 0);
            cudaGraphDestroy(g);
            OWL_CUDA(e3);
            gc.sig = sig;
        }
        OWL_CUDA(cudaGraphLaunch(gc.exec, stream));
        launches += 3LL * n;
    }

    void set_step(int v) {
        int h[2] = {v, 0};
        OWL_CUDA(cudaMemcpyAsync(ctr.p, h, 2 * sizeof(int), cudaMemcpyHostToDevice, stream));
    }

    bool tune = false;
    int spt_f = 1, spt_a = 1, tz_f = 8, tz_a = 8;
    void resolve_opts(const owl_run_opts& o, int nshots, int& B, int& k, bool& graph) {
        tune = o.shots_per_cta <= 0 && o.tile_z <= 0;
        B = o.shots_per_launch > 0 ? o.shots_per_launch : std::max(1, desc.max_shots);
        B = std::min(B, std::max(1, nshots));
        k = o.checkpoint_interval > 0 ? o.checkpoint_interval : 50;
        k = std::min(k, desc.nt);
        spt_f = spt_a = std::min(o.shots_per_cta > 0 ? o.shots_per_cta : 1, B);
        graph = o.use_graph >= 0;  // default on; -1 disables
        tile_x = o.tile_x > 0 ? o.tile_x : 32;
        tz_f = tz_a = o.tile_z > 0 ? o.tile_z : 8;
        OWL_CHECK(tile_x % 32 == 0 && tz_f >= 1 && tile_x * tz_f <= 512, OWL_ERR_INVALID,
                  "tile_x must be a multiple of 32 and tile_x * tile_z <= 512");
    }

    // Autotuner: times the stencil kernels of one step for each (shots per CTA,
    // tile height) candidate on this batch's buffers and keeps the fastest, for
    // the forward pair and the adjoint pair separately. Cached per batch size.
    // The buffers' contents are reset by the caller afterwards.
    std::map<std::pair<int, int>, std::array<int, 4>> tune_cache;
    void autotune(int S, int k, bool grad) {
        auto key = std::make_pair(S, grad ? 1 : 0);
        auto it = tune_cache.find(key);
        if (it != tune_cache.end()) {
            spt_f = it->second[0]; tz_f = it->second[1]; spt_a = it->second[2]; tz_a = it->second[3];
            return;
        }
        set_step(k);
        for (int pass = 0; pass < (grad ? 2 : 1); ++pass) {
            float best = 1e30f;
            int bs = 1, bt = 8;
            for (int spt : {1, 2, 4, 8, 16, 32}) {
                if (spt > S) break;
                for (int tz : {4, 8, 16}) {
                    if (pass == 0) { spt_f = spt; tz_f = tz; } else { spt_a = spt; tz_a = tz; }
                    Ac2dDev a = dev(S, k);
                    auto run = [&]() {
                        if (pass == 0) { launch_kernel(OWL_K_FWD_P, a, S); launch_kernel(OWL_K_FWD_V, a, S); }
                        else { launch_kernel(OWL_K_ADJ_P, a, S); launch_kernel(OWL_K_ADJ_V, a, S); }
                    };
                    run();
                    OWL_LAUNCH_CHECK();
                    EventTimer tm(stream);
                    for (int i = 0; i < 5; ++i) run();
                    float ms = (float)tm.stop_ms();
                    launches += 12;
                    if (ms < best) { best = ms; bs = spt; bt = tz; }
                }
            }
            if (pass == 0) { spt_f = bs; tz_f = bt; } else { spt_a = bs; tz_a = bt; }
        }
        tune_cache[key] = {spt_f, tz_f, spt_a, tz_a};
    }

    size_t seis_count(int n, const owl_shot* shots) const {
        size_t c = 0;
        for (int s = 0; s < n; ++s) c += (size_t)shots[s].nrec * desc.nt;
        return c;
    }

    // forward pass of one batch (state zeroed); optional checkpoints
    void forward_batch(int S, int k, bool graph, bool save_ckpt) {
        const int nt = desc.nt;
        Ac2dDev a = dev(S, k);
        PointDev q = pdev(S, false, false);
        OWL_CUDA(cudaMemsetAsync(st.p, 0, sizeof(float) * 7 * S * fs, stream));
        set_step(0);
        k_point_fwd<<<S, 256, 0, stream>>>(q, PT_SAMPLE);
        OWL_LAUNCH_CHECK();
        launches++;
        int nseg = (nt + k - 1) / k;
        long long F7 = 7LL * S * fs;
        for (int sg = 0; sg < nseg; ++sg) {
            if (save_ckpt)
                OWL_CUDA(cudaMemcpyAsync(ckpt.p + sg * F7, st.p, sizeof(float) * F7, cudaMemcpyDeviceToDevice, stream));
            int n = std::min(k, nt - sg * k);
            run_steps(0, n, a, q, S, graph && n == k);
        }
    }

    void check_nonfinite(const float* f, size_t n) {
        OWL_CUDA(cudaMemsetAsync(ctr.p + 2, 0, sizeof(int), stream));
        launch_check_finite(f, n, ctr.p + 2, stream);
        launches++;
        int flag = 0;
        OWL_CUDA(cudaMemcpyAsync(&flag, ctr.p + 2, sizeof(int), cudaMemcpyDeviceToHost, stream));
        OWL_CUDA(cudaStreamSynchronize(stream));
        if (flag) throw OwlError(OWL_ERR_NONFINITE, "non-finite values in the wavefield");
    }

    void copy_out(void* dst, const void* src, size_t bytes, int mem) {
        OWL_CUDA(cudaMemcpyAsync(dst, src, bytes, mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                 stream));
    }

    void forward(int nshots, const owl_shot* shots, const owl_run_opts& o, float* seis, int mem,
                 owl_run_info& info) override {
        OWL_CHECK(model_set, OWL_ERR_INVALID, "set_model must be called first");
        int B, k;
        bool graph;
        resolve_opts(o, nshots, B, k, graph);
        launches = 0;
        EventTimer tm(stream);
        size_t out_off = 0;
        int batches = 0;
        for (int b0 = 0; b0 < nshots; b0 += B) {
            int S = std::min(B, nshots - b0);
            build_tables(S, shots + b0, false);
            ensure_state(S, S, k, false);
            if (tune) autotune(S, k, false);
            rec.reserve((size_t)desc.nt * std::max(rtot, 1));
            OWL_CUDA(cudaMemsetAsync(rec.p, 0, sizeof(float) * desc.nt * std::max(rtot, 1), stream));
            forward_batch(S, k, graph, false);
            cur_S = S; cur_k = k;
            if (o.check_every > 0) check_nonfinite(st.p, (size_t)S * fs);
            size_t n = (size_t)rtot * desc.nt;
            if (n) {
                seis_tmp.reserve(n);
                launch_transpose_rec_to_seis(rec.p, seis_tmp.p, desc.nt, rtot, stream);
                launches++;
                copy_out(seis + out_off, seis_tmp.p, n * sizeof(float), mem);
            }
            out_off += n;
            batches++;
        }
        info.elapsed_ms = tm.stop_ms();
        info.gpu_launches = launches;
        info.steps_cell_updates = (double)NXp * NZp * desc.nt * nshots;
        info.dt_used = dt;
        info.dt_stable = dt_stable_;
        info.shots_per_cta = spt_f;
        info.tile_x = tile_x;
        info.tile_z = tz_f;
        info.batches = batches;
    }

    void gradient_impl(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                       double* misfit, float* grad, float* seis_out, float* stf_grad, int mem, owl_run_info& info) {
        OWL_CHECK(model_set, OWL_ERR_INVALID, "set_model must be called first");
        OWL_CHECK(adj_kind == OWL_ADJ_L2_RESIDUAL || adj_kind == OWL_ADJ_GIVEN, OWL_ERR_INVALID, "bad adj_kind");
        OWL_CHECK(o.checkpoint_precision == OWL_CKPT_FP32, OWL_ERR_UNSUPPORTED,
                  "acoustic 2D checkpoints are FP32 in this build");
        int B, k;
        bool graph;
        resolve_opts(o, nshots, B, k, graph);
        launches = 0;
        const int nt = desc.nt;
        const int nxq = NXp + 2, nzq = NZp + 2;
        EventTimer tm(stream);
        gpad.reserve((size_t)2 * nxq * nzq);
        OWL_CUDA(cudaMemsetAsync(gpad.p, 0, sizeof(double) * 2 * nxq * nzq, stream));
        size_t data_off = 0;
        size_t stf_off = 0;
        int batches = 0;
        int shot0 = 0;
        for (int b0 = 0; b0 < nshots; b0 += B) {
            int S = std::min(B, nshots - b0);
            const owl_shot* sh = shots + b0;
            build_tables(S, sh, true);
            ensure_state(S, S, k, true);
            if (tune) autotune(S, k, true);
            int groups = (S + spt_a - 1) / spt_a;
            int nseg = (nt + k - 1) / k;
            ckpt.reserve((size_t)nseg * 7 * S * fs);
            size_t nrt = (size_t)nt * std::max(rtot, 1);
            rec.reserve(nrt);
            res.reserve(nrt);
            obs_t.reserve(nrt);
            OWL_CUDA(cudaMemsetAsync(rec.p, 0, sizeof(float) * nrt, stream));
            bool want_src = stf_grad != nullptr;
            for (size_t it = 0; it < item_rho_cell.size(); ++it) want_src |= item_rho_cell[it] >= 0;
            size_t nitems = item_src.size();
            src_adj.reserve(std::max<size_t>(1, nitems * nt));
            if (want_src) OWL_CUDA(cudaMemsetAsync(src_adj.p, 0, sizeof(float) * std::max<size_t>(1, nitems * nt), stream));
            // 1. forward with checkpoints
            forward_batch(S, k, graph, true);
            cur_S = S; cur_k = k;
            if (o.check_every > 0) check_nonfinite(st.p, (size_t)S * fs);
            // 2. adjoint source
            size_t n = (size_t)rtot * nt;
            misfit_d.reserve(S);
            OWL_CUDA(cudaMemsetAsync(misfit_d.p, 0, sizeof(double) * S, stream));
            if (n) {
                seis_tmp.reserve(n);
                OWL_CUDA(cudaMemcpyAsync(seis_tmp.p, data + data_off, n * sizeof(float),
                                         mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                         stream));
                launch_transpose_seis_to_rec(seis_tmp.p, obs_t.p, nt, rtot, stream);
                launches++;
                if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
                    launch_residual_l2(rec.p, obs_t.p, res.p, live.p, rec_shot_ptr.p, S, nt, rtot, misfit_d.p, stream);
                } else {
                    OWL_CUDA(cudaMemcpyAsync(res.p, obs_t.p, n * sizeof(float), cudaMemcpyDeviceToDevice, stream));
                }
                launches++;
                if (seis_out) {
                    launch_transpose_rec_to_seis(rec.p, seis_tmp.p, nt, rtot, stream);
                    launches++;
                    copy_out(seis_out + data_off, seis_tmp.p, n * sizeof(float), mem);
                }
            }
            if (misfit) copy_out(misfit + shot0, misfit_d.p, sizeof(double) * S, mem);
            // 3. reverse sweep
            long long F = (long long)S * fs;
            OWL_CUDA(cudaMemsetAsync(ad.p, 0, sizeof(float) * 11 * F, stream));
            OWL_CUDA(cudaMemsetAsync(G.p, 0, sizeof(float) * 6 * groups * fs, stream));
            Ac2dDev a = dev(S, k);
            PointDev qf = pdev(S, false, false);
            PointDev qa = pdev(S, true, want_src);
            for (int sg = nseg - 1; sg >= 0; --sg) {
                int n0 = sg * k, nn = std::min(k, nt - n0);
                OWL_CUDA(cudaMemcpyAsync(st.p, ckpt.p + sg * 7 * F, sizeof(float) * 7 * F, cudaMemcpyDeviceToDevice, stream));
                set_step(n0);
                run_steps(1, nn, a, qf, S, graph && nn == k);
                run_steps(2, nn, a, qa, S, graph && nn == k);
            }
            if (o.check_every > 0) check_nonfinite(ad.p, (size_t)S * fs);
            // 4. chain rule (FP64) into the padded accumulators
            dim3 b(32, 8), g((nxq + 31) / 32, (nzq + 7) / 8);
            k_ac2d_chain<<<g, b, 0, stream>>>(a, groups, vpp.p, rhop.p, (double)dt, gpad.p, gpad.p + (size_t)nxq * nzq,
                                              nxq, nzq);
            OWL_LAUNCH_CHECK();
            launches++;
            // 5. source-side terms: rho at force points, STF gradient
            if (want_src && nitems) {
                std::vector<float> hsa(nitems * nt);
                OWL_CUDA(cudaMemcpyAsync(hsa.data(), src_adj.p, sizeof(float) * nitems * nt, cudaMemcpyDeviceToHost,
                                         stream));
                std::vector<float> hamp(nitems * nt);
                OWL_CUDA(cudaMemcpyAsync(hamp.data(), amp.p, sizeof(float) * nitems * nt, cudaMemcpyDeviceToHost, stream));
                OWL_CUDA(cudaStreamSynchronize(stream));
                std::map<int, double> pts;
                for (size_t it = 0; it < nitems; ++it) {
                    if (item_rho_cell[it] < 0) continue;
                    double acc = 0;
                    for (int t = 0; t < nt; ++t) acc += (double)hamp[it * nt + t] * (double)hsa[it * nt + t];
                    // w = sin|cos(polar)/rho * taps -> d/drho (A w lambda) = -A w lambda / rho
                    pts[(int)item_rho_cell[it] + nxq * nzq] += -acc / (double)item_rho[it];
                }
                if (!pts.empty()) {
                    std::vector<int> hi;
                    std::vector<double> hv;
                    for (auto& kv : pts) { hi.push_back(kv.first); hv.push_back(kv.second); }
                    pt_idx.upload(hi.data(), hi.size(), stream);
                    pt_val.upload(hv.data(), hv.size(), stream);
                    k_add_points_f64<<<(int)(hi.size() + 127) / 128, 128, 0, stream>>>(gpad.p, pt_idx.p, pt_val.p,
                                                                                       (int)hi.size());
                    OWL_LAUNCH_CHECK();
                    launches++;
                }
                if (stf_grad) {
                    // dJ/dstf_k(t - nbeg + 1) = sum over components of src_adj * amp * dt, per step t
                    for (int s = 0; s < S; ++s) {
                        const owl_shot& shs = sh[s];
                        for (int kk = 0; kk < shs.nsrc; ++kk) {
                            float* outk = stf_grad + stf_off + (size_t)kk * nt;
                            for (int t = 0; t < nt; ++t) outk[t] = 0.f;
                        }
                        for (size_t it = 0; it < nitems; ++it) {
                            if (item_shot[it] != s) continue;
                            const owl_source& q = shs.src[item_src[it]];
                            float* outk = stf_grad + stf_off + (size_t)item_src[it] * nt;
                            for (int t = 0; t < nt; ++t)
                                outk[t] += (float)((double)hsa[it * nt + t] * (double)q.amp * (double)dt);
                        }
                        stf_off += (size_t)shs.nsrc * nt;
                    }
                }
            }
            data_off += n;
            shot0 += S;
            batches++;
        }
        if (grad) {
            size_t nm = (size_t)nx * nz;
            seis_tmp.reserve(2 * nm);
            dim3 b(32, 8), g((nz + 31) / 32, (nx + 7) / 8);
            k_fold2d<<<g, b, 0, stream>>>(gpad.p, nxq, nzq, P, nx, nz, seis_tmp.p);
            k_fold2d<<<g, b, 0, stream>>>(gpad.p + (size_t)nxq * nzq, nxq, nzq, P, nx, nz, seis_tmp.p + nm);
            OWL_LAUNCH_CHECK();
            launches += 2;
            copy_out(grad, seis_tmp.p, 2 * nm * sizeof(float), mem);
        }
        info.elapsed_ms = tm.stop_ms();
        info.gpu_launches = launches;
        info.steps_cell_updates = 3.0 * NXp * NZp * nt * nshots;
        info.dt_used = dt;
        info.dt_stable = dt_stable_;
        info.shots_per_cta = spt_a;
        info.tile_x = tile_x;
        info.tile_z = tz_a;
        info.batches = batches;
    }

    // compulsory bytes of one launch of a kernel (each state field read / written
    // once per shot, materials once per launch, PML memory only inside the PML,
    // gradient accumulators once per shot group)
    double alg_bytes(int id, int S, int groups) const {
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

    void kernel_time(int id, int nlaunch, double* avg_ms, double* bytes) override {
        OWL_CHECK(cur_S > 0, OWL_ERR_INVALID, "no batch has run on this handle");
        OWL_CHECK(id >= OWL_K_FWD_P && id <= OWL_K_ADJ_V, OWL_ERR_INVALID, "bad kernel id");
        const int S = cur_S, k = cur_k;
        OWL_CHECK(id < OWL_K_ADJ_P || (ad.p && G.p && Sbuf.p), OWL_ERR_INVALID,
                  "adjoint kernels need a gradient call first");
        Ac2dDev a = dev(S, k);
        if (id >= OWL_K_ADJ_P)
            OWL_CHECK(a.ap && a.Sp, OWL_ERR_INVALID, "adjoint buffers too small for the last batch");
        set_step(k);
        auto launch = [&]() { launch_kernel(id, a, S); };
        for (int i = 0; i < 3; ++i) launch();
        OWL_LAUNCH_CHECK();
        EventTimer tm(stream);
        for (int i = 0; i < nlaunch; ++i) launch();
        OWL_LAUNCH_CHECK();
        *avg_ms = tm.stop_ms() / nlaunch;
        *bytes = alg_bytes(id, S, (S + spt_a - 1) / spt_a);
    }

    void gradient(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                  double* misfit, float* grad, float* seis_out, int mem, owl_run_info& info) override {
        gradient_impl(nshots, shots, data, adj_kind, o, misfit, grad, seis_out, nullptr, mem, info);
    }

    void source_gradient(int nshots, const owl_shot* shots, const float* adj, const owl_run_opts& o, float* stf_grad,
                         int mem, owl_run_info& info) override {
        OWL_CHECK(mem == OWL_MEM_HOST, OWL_ERR_UNSUPPORTED, "source_gradient takes host buffers");
        gradient_impl(nshots, shots, adj, OWL_ADJ_GIVEN, o, nullptr, nullptr, nullptr, stf_grad, mem, info);
    }
};

Engine* make_ac2d_engine(const owl_ssg_desc& d) { return new Ac2dEngine(d); }

}  // namespace owl
