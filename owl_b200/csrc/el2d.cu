// el2d.cu -- 2D elastic VTI / tilted-TI SSG solver for B200 (sm_100a).
//
// Forward (replaces update_wavefield / update_wavefield_free_surface /
// add_source and the surface images + sampling of compute_forward,
// src/solver/elastic_vhtiort_2d/module_wavefield.f90:42-403 and
// submodule_forward_modeling.f90:58-197) on the uniform grid
// (free_surface_dz_refine = 1), and the exact discrete adjoint with every-k-step
// checkpoints, strain-stress correlations for (c11, c13, c33, c55, rho) and the
// FP64 chain rule to the model parameters (replaces compute_adjoint /
// compute_gradient, submodule_fwi_gradient.f90:31-557, whose time-reversed
// propagation is not the transpose of the forward).
//
// Nodes. sigma_xx, sigma_zz at integer nodes (i, j); sigma_xz at (i-1/2, j-1/2);
// vx at (i-1/2, j); vz at (i, j-1/2); every field is stored at the reference's
// own index, x = i + pml + R - 1 (same for z), in (NZs x pitch) float32 planes,
// x fastest, shot-major. Forward state per shot: the 5 fields and the 8 CFS-MPML
// memory planes (touched only inside the PML). Materials shared by the shots:
// c11, c13, c33, the harmonic c55 of the sigma_xz nodes, dt/rho_x, dt/rho_z and,
// per staggered position (ii, hh, hi, ih), the M-PML coefficients (a_x, b_x,
// a_z, b_z) as one float4 (read only inside the PML).
//
// One time step is three launches over all shots of a batch:
//   k_el2d_fwd_s : sigma_xx, sigma_zz, sigma_xz (free surface: row-1 traction
//                  condition, sigma_zz(1) = 0 and the odd images of sigma_zz and
//                  sigma_xz, fused)
//   k_el2d_fwd_v : vx, vz
//   point kernel : add_source(t), receivers of step t+1, step counter
// The adjoint of a step is k_el2d_adj_v (velocity nodes), an optional point
// kernel (source-side adjoint), k_el2d_adj_s (stress nodes) and the point
// kernel of the residual injection; each node computes the adjoint PML terms e
// of its own derivatives once, and its neighbours apply the transposed stencil
// to them in the next launch.
#include <algorithm>
#include <cmath>
#include <complex>

#include "ssg_base.cuh"
#include "vec4.cuh"
#include "vmesh.hpp"

namespace owl {

__constant__ float c_fde[8];

// state planes of one shot
enum { EL_SXX = 0, EL_SZZ, EL_SXZ, EL_VX, EL_VZ, EL_M0 };
// memory / adjoint-PML-term order: d_x vx, d_z vz (sigma nodes), d_z vx, d_x vz
// (sigma_xz nodes), d_x sxx, d_z sxz (vx nodes), d_x sxz, d_z szz (vz nodes)
enum { M_DXVX = 0, M_DZVZ, M_DZVX, M_DXVZ, M_DXXX, M_DZXZ, M_DXXZ, M_DZZZ };
constexpr int EL_NST = 13;        // forward planes per shot
constexpr int EL_NAD = 5 + 8 + 8; // adjoint fields, memory adjoints, e terms

struct El2dDev {
    int nx, nz, P, R, pr, pitch;
    long long fs, sst, sad;
    int x0, x1, z1, zs0, zxz0, zvx0, zvz0, fsurf;
    float idx, idz, dt;
    int nshots, spt;
    const float *c11, *c13, *c33, *c55e, *bx, *bz;
    const float4 *pii, *phh, *phi, *pih;
    // per storage row: dz / dz_i and dz / dz_h of the depth-refined mesh, the
    // factors of the z derivatives at integer-z nodes (sigma_xx, sigma_zz, vx)
    // and half-z nodes (sigma_xz, vz); 1 on the uniform grid
    const float *zfi, *zfh;
    float* st;   // forward state (shot 0)
    float* S;    // stored stencil terms: [term][slot][shot][fs]
    long long sslot, sterm;
    int k;
    int* d_step;
    float* ad;   // adjoint state (shot 0)
    float* G;    // [6][group][fs] sums, then [6][group][fs] Kahan compensations
    long long gg;
};

__device__ __forceinline__ bool el_pml_int(int x, int pr, int n) { return x < pr || x >= pr + n; }
__device__ __forceinline__ bool el_pml_half(int x, int pr, int n) { return x <= pr || x >= pr + n; }

// adjoint of psi_new = a D + b psi_old, D' = D + psi_new, given q = adjoint of D'
__device__ __forceinline__ float pml_e(float q, float a, float b, float psih, float* dst) {
    const float u = q + psih;
    *dst = b * u;
    return q + a * u;
}

// ------------------------------- forward ------------------------------------
// 48 registers at R = 4 (no spills): five 256-thread CTAs per SM instead of four
// ZR: the depth-refined free-surface mesh (per-row dz scalings); the uniform
// grid's instances leave them out
template <int R, bool STORE, bool ZR>
__global__ void __maxnreg__(R == 4 ? 48 : 128) k_el2d_fwd_s(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = a.zs0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const int pt = a.pitch;
    const bool row1 = a.fsurf && z == a.pr;
    const bool dxz = z >= a.zxz0;
    const bool px_i = el_pml_int(x, a.pr, a.nx);
    const bool pii = px_i || (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool phh = el_pml_half(x, a.pr, a.nx) || (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float4 cii = pii ? __ldg(a.pii + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 chh = (phh && dxz) ? __ldg(a.phh + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float c11 = __ldg(a.c11 + o), c13 = __ldg(a.c13 + o), c33 = __ldg(a.c33 + o);
    const float c55dt = dxz ? a.dt * __ldg(a.c55e + o) : 0.f;
    // 1/dz times the row's dz scaling (refined mesh)
    const float zsi = ZR ? a.idz * __ldg(a.zfi + z) : a.idz, zsh = ZR ? a.idz * __ldg(a.zfh + z) : a.idz;
    const bool mir = a.fsurf && z > a.pr && z <= a.pr + a.R;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    for (int s = s0; s < s1; ++s) {
        float* st = a.st + s * a.sst;
        const float* vx = st + EL_VX * a.fs + o;
        const float* vz = st + EL_VZ * a.fs + o;
        float* mem = st + EL_M0 * a.fs + o;
        float* sxx = st + EL_SXX * a.fs + o;
        float* szz = st + EL_SZZ * a.fs + o;
        float* sxzp = st + EL_SXZ * a.fs + o;
        // the cell's own stresses and memories are read ahead of its stores:
        // the fields share one allocation, so no plain read could move above a
        // store and each would cost its own round trip
        const float xx0 = *sxx, zz0 = row1 ? 0.f : *szz, xz0 = dxz ? *sxzp : 0.f;
        const float mxv = (row1 ? px_i : pii) ? mem[M_DXVX * a.fs] : 0.f;
        const float mzv = !row1 && pii ? mem[M_DZVZ * a.fs] : 0.f;
        const float mxz = dxz && phh ? mem[M_DXVZ * a.fs] : 0.f, mzx = dxz && phh ? mem[M_DZVX * a.fs] : 0.f;
        // sigma_xx, sigma_zz
        float sx = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(vx + (k)) - __ldg(vx + (1 - k)));
        float dxv = a.idx * sx, dzv;
        if (row1) {
            if (px_i) {
                const float m = cii.x * dxv + cii.y * mxv;
                mem[M_DXVX * a.fs] = m;
                dxv = dxv + m;
            }
            dzv = -(c13 / c33 * dxv);
        } else {
            float sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(vz + (k * pt)) - __ldg(vz + ((1 - k) * pt)));
            dzv = zsi * sz;
            if (pii) {
                const float m1 = cii.x * dxv + cii.y * mxv;
                mem[M_DXVX * a.fs] = m1;
                dxv = dxv + m1;
                const float m2 = cii.z * dzv + cii.w * mzv;
                mem[M_DZVZ * a.fs] = m2;
                dzv = dzv + m2;
            }
        }
        *sxx = xx0 + a.dt * (c11 * dxv + c13 * dzv);
        if (row1) {
            *szz = 0.f;
        } else {
            const float zn = zz0 + a.dt * (c13 * dxv + c33 * dzv);
            *szz = zn;
            if (mir) st[EL_SZZ * a.fs + (long long)(2 * a.pr - z) * pt + x] = -zn;
        }
        if (STORE) {
            a.S[slot + s * a.fs + o] = dxv;
            a.S[a.sterm + slot + s * a.fs + o] = dzv;
        }
        // sigma_xz
        if (dxz) {
            float szx = 0.f, sxz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) szx = szx + c_fde[k - 1] * (__ldg(vx + ((k - 1) * pt)) - __ldg(vx + (-k * pt)));
#pragma unroll
            for (int k = 1; k <= R; ++k) sxz = sxz + c_fde[k - 1] * (__ldg(vz + (k - 1)) - __ldg(vz + (-k)));
            float dzvx = zsh * szx, dxvz = a.idx * sxz;
            if (phh) {
                const float m3 = chh.x * dxvz + chh.y * mxz;
                mem[M_DXVZ * a.fs] = m3;
                dxvz = dxvz + m3;
                const float m4 = chh.z * dzvx + chh.w * mzx;
                mem[M_DZVX * a.fs] = m4;
                dzvx = dzvx + m4;
            }
            const float g = dzvx + dxvz;
            const float xn = xz0 + c55dt * g;
            *sxzp = xn;
            if (mir) st[EL_SXZ * a.fs + (long long)(2 * a.pr + 1 - z) * pt + x] = -xn;
            if (STORE) a.S[2 * a.sterm + slot + s * a.fs + o] = g;
        }
    }
}

template <int R, bool STORE, bool ZR>
__global__ void __launch_bounds__(512) k_el2d_fwd_v(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = a.zvx0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const int pt = a.pitch;
    const bool dvz = z >= a.zvz0;
    const bool phi = el_pml_half(x, a.pr, a.nx) || (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool pih = el_pml_int(x, a.pr, a.nx) || (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float4 chi = phi ? __ldg(a.phi + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 cih = (pih && dvz) ? __ldg(a.pih + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float bx = __ldg(a.bx + o), bz = dvz ? __ldg(a.bz + o) : 0.f;
    const float zsi = ZR ? a.idz * __ldg(a.zfi + z) : a.idz, zsh = ZR ? a.idz * __ldg(a.zfh + z) : a.idz;  // see k_el2d_fwd_s
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    for (int s = s0; s < s1; ++s) {
        float* st = a.st + s * a.sst;
        const float* sxx = st + EL_SXX * a.fs + o;
        const float* szz = st + EL_SZZ * a.fs + o;
        const float* sxz = st + EL_SXZ * a.fs + o;
        float* mem = st + EL_M0 * a.fs + o;
        // own velocities and memories ahead of the stores (see k_el2d_fwd_s)
        const float vx0 = st[EL_VX * a.fs + o], vz0 = dvz ? st[EL_VZ * a.fs + o] : 0.f;
        const float m_xxx = phi ? mem[M_DXXX * a.fs] : 0.f, m_zxz = phi ? mem[M_DZXZ * a.fs] : 0.f;
        const float m_xxz = dvz && pih ? mem[M_DXXZ * a.fs] : 0.f, m_zzz = dvz && pih ? mem[M_DZZZ * a.fs] : 0.f;
        {
            float sx = 0.f, sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(sxx + (k - 1)) - __ldg(sxx + (-k)));
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(sxz + (k * pt)) - __ldg(sxz + ((1 - k) * pt)));
            float hx = a.idx * sx, hz = zsi * sz;
            if (phi) {
                const float m1 = chi.x * hx + chi.y * m_xxx;
                mem[M_DXXX * a.fs] = m1;
                hx = hx + m1;
                const float m2 = chi.z * hz + chi.w * m_zxz;
                mem[M_DZXZ * a.fs] = m2;
                hz = hz + m2;
            }
            const float h = hx + hz;
            st[EL_VX * a.fs + o] = vx0 + bx * h;
            if (STORE) a.S[3 * a.sterm + slot + s * a.fs + o] = h;
        }
        if (dvz) {
            float sx = 0.f, sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(sxz + (k)) - __ldg(sxz + (1 - k)));
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(szz + ((k - 1) * pt)) - __ldg(szz + (-k * pt)));
            float hx = a.idx * sx, hz = zsh * sz;
            if (pih) {
                const float m1 = cih.x * hx + cih.y * m_xxz;
                mem[M_DXXZ * a.fs] = m1;
                hx = hx + m1;
                const float m2 = cih.z * hz + cih.w * m_zzz;
                mem[M_DZZZ * a.fs] = m2;
                hz = hz + m2;
            }
            const float h = hx + hz;
            st[EL_VZ * a.fs + o] = vz0 + bz * h;
            if (STORE) a.S[4 * a.sterm + slot + s * a.fs + o] = h;
        }
    }
}

#include "el2d_vec.cuh"

// ------------------------------- adjoint ------------------------------------
// Adjoint state planes of one shot: 0..4 the fields' adjoints (sxx, szz, sxz,
// vx, vz), 5..12 the memory adjoints, 13..20 the e terms (same order as the
// memories). An e plane is written only at the owner nodes of its derivative;
// everywhere else it stays zero.
__device__ __forceinline__ void kahan_g(float* G, long long gg, long long go, int q, float v) {
    float sm = G[q * gg + go], c = G[(6 + q) * gg + go];
    kahan_add(sm, c, v);
    G[q * gg + go] = sm;
    G[(6 + q) * gg + go] = c;
}

// velocity nodes: finish the adjoint of the stress update of step t+1
// (v^ += D^T e of the sigma nodes), correlate v^ with the stored terms of step
// t (rho gradient), then the adjoint PML terms of the velocity update of step t
template <int R, bool ZR>
__global__ void __launch_bounds__(512) k_el2d_adj_v(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = a.zvx0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const int pt = a.pitch;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool dvz = z >= a.zvz0;
    const bool phi = el_pml_half(x, a.pr, a.nx) || (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool pih = el_pml_int(x, a.pr, a.nx) || (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float4 chi = phi ? __ldg(a.phi + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 cih = (pih && dvz) ? __ldg(a.pih + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float bx = __ldg(a.bx + o), bz = dvz ? __ldg(a.bz + o) : 0.f;
    // the z-derivative e terms carry the node's dz scaling, so that the
    // neighbours' transposed stencils stay plain
    const float zsi = ZR ? __ldg(a.zfi + z) : 1.f, zsh = ZR ? __ldg(a.zfh + z) : 1.f;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    float gbx = 0.f, gbz = 0.f;
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        float* e = ad + 13 * a.fs + o;
        float* mh = ad + 5 * a.fs + o;
        const long long so = slot + s * a.fs + o;
        // own adjoint velocities and memories ahead of the stores (see k_el2d_fwd_s)
        const float vx0 = ad[EL_VX * a.fs + o], vz0 = dvz ? ad[EL_VZ * a.fs + o] : 0.f;
        const float m_xxx = phi ? mh[M_DXXX * a.fs] : 0.f, m_zxz = phi ? mh[M_DZXZ * a.fs] : 0.f;
        const float m_xxz = dvz && pih ? mh[M_DXXZ * a.fs] : 0.f, m_zzz = dvz && pih ? mh[M_DZZZ * a.fs] : 0.f;
        {
            const float* e1 = e + M_DXVX * a.fs;
            const float* e2 = e + M_DZVX * a.fs;
            float sx = 0.f, sz = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(e1 + (-k)) - __ldg(e1 + (k - 1)));
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(e2 + ((1 - k) * pt)) - __ldg(e2 + (k * pt)));
            const float v = vx0 + (a.idx * sx + a.idz * sz);
            ad[EL_VX * a.fs + o] = v;
            gbx += v * __ldg(a.S + 3 * a.sterm + so);
            const float q = bx * v;
            float ex = q, ez = q;
            if (phi) {
                ex = pml_e(q, chi.x, chi.y, m_xxx, mh + M_DXXX * a.fs);
                ez = pml_e(q, chi.z, chi.w, m_zxz, mh + M_DZXZ * a.fs);
            }
            e[M_DXXX * a.fs] = ex;
            e[M_DZXZ * a.fs] = ZR ? ez * zsi : ez;
        }
        if (dvz) {
            const float* e4 = e + M_DZVZ * a.fs;
            const float* e3 = e + M_DXVZ * a.fs;
            float sz = 0.f, sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(e4 + (-k * pt)) - __ldg(e4 + ((k - 1) * pt)));
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(e3 + (1 - k)) - __ldg(e3 + (k)));
            const float v = vz0 + (a.idz * sz + a.idx * sx);
            ad[EL_VZ * a.fs + o] = v;
            gbz += v * __ldg(a.S + 4 * a.sterm + so);
            const float q = bz * v;
            float ex = q, ez = q;
            if (pih) {
                ex = pml_e(q, cih.x, cih.y, m_xxz, mh + M_DXXZ * a.fs);
                ez = pml_e(q, cih.z, cih.w, m_zzz, mh + M_DZZZ * a.fs);
            }
            e[M_DXXZ * a.fs] = ex;
            e[M_DZZZ * a.fs] = ZR ? ez * zsh : ez;
        }
    }
    const long long go = (long long)blockIdx.z * a.fs + o;
    kahan_g(a.G, a.gg, go, 4, gbx);
    if (dvz) kahan_g(a.G, a.gg, go, 5, gbz);
}

// stress nodes: finish the adjoint of the velocity update of step t
// (sigma^ += D^T e of the velocity nodes, free-surface images folded back with
// a minus), correlate sigma^ with the stored terms of step t (Cij gradients),
// then the adjoint PML terms of the stress update of step t
// 64 registers at R = 4 (a few bytes spilled) instead of the 128 that a
// 512-thread bound allows: four 256-thread CTAs per SM instead of two, which
// hides more of the load latency this kernel is bound by
template <int R, bool ZR>
__global__ void __maxnreg__(R == 4 ? 64 : 128) k_el2d_adj_s(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = a.zs0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const int pt = a.pitch;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool row1 = a.fsurf && z == a.pr;
    const bool dxz = z >= a.zxz0;
    const bool px_i = el_pml_int(x, a.pr, a.nx);
    const bool pii = px_i || (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool phh = el_pml_half(x, a.pr, a.nx) || (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float4 cii = pii ? __ldg(a.pii + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 chh = (phh && dxz) ? __ldg(a.phh + o) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float c11 = __ldg(a.c11 + o), c13 = __ldg(a.c13 + o), c33 = __ldg(a.c33 + o);
    const float c55dt = dxz ? a.dt * __ldg(a.c55e + o) : 0.f;
    const bool mir = a.fsurf && z > a.pr && z <= a.pr + a.R;
    const long long ozz = (long long)(2 * a.pr - z) * pt + x;      // sigma_zz image row
    const long long oxz = (long long)(2 * a.pr + 1 - z) * pt + x;  // sigma_xz image row
    const float r13 = c13 / c33;
    const float zsi = ZR ? __ldg(a.zfi + z) : 1.f, zsh = ZR ? __ldg(a.zfh + z) : 1.f;  // see k_el2d_adj_v
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    float g11 = 0.f, g13 = 0.f, g33 = 0.f, g55 = 0.f;
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        float* e = ad + 13 * a.fs;
        float* mh = ad + 5 * a.fs + o;
        const long long so = slot + s * a.fs + o;
        float* xhp = ad + EL_SXX * a.fs + o;
        float* zhp = ad + EL_SZZ * a.fs + o;
        float* shp = ad + EL_SXZ * a.fs + o;
        // own adjoint stresses and memories ahead of the stores (see k_el2d_fwd_s)
        const float xx0 = *xhp, zz0 = row1 ? 0.f : *zhp, xz0 = dxz ? *shp : 0.f;
        const float m_xvx = (row1 ? px_i : pii) ? mh[M_DXVX * a.fs] : 0.f;
        const float m_zvz = !row1 && pii ? mh[M_DZVZ * a.fs] : 0.f;
        const float m_xvz = dxz && phh ? mh[M_DXVZ * a.fs] : 0.f, m_zvx = dxz && phh ? mh[M_DZVX * a.fs] : 0.f;
        // sigma_xx, sigma_zz
        const float* e5 = e + M_DXXX * a.fs + o;
        const float* e8 = e + M_DZZZ * a.fs + o;
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (__ldg(e5 + (1 - k)) - __ldg(e5 + (k)));
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fde[k - 1] * (__ldg(e8 + ((1 - k) * pt)) - __ldg(e8 + (k * pt)));
        const float xh = xx0 + a.idx * sx;
        float zh = 0.f;
        if (!row1) {
            float dz = a.idz * sz;
            if (mir) {
                // the image row 2 - j collects -e_dzzz(image + k) from the vz
                // nodes below it (no vz node lies above the surface)
                const float* em = e + M_DZZZ * a.fs + ozz;
                float sm = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) sm = sm + c_fde[k - 1] * __ldg(em + (k * pt));
                dz = dz + a.idz * sm;
            }
            zh = zz0 + dz;
        }
        *xhp = xh;
        *zhp = zh;
        const float S0 = __ldg(a.S + so), S1 = __ldg(a.S + a.sterm + so);
        float ex, ez = 0.f;
        if (row1) {
            g11 += xh * S0;
            g13 += -2.f * r13 * xh * S0;
            g33 += r13 * r13 * xh * S0;
            const float q = a.dt * c11 * xh - r13 * (a.dt * c13 * xh);
            ex = px_i ? pml_e(q, cii.x, cii.y, m_xvx, mh + M_DXVX * a.fs) : q;
        } else {
            g11 += xh * S0;
            g13 += xh * S1 + zh * S0;
            g33 += zh * S1;
            const float qx = a.dt * (c11 * xh + c13 * zh);
            const float qz = a.dt * (c13 * xh + c33 * zh);
            ex = qx;
            ez = qz;
            if (pii) {
                ex = pml_e(qx, cii.x, cii.y, m_xvx, mh + M_DXVX * a.fs);
                ez = pml_e(qz, cii.z, cii.w, m_zvz, mh + M_DZVZ * a.fs);
            }
            e[M_DZVZ * a.fs + o] = ZR ? ez * zsi : ez;
        }
        e[M_DXVX * a.fs + o] = ex;
        // sigma_xz
        if (dxz) {
            const float* e6 = e + M_DZXZ * a.fs + o;
            const float* e7 = e + M_DXXZ * a.fs + o;
            float tz = 0.f, tx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) tz = tz + c_fde[k - 1] * (__ldg(e6 + (-k * pt)) - __ldg(e6 + ((k - 1) * pt)));
#pragma unroll
            for (int k = 1; k <= R; ++k) tx = tx + c_fde[k - 1] * (__ldg(e7 + (-k)) - __ldg(e7 + (k - 1)));
            float dsum = a.idz * tz + a.idx * tx;
            if (mir) {
                // the image row collects -e_dzxz(image + k - 1) from the vx nodes at
                // and below the surface; no vx node lies above it and no vz node
                // on or above it, so the other terms vanish
                const float* em6 = e + M_DZXZ * a.fs + oxz;
                float mz = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) mz = mz + c_fde[k - 1] * __ldg(em6 + ((k - 1) * pt));
                dsum = dsum + a.idz * mz;
            }
            const float sh = xz0 + dsum;
            *shp = sh;
            g55 += sh * __ldg(a.S + 2 * a.sterm + so);
            const float q = c55dt * sh;
            float ezx = q, exz = q;
            if (phh) {
                exz = pml_e(q, chh.x, chh.y, m_xvz, mh + M_DXVZ * a.fs);
                ezx = pml_e(q, chh.z, chh.w, m_zvx, mh + M_DZVX * a.fs);
            }
            e[M_DZVX * a.fs + o] = ZR ? ezx * zsh : ezx;
            e[M_DXVZ * a.fs + o] = exz;
        }
    }
    const long long go = (long long)blockIdx.z * a.fs + o;
    kahan_g(a.G, a.gg, go, 0, g11);
    kahan_g(a.G, a.gg, go, 1, g13);
    kahan_g(a.G, a.gg, go, 2, g33);
    if (dxz) kahan_g(a.G, a.gg, go, 3, g55);
}

// ------------------------- FP64 chain rule ---------------------------------
// d J / d (c11, c13, c33, c55, rho) on the padded model grid [-P, n+P+1] from
// the time-summed correlations (value = sum - compensation), then the model
// parameters through the per-cell Jacobian jac[p][5][cell] of the Cij set-up:
//   sigma += dt (C . D)           -> dJ/dc   = dt G_c
//   sigma_xz += dt c55e D         -> dJ/dc55 = dt G_55 c55e^2 / (4 c55^2), 4 nodes
//   v += (dt / rho_eff) H         -> dJ/drho = -0.5 dt G_b / rho_eff^2, 2 + 2 nodes
// With jac null (the depth-refined mesh) the five d J / d (c11, c13, c33, c55,
// rho) of the mesh cells go to gpad's planes 0..4 as they are; k_el2d_zmap
// carries them to the regular rows and through the Jacobian.
__global__ void k_el2d_chain(El2dDev a, int ngroups, const float* __restrict__ c55p, const float* __restrict__ rhop,
                             const double* __restrict__ jac, int np, long long npad, double* __restrict__ gpad,
                             int nxq, int nzq) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= nxq || iz >= nzq) return;
    const int x = a.R - 1 + ix, z = a.R - 1 + iz;
    const long long o = (long long)z * a.pitch + x;
    auto sumG = [&](int q, long long oo) {
        double v = 0;
        for (int g = 0; g < ngroups; ++g)
            v += (double)a.G[q * a.gg + g * a.fs + oo] - (double)a.G[(6 + q) * a.gg + g * a.fs + oo];
        return v;
    };
    const double dt = a.dt;
    double dc[5] = {0, 0, 0, 0, 0};
    if (x >= a.x0 && x < a.x1 && z >= a.zs0 && z < a.z1) {
        dc[0] = dt * sumG(0, o);
        dc[1] = dt * sumG(1, o);
        dc[2] = dt * sumG(2, o);
    }
    const double c55 = c55p[o];
    for (int dz = 0; dz <= 1; ++dz)
        for (int dx = 0; dx <= 1; ++dx) {
            const int m = x + dx, n = z + dz;
            if (m < a.x0 || m >= a.x1 || n < a.zxz0 || n >= a.z1) continue;
            const long long on = (long long)n * a.pitch + m;
            const double ce = a.c55e[on];
            if (ce != 0.0) dc[3] += dt * sumG(3, on) * ce * ce / (4.0 * c55 * c55);
        }
    for (int d = 0; d <= 1; ++d) {
        const int m = x + d;
        if (m >= a.x0 && m < a.x1 && z >= a.zvx0 && z < a.z1) {
            const long long om = (long long)z * a.pitch + m;
            const double re = 0.5 * ((double)rhop[om - 1] + (double)rhop[om]);
            dc[4] -= 0.5 * dt * sumG(4, om) / (re * re);
        }
        const int n = z + d;
        if (x >= a.x0 && x < a.x1 && n >= a.zvz0 && n < a.z1) {
            const long long on = (long long)n * a.pitch + x;
            const double re = 0.5 * ((double)rhop[on - a.pitch] + (double)rhop[on]);
            dc[4] -= 0.5 * dt * sumG(5, on) / (re * re);
        }
    }
    const long long cell = (long long)iz * nxq + ix;
    if (!jac) {
        for (int q = 0; q < 5; ++q) gpad[(long long)q * npad + cell] += dc[q];
        return;
    }
    for (int p = 0; p < np; ++p) {
        double g = 0;
        for (int q = 0; q < 5; ++q) g += jac[((long long)p * 5 + q) * npad + cell] * dc[q];
        gpad[(long long)p * npad + cell] += g;
    }
}

// Gradient of the regular padded rows from the mesh cells' d J / d (c11, c13,
// c33, c55, rho): the transpose of the row interpolation that maps the regular
// Cij to the mesh (regular row r gets sum over mesh rows f of w(f, r) g(f), the
// pairs in zptr / zrow / zw), then the per-cell Jacobian to the model
// parameters. One thread per regular padded cell, FP64.
__global__ void k_el2d_zmap(const double* __restrict__ gmesh, long long npad_m, const int* __restrict__ zptr,
                            const int* __restrict__ zrow, const double* __restrict__ zw,
                            const double* __restrict__ jac, int np, long long npad_r, double* __restrict__ gout,
                            int nxq, int nzq_r) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x, iz = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= nxq || iz >= nzq_r) return;
    double dc[5] = {0, 0, 0, 0, 0};
    for (int e = zptr[iz]; e < zptr[iz + 1]; ++e) {
        const long long cm = (long long)zrow[e] * nxq + ix;
        const double w = zw[e];
        for (int q = 0; q < 5; ++q) dc[q] += w * gmesh[(long long)q * npad_m + cm];
    }
    const long long cell = (long long)iz * nxq + ix;
    for (int p = 0; p < np; ++p) {
        double g = 0;
        for (int q = 0; q < 5; ++q) g += jac[((long long)p * 5 + q) * npad_r + cell] * dc[q];
        gout[(long long)p * npad_r + cell] = g;
    }
}

// ============================================================================
// host: model set-up restated from the reference
// ============================================================================
namespace {

template <typename T>
inline double re_(const T& v) { return std::real(v); }

template <typename T>
inline T abs_cs(const T& v) { return re_(v) < 0 ? -v : v; }

int el_nparam(int aniso) {
    switch (aniso) {
        case OWL_ANISO_ISO: return 3;
        case OWL_ANISO_THOMSEN:
        case OWL_ANISO_AT: return 6;
        case OWL_ANISO_CIJ: return 5;
    }
    return -1;
}

// Cij of one cell (thomsen_to_cij2d / alkhalifah_tsvankin_to_cij2d,
// src/lib/module_anisotropy.f90:310-402, and the iso / cij cases of
// src/solver/elastic_vhtiort_2d/module_vars.f90:235-286), evaluated in T with
// the reference's operation order. A tilt rotates the tensor about y; only
// c11, c13, c33, c55 are used by the 2D stencils.
template <typename T>
void cij_of(int aniso, const T* p, T& c11, T& c13, T& c33, T& c55, T& rho) {
    T the = T(0);
    switch (aniso) {
        case OWL_ANISO_ISO:
            rho = p[2];
            c33 = rho * (p[0] * p[0]);
            c55 = rho * (p[1] * p[1]);
            c11 = c33;
            c13 = c33 - T(2) * c55;
            return;
        case OWL_ANISO_THOMSEN: {
            rho = p[5];
            the = p[4];
            c33 = (p[0] * p[0]) * rho;
            c55 = (p[1] * p[1]) * rho;
            c11 = c33 * (T(1) + T(2) * p[2]);
            const T tmp = T(2) * c33 * (c33 - c55) * p[3] + (c33 - c55) * (c33 - c55);
            c13 = std::sqrt(abs_cs(tmp)) - c55;
            break;
        }
        case OWL_ANISO_AT: {
            rho = p[5];
            the = p[4];
            const T vp2 = p[0] * p[0], vs2 = p[1] * p[1];
            c11 = vp2 * rho;
            c55 = vs2 * rho;
            c33 = c11 / (T(1) + T(2) * p[2]);
            c13 = rho * (std::sqrt(abs_cs((vp2 / (T(1) + T(2) * p[2]) - vs2) * (vp2 / (T(1) + T(2) * p[3]) - vs2))) - vs2);
            break;
        }
        default:
            c11 = p[0]; c13 = p[1]; c33 = p[2]; c55 = p[3]; rho = p[4];
            return;
    }
    if (re_(the) != 0.0) {
        const T cs = std::cos(-the), sn = std::sin(-the);
        const T c2 = cs * cs, s2 = sn * sn, x = c2 * s2, q4 = c2 * c2 + s2 * s2;
        const T a11 = c11, a13 = c13, a33 = c33, a55 = c55;
        c11 = a11 * (c2 * c2) + T(2) * (a13 + T(2) * a55) * x + a33 * (s2 * s2);
        c33 = a11 * (s2 * s2) + T(2) * (a13 + T(2) * a55) * x + a33 * (c2 * c2);
        c13 = (a11 + a33 - T(4) * a55) * x + a13 * q4;
        c55 = (a11 + a33 - T(2) * a13 - T(2) * a55) * x + a55 * q4;
    }
}

// M-PML damping ratio of one boundary cell (damp_ratio,
// src/solver/elastic_vhtiort_2d/module_cfspml.f90:174-223), called as the 2D
// solver does with c15 = c35 = 0 (:240-270). The Christoffel eigenvalues are
// then purely imaginary, so the reference's complex arithmetic is real
// arithmetic on their squares (E2 < 0) and fourth powers.
float eig_sq(float c11, float c13, float c33, float c55, float rho, bool mode1, float k1, float k3) {
    const float A = (c11 + c55) * (k1 * k1) + (c33 + c55) * (k3 * k3);
    const float B = -(c11 * c55) * ((k1 * k1) * (k1 * k1)) + (c13 * c13 - c11 * c33 + 2 * c13 * c55) * (k1 * k1) * (k3 * k3) -
                    (c33 * c55) * ((k3 * k3) * (k3 * k3));
    const float sq = std::sqrt((A * A + 4 * B) * (rho * rho));
    const float v = mode1 ? -((A * rho + sq) / (rho * rho)) : (-(A * rho) + sq) / (rho * rho);
    const float b = std::sqrt(std::fabs(v)) / std::sqrt(2.0f);
    return v <= 0 ? -(b * b) : b * b;
}

float eig_deriv(float c11, float c13, float c33, float c55, float rho, bool zdir, float E2, float r, float k1, float k3) {
    const float E4 = E2 * E2, k12 = k1 * k1, k32 = k3 * k3;
    const float A = (c11 + c55) * k12 + (c33 + c55) * k32;
    const float B = -(c11 * c55) * (k12 * k12) + (c13 * c13 - c11 * c33 + 2 * c13 * c55) * k12 * k32 - (c33 * c55) * (k32 * k32);
    const float den = 2 * B - 3 * E2 * A * rho - 4 * E4 * (rho * rho);
    float num;
    if (!zdir)
        num = 2 * c33 * c55 * (k32 * k32) - c13 * c13 * k12 * k32 * (1 + r) - c13 * k1 * k3 * (k3 * (2 * c55 * k1 * (1 + r))) +
              E2 * (k3 * (c33 * k3 * (2 + r)) + c55 * (k32 * (2 + r) + k12 * (1 + 2 * r))) * rho +
              2 * E4 * (1 + r) * (rho * rho) + c11 * k12 * (2 * c55 * k12 * r + c33 * k32 * (1 + r) + E2 * (1 + 2 * r) * rho);
    else
        num = k32 * (-(2 * (-(c33 * c55)) * k32 * r) - c13 * c13 * k12 * (1 + r) - c13 * k1 * (2 * c55 * k1 * (1 + r))) +
              E2 * (k3 * (c33 * k3 * (1 + 2 * r)) + c55 * (k12 * (2 + r) + k32 * (1 + 2 * r))) * rho +
              2 * E4 * (1 + r) * (rho * rho) + c11 * k12 * (2 * c55 * k12 + k3 * (c33 * k3 * (1 + r)) + E2 * (2 + r) * rho);
    return num / den;
}

float mpml_ratio(float c11, float c13, float c33, float c55, float rho, bool zdir) {
    const float dtheta = (float)(3.14159265358979323846 / 180.0);
    const float sc = 1.0e-9f;
    float r = 0.f;
    for (int i = 1; i <= 180; ++i) {
        const float th = ((float)i + 0.5f) * dtheta;
        const float kx = std::sin(th), kz = std::cos(th);
        const float e1 = eig_sq(c11, c13, c33, c55, rho, true, kx, kz);
        const float e2 = eig_sq(c11, c13, c33, c55, rho, false, kx, kz);
        auto worst = [&]() {
            return std::max(eig_deriv(c11 * sc, c13 * sc, c33 * sc, c55 * sc, rho * sc, zdir, e1, r, kx, kz),
                            eig_deriv(c11 * sc, c13 * sc, c33 * sc, c55 * sc, rho * sc, zdir, e2, r, kx, kz));
        };
        float d = worst();
        while (d >= -0.01f && r < 1.0f) {
            r = r + 0.002f;
            d = worst();
        }
    }
    return r;
}

// CFS-MPML coefficients of one node (damp_coef, module_cfspml.f90:286-327,
// kmax = 1); distances normalised by the PML width
float4 mpml_coef(float vp, float xd, float zd, float dx, float dz, int pml, float dt, float alphamax, float rx,
                 float rz) {
    const float R0 = 1.0e-5f;
    float dampx = vp * 3.0f * std::log(1.0f / R0) / (2.0f * (float)pml * dx) * (xd * xd);
    float dampz = vp * 3.0f * std::log(1.0f / R0) / (2.0f * (float)pml * dz) * (zd * zd);
    const float wx = dampx + rz * dampz, wz = dampz + rx * dampx;
    dampx = wx;
    dampz = wz;
    const float adt = std::fabs(dt);
    const float alx = std::max(alphamax * (1.0f - xd), 0.25f * alphamax);
    const float alz = std::max(alphamax * (1.0f - zd), 0.25f * alphamax);
    float4 c;
    c.x = -2.0f * adt * dampx / (2.0f + adt * (alx + dampx));
    c.y = (2.0f - adt * (alx + dampx)) / (2.0f + adt * (alx + dampx));
    c.z = -2.0f * adt * dampz / (2.0f + adt * (alz + dampz));
    c.w = (2.0f - adt * (alz + dampz)) / (2.0f + adt * (alz + dampz));
    return c;
}

VMesh checked_vmesh(const owl_ssg_desc& d) {
    try {
        return build_vmesh(d);
    } catch (const std::invalid_argument& e) {
        throw OwlError(OWL_ERR_INVALID, e.what());
    }
}

owl_ssg_desc with_rows(owl_ssg_desc d, int nz) {
    d.nz = nz;
    return d;
}

}  // namespace

// ============================================================================
// host engine
// ============================================================================
// With the depth-refined free-surface mesh the engine runs on the mesh's rows
// (nz of the base = the computational rows); the model and the gradient stay on
// the regular nz_model rows.
struct El2dEngine : SsgBase {
    int aniso;
    float idx, idz;
    VMesh vm;
    int nz_model;
    ZInterp zt;
    DevBuf<float> c11, c13, c33, c55e, bxp, bzp, c55p, rhop, zfi, zfh;
    DevBuf<float4> pii, phh, phi, pih;
    DevBuf<double> jac, zw, gzmap;
    DevBuf<int> zptr, zrow;

    explicit El2dEngine(const owl_ssg_desc& d) : El2dEngine(d, checked_vmesh(d)) {}
    El2dEngine(const owl_ssg_desc& d, VMesh m) : SsgBase(with_rows(d, m.nz), 2), vm(std::move(m)), nz_model(d.nz) {
        aniso = d.aniso;
        OWL_CHECK(el_nparam(aniso) > 0, OWL_ERR_INVALID, "unknown elastic parameterisation (aniso)");
        idx = (float)(1.0 / (double)d.dx);
        idz = (float)(1.0 / (double)d.dz);
        OWL_CUDA(cudaMemcpyToSymbol(c_fde, fd_coefs(R), sizeof(float) * R));
        sst = EL_NST * fs;
        sad = EL_NAD * fs;
        nS = 5;
        ngrad = 6;
        nparam = el_nparam(aniso);
        ncomp = 2;
        for (int f = 0; f < EL_NST; ++f) st_segments.push_back({f * fs, fs});
        // dz scalings of the storage rows (1 outside the mesh arrays and on the uniform grid)
        std::vector<float> hi(NZs, 1.f), hh(NZs, 1.f);
        if (vm.refined) {
            for (int z = 0; z < NZs; ++z) {
                const int j = z - pr + 1;
                if (j < -P || j > nz + P + 1) continue;
                hi[z] = vm.get(vm.si, j);
                hh[z] = vm.get(vm.sh, j);
            }
            zt = build_zinterp(vm, nz_model, d.dz);
            // transpose of the row interpolation, per regular padded row
            const int nzr = nz_model + 2 * P + 2;
            std::vector<std::vector<std::pair<int, double>>> by(nzr);
            for (int f = -P; f <= nz + P + 1; ++f) {
                const int r0 = zt.r0[(size_t)(f + P)];
                const double w = zt.w[(size_t)(f + P)];
                by[(size_t)(r0 + P)].push_back({f + P, 1.0 - w});
                by[(size_t)(r0 + 1 + P)].push_back({f + P, w});
            }
            std::vector<int> hp(1, 0), hr;
            std::vector<double> hw;
            for (auto& v : by) {
                for (auto& e : v) { hr.push_back(e.first); hw.push_back(e.second); }
                hp.push_back((int)hr.size());
            }
            zptr.upload(hp.data(), hp.size(), stream);
            zrow.upload(hr.data(), hr.size(), stream);
            zw.upload(hw.data(), hw.size(), stream);
        }
        zfi.upload(hi.data(), hi.size(), stream);
        zfh.upload(hh.data(), hh.size(), stream);
        OWL_CUDA(cudaStreamSynchronize(stream));
    }

    // refined mesh: gpad holds the mesh cells' d J / d (c11, c13, c33, c55, rho)
    int grad_planes() const override { return vm.refined ? 5 : nparam; }

    float* st_field(int f) const override { return f < 5 ? st.p + f * fs : nullptr; }
    float* ad_field(int f) const override { return f < 5 ? ad.p + f * fs : nullptr; }
    int rho_param() const override { return vm.refined ? 4 : nparam - 1; }

    void set_model(int np, const float* const* f) override {
        OWL_CHECK(np == nparam && f, OWL_ERR_INVALID,
                  "elastic 2D model needs " + std::to_string(nparam) + " parameters for this parameterisation");
        for (int q = 0; q < np; ++q) OWL_CHECK(f[q], OWL_ERR_INVALID, "null model parameter");
        const int nxq_ = nxq(), nzr = nz_model;
        const size_t npr = (size_t)nxq_ * (nzr + 2 * P + 2);  // regular padded cells
        // padded parameters and Cij of the regular rows (padding by pml+1 with
        // edge values, module_vars.f90:297-301)
        std::vector<float> r11(npr), r13(npr), r33(npr), r55(npr), rrho(npr);
        std::vector<double> hjac((size_t)np * 5 * npr, 0.0);
        std::vector<float> p(np);
        std::vector<std::complex<double>> pc(np);
        auto rc = [&](int i, int j) { return (size_t)(j + P) * nxq_ + (size_t)(i + P); };
        for (int j = -P; j <= nzr + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                const int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), nzr);
                const size_t src = (size_t)(ii - 1) * nzr + (jj - 1);
                for (int q = 0; q < np; ++q) p[q] = f[q][src];
                for (int q = 0; q < np; ++q)
                    OWL_CHECK(std::isfinite(p[q]), OWL_ERR_INVALID, "model parameters must be finite");
                float a11, a13, a33, a55, r;
                cij_of<float>(aniso, p.data(), a11, a13, a33, a55, r);
                OWL_CHECK(r > 0 && a11 > 0 && a33 > 0 && a55 > 0, OWL_ERR_INVALID,
                          "rho, c11, c33 and c55 must be positive");
                const size_t cell = rc(i, j);
                r11[cell] = a11; r13[cell] = a13; r33[cell] = a33; r55[cell] = a55; rrho[cell] = r;
                // Jacobian d(c11, c13, c33, c55, rho) / d(param) by complex step in FP64
                for (int q = 0; q < np; ++q) {
                    for (int r2 = 0; r2 < np; ++r2) pc[r2] = std::complex<double>(p[r2], r2 == q ? 1e-30 : 0.0);
                    std::complex<double> o5[5];
                    cij_of(aniso, pc.data(), o5[0], o5[1], o5[2], o5[3], o5[4]);
                    for (int k = 0; k < 5; ++k) hjac[((size_t)q * 5 + k) * npr + cell] = o5[k].imag() / 1e-30;
                }
            }
        // the engine's rows: the regular ones, or on the refined mesh the Cij
        // interpolated linearly in depth (map_regular_to_irregular, module_vars.f90:139-169)
        std::vector<float> hc11(fs, 0.f), hc13(fs, 0.f), hc33(fs, 0.f), hc55(fs, 0.f), hrho(fs, 0.f);
        for (int j = -P; j <= nz + P + 1; ++j)
            for (int i = -P; i <= nx + P + 1; ++i) {
                const long long o = soff(i, 1, j);
                if (!vm.refined) {
                    const size_t cell = rc(i, j);
                    hc11[o] = r11[cell]; hc13[o] = r13[cell]; hc33[o] = r33[cell]; hc55[o] = r55[cell];
                    hrho[o] = rrho[cell];
                    continue;
                }
                const int r0 = zt.r0[(size_t)(j + P)];
                const size_t c0 = rc(i, r0), c1 = rc(i, r0 + 1);
                hc11[o] = zinterp_apply(zt, j, P, r11[c0], r11[c1]);
                hc13[o] = zinterp_apply(zt, j, P, r13[c0], r13[c1]);
                hc33[o] = zinterp_apply(zt, j, P, r33[c0], r33[c1]);
                hc55[o] = zinterp_apply(zt, j, P, r55[c0], r55[c1]);
                hrho[o] = zinterp_apply(zt, j, P, rrho[c0], rrho[c1]);
            }
        // harmonic c55 at the sigma_xz nodes and buoyancies (module_wavefield.f90:31-35)
        std::vector<float> hc55e(fs, 0.f), hbx(fs, 0.f), hbz(fs, 0.f);
        for (int n = -P + 1; n <= nz + P; ++n)
            for (int m = -P + 1; m <= nx + P; ++m) {
                const long long o = soff(m, 1, n);
                const float s = 1.0f / hc55[soff(m - 1, 1, n - 1)] + 1.0f / hc55[soff(m, 1, n - 1)] +
                                1.0f / hc55[soff(m - 1, 1, n)] + 1.0f / hc55[o];
                hc55e[o] = 4.0f / s;
                hbx[o] = dt / (0.5f * (hrho[soff(m - 1, 1, n)] + hrho[o]));
                hbz[o] = dt / (0.5f * (hrho[soff(m, 1, n - 1)] + hrho[o]));
            }
        // pmlvp from the regular model's edges (module_vars.f90:298-302) and the
        // stability bound (:381-420; on the refined mesh the least over the
        // cells with the row's smaller spacing)
        float pv = -1e30f, maxv = 0.f;
        auto edge = [&](int i, int j) {
            const size_t cell = rc(i, j);
            pv = std::max({pv, r11[cell] / rrho[cell], r33[cell] / rrho[cell]});
        };
        for (int j = 1; j <= nzr; ++j) { edge(1, j); edge(nx, j); }
        for (int i = 1; i <= nx; ++i) { edge(i, 1); edge(i, nzr); }
        const float pmlvp = std::sqrt(pv);
        const float* c = fd_coefs(R);
        float temp = 0.f;
        for (int k = 0; k < R; ++k) temp += std::fabs(c[k]);
        if (!vm.refined) {
            for (int j = 1; j <= nz; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const long long o = soff(i, 1, j);
                    maxv = std::max({maxv, std::sqrt(hc11[o] / hrho[o]), std::sqrt(hc33[o] / hrho[o])});
                }
            dt_stable_ = 1.0f / (temp * maxv * std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (desc.dz * desc.dz)));
        } else {
            float best = 3.0e38f;
            for (int j = 1; j <= nz; ++j) {
                const float hz = std::min(vm.get(vm.dzi, j), vm.get(vm.dzh, j));
                for (int i = 1; i <= nx; ++i) {
                    const long long o = soff(i, 1, j);
                    const float mv = std::max(std::sqrt(hc11[o] / hrho[o]), std::sqrt(hc33[o] / hrho[o]));
                    best = std::min(best, 1.0f / (temp * mv * std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (hz * hz))));
                }
            }
            dt_stable_ = best;
        }
        if (dt > dt_stable_ && !desc.allow_dt_adjust)
            throw OwlError(OWL_ERR_UNSTABLE, "dt = " + std::to_string(dt) + " exceeds the stable dt " +
                                                 std::to_string(dt_stable_));
        // M-PML ratios on the four model edges (module_cfspml.f90:229-276), zero when isotropic
        std::vector<float> rl(nz + 2 * P + 2, 0.f), rr(nz + 2 * P + 2, 0.f), rt(nx + 2 * P + 2, 0.f),
            rb(nx + 2 * P + 2, 0.f);
        if (aniso != OWL_ANISO_ISO) {
            auto ratio = [&](int i, int j, bool zdir) {
                const long long o = soff(i, 1, j);
                return mpml_ratio(hc11[o], hc13[o], hc33[o], hc55[o], hrho[o], zdir);
            };
            for (int j = -P; j <= nz + P + 1; ++j) { rl[j + P] = ratio(1, j, false); rr[j + P] = ratio(nx, j, false); }
            for (int i = -P; i <= nx + P + 1; ++i) { rt[i + P] = ratio(i, 1, true); rb[i + P] = ratio(i, nz, true); }
        }
        // 2D CFS-MPML coefficients of the four staggered positions (module_cfspml.f90:329-575)
        std::vector<float4> hii(fs, make_float4(0, 0, 0, 0)), hhh(fs, make_float4(0, 0, 0, 0)),
            hhi(fs, make_float4(0, 0, 0, 0)), hih(fs, make_float4(0, 0, 0, 0));
        const float alphamax = (float)(1.0 * (double)desc.f0_max * 3.14159265358979323846);
        for (int j = -P + 1; j <= nz + P; ++j)
            for (int i = -P + 1; i <= nx + P; ++i) {
                if (i > 1 && i < nx && j > 1 && j < nz) continue;
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
                float rx = 0.f, rz = 0.f;
                if (i <= 1) rx = rl[j + P]; else if (i >= nx) rx = rr[j + P];
                if (j <= 1) rz = rt[i + P]; else if (j >= nz) rz = rb[i + P];
                const long long o = soff(i, 1, j);
                // the row's own spacing dz_i(j) on the refined mesh (module_cfspml.f90:446-473)
                const float dzj = vm.refined ? vm.get(vm.dzi, j) : desc.dz;
                hii[o] = mpml_coef(pmlvp, xdi, zdi, desc.dx, dzj, P, dt, alphamax, rx, rz);
                hih[o] = mpml_coef(pmlvp, xdi, zdh, desc.dx, dzj, P, dt, alphamax, rx, rz);
                hhi[o] = mpml_coef(pmlvp, xdh, zdi, desc.dx, dzj, P, dt, alphamax, rx, rz);
                hhh[o] = mpml_coef(pmlvp, xdh, zdh, desc.dx, dzj, P, dt, alphamax, rx, rz);
            }
        c11.upload(hc11.data(), fs, stream);
        c13.upload(hc13.data(), fs, stream);
        c33.upload(hc33.data(), fs, stream);
        c55e.upload(hc55e.data(), fs, stream);
        bxp.upload(hbx.data(), fs, stream);
        bzp.upload(hbz.data(), fs, stream);
        c55p.upload(hc55.data(), fs, stream);
        rhop.upload(hrho.data(), fs, stream);
        pii.upload(hii.data(), fs, stream);
        phh.upload(hhh.data(), fs, stream);
        phi.upload(hhi.data(), fs, stream);
        pih.upload(hih.data(), fs, stream);
        jac.upload(hjac.data(), hjac.size(), stream);
        OWL_CUDA(cudaStreamSynchronize(stream));
        h_rhop = std::move(hrho);
        model_set = true;
        invalidate_graphs();
    }

    // ---- sources / receivers (module_wavefield.f90:294-403, submodule_forward_modeling.f90:86-112)
    int src_ncomp(const owl_source& q) const override {
        OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION || q.mechanism == OWL_SRC_FORCE || q.mechanism == OWL_SRC_MT,
                  OWL_ERR_UNSUPPORTED, "unknown source mechanism");
        return q.mechanism == OWL_SRC_FORCE ? 2 : 1;
    }
    void src_taps(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rc, float& rv) const override {
        const bool fsf = desc.free_surface != 0;
        if (q.mechanism == OWL_SRC_FORCE) {
            const int ci = comp == 0 ? q.hx : q.gx, ck = comp == 0 ? q.gz : q.hz;
            OWL_CHECK(in_wavefield(ci, 1, ck), OWL_ERR_INVALID, "force source outside the grid");
            rv = h_rhop[soff(ci, 1, ck)];
            rc = pad_index(ci, 1, ck);
            for (int irz = -4; irz <= 4; ++irz)
                for (int irx = -4; irx <= 4; ++irx) {
                    if (comp == 0) {
                        if (fsf && q.gz + irz < 2) continue;
                        taps.push_back(TapPt{EL_VX, q.hx + irx, 1, q.gz + irz,
                                             std::sin(q.polar) / rv * q.interp_hx[irx + 4] * q.interp_iz[irz + 4]});
                    } else {
                        if (fsf && q.hz + irz < 2) continue;
                        taps.push_back(TapPt{EL_VZ, q.gx + irx, 1, q.hz + irz,
                                             std::cos(q.polar) / rv * q.interp_ix[irx + 4] * q.interp_hz[irz + 4]});
                    }
                }
            return;
        }
        // explosion / moment tensor: stress drop amp / (dx dz_s), dz_s the local
        // spacing dz_i(gz) on the refined mesh, module_wavefield.f90:305-399
        const bool mt = q.mechanism == OWL_SRC_MT;
        OWL_CHECK(!vm.refined || (q.gz >= -P && q.gz <= nz + P + 1), OWL_ERR_INVALID, "source outside the grid");
        const float dzs = vm.refined ? vm.get(vm.dzi, q.gz) : desc.dz;
        const float inv = 1.0f / (desc.dx * dzs);
        const float mxx = mt ? q.mt[0] : 1.f, mzz = mt ? q.mt[2] : 1.f, mxz = q.mt[4];
        for (int irz = -4; irz <= 4; ++irz)
            for (int irx = -4; irx <= 4; ++irx) {
                if (!fsf || q.gz + irz >= 2) {
                    const float w = q.interp_ix[irx + 4] * q.interp_iz[irz + 4];
                    taps.push_back(TapPt{EL_SXX, q.gx + irx, 1, q.gz + irz, -inv * mxx * w});
                    taps.push_back(TapPt{EL_SZZ, q.gx + irx, 1, q.gz + irz, -inv * mzz * w});
                }
                if (mt && (!fsf || q.hz + irz >= 2))
                    taps.push_back(TapPt{EL_SXZ, q.hx + irx, 1, q.hz + irz,
                                         -inv * mxz * q.interp_hx[irx + 4] * q.interp_hz[irz + 4]});
            }
    }
    // comp 0: vx at (hx, gz); comp 1: vz at (gx, hz). With a free surface the
    // reference samples the even images vx(1-j) = vx(1+j), vz(2-j) = vz(1+j),
    // j = 1..R (submodule_forward_modeling.f90:75-83); rows beyond them are zero.
    void rec_taps(const owl_receiver& q, int comp, std::vector<TapPt>& taps) const override {
        const bool fsf = desc.free_surface != 0;
        for (int irz = -4; irz <= 4; ++irz)
            for (int irx = -4; irx <= 4; ++irx) {
                if (comp == 0) {
                    int k = q.gz + irz;
                    const float w = q.interp_hx[irx + 4] * q.interp_iz[irz + 4] * q.weight;
                    if (fsf && k <= 0) {
                        if (k < 1 - R) continue;
                        k = 2 - k;
                    }
                    taps.push_back(TapPt{EL_VX, q.hx + irx, 1, k, w});
                } else {
                    int k = q.hz + irz;
                    const float w = q.interp_ix[irx + 4] * q.interp_hz[irz + 4] * q.weight;
                    if (fsf && k <= 1) {
                        if (k < 2 - R) continue;
                        k = 3 - k;
                    }
                    taps.push_back(TapPt{EL_VZ, q.gx + irx, 1, k, w});
                }
            }
    }

    El2dDev dev(int S) const {
        El2dDev a{};
        a.nx = nx; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch;
        a.fs = fs; a.sst = sst; a.sad = sad;
        a.x0 = R; a.x1 = R + NXp; a.z1 = R + NZp;
        a.fsurf = desc.free_surface != 0;
        a.zs0 = a.fsurf ? pr : R;
        a.zxz0 = a.fsurf ? pr + 1 : R;
        a.zvx0 = a.fsurf ? pr : R;
        a.zvz0 = a.fsurf ? pr + 1 : R;
        a.idx = idx; a.idz = idz; a.dt = dt;
        a.nshots = S;
        a.c11 = c11.p; a.c13 = c13.p; a.c33 = c33.p; a.c55e = c55e.p; a.bx = bxp.p; a.bz = bzp.p;
        a.pii = pii.p; a.phh = phh.p; a.phi = phi.p; a.pih = pih.p;
        a.zfi = zfi.p; a.zfh = zfh.p;
        a.st = st.p;
        a.k = std::max(1, cur_k);
        a.d_step = ctr.p;
        const long long F = (long long)S * fs;
        if (Sbuf.p && Sbuf.n >= (size_t)nS * a.k * F) {
            a.S = Sbuf.p;
            a.sslot = F;
            a.sterm = (long long)a.k * F;
        }
        if (ad.p && ad.n >= (size_t)sad * S) a.ad = ad.p;
        if (G.p) {
            a.G = G.p;
            a.gg = (long long)((S + spt_a - 1) / spt_a) * fs;
        }
        return a;
    }

    // tile heights of the autotuner: 4, 8, 16 rows of one-cell threads (32 x
    // tz); forward pass also 100 + 2, 4, 8: rows of four-cell threads
    // (k_el2d_fwd_*4, 32 x tz threads covering 128 x tz cells)
    std::vector<int> tune_tz(int pass) const override {
        if (pass == 0) return {4, 8, 16, 102, 104, 108};
        return {4, 8, 16};
    }
    void launch_params(const owl_run_opts& o) override {
        const bool vec = o.tile_z >= 100;
        owl_run_opts q = o;
        if (vec) q.tile_z = o.tile_z - 100;
        SsgBase::launch_params(q);
        if (vec) {
            OWL_CHECK(o.tile_z < 200 && tile_x == 32 && q.tile_z >= 1 && q.tile_z <= 8, OWL_ERR_INVALID,
                      "four-cell tiles: tile_x 32 and tile_z 100 + (1 .. 8)");
            tz_f = o.tile_z;  // the adjoint kernels take the rows with one-cell threads
        }
    }

    template <int RR, bool ZR>
    void launch_r(int id, int S, bool store) {
        El2dDev a = dev(S);
        const int rows_s = a.z1 - a.zs0, rows_v = a.z1 - a.zvx0;
        if (id == OWL_K_FWD_P || id == OWL_K_FWD_V) {
            OWL_CHECK(!store || a.S, OWL_ERR_INVALID, "stencil-term buffer not allocated");
            a.spt = spt_f;
            if (tz_f >= 100) {
                // four-cell threads: 32 x ty threads over 128 x ty cells
                const int ty = tz_f - 100;
                const dim3 b(32, ty);
                auto grid = [&](int rows) {
                    return dim3((NXp + 127) / 128, (rows + ty - 1) / ty, (S + spt_f - 1) / spt_f);
                };
                if (id == OWL_K_FWD_P) {
                    if (store) launch_pdl(k_el2d_fwd_s4<RR, true, ZR>, grid(rows_s), b, 0, stream, a);
                    else launch_pdl(k_el2d_fwd_s4<RR, false, ZR>, grid(rows_s), b, 0, stream, a);
                } else {
                    if (store) launch_pdl(k_el2d_fwd_v4<RR, true, ZR>, grid(rows_v), b, 0, stream, a);
                    else launch_pdl(k_el2d_fwd_v4<RR, false, ZR>, grid(rows_v), b, 0, stream, a);
                }
                return;
            }
            const dim3 b(tile_x, tz_f);
            if (id == OWL_K_FWD_P) {
                if (store) launch_pdl(k_el2d_fwd_s<RR, true, ZR>, grid_for(rows_s, S, spt_f, tz_f), b, 0, stream, a);
                else launch_pdl(k_el2d_fwd_s<RR, false, ZR>, grid_for(rows_s, S, spt_f, tz_f), b, 0, stream, a);
            } else {
                if (store) launch_pdl(k_el2d_fwd_v<RR, true, ZR>, grid_for(rows_v, S, spt_f, tz_f), b, 0, stream, a);
                else launch_pdl(k_el2d_fwd_v<RR, false, ZR>, grid_for(rows_v, S, spt_f, tz_f), b, 0, stream, a);
            }
        } else {
            OWL_CHECK(a.ad && a.S && a.G, OWL_ERR_INVALID, "adjoint buffers not allocated");
            a.spt = spt_a;
            const dim3 b(tile_x, tz_a);
            if (id == OWL_K_ADJ_P) launch_pdl(k_el2d_adj_v<RR, ZR>, grid_for(rows_v, S, spt_a, tz_a), b, 0, stream, a);
            else launch_pdl(k_el2d_adj_s<RR, ZR>, grid_for(rows_s, S, spt_a, tz_a), b, 0, stream, a);
        }
    }
    void launch_kernel(int id, int S, bool store) override {
        if (vm.refined) {
            if (R == 4) launch_r<4, true>(id, S, store);
            else launch_r<8, true>(id, S, store);
        } else {
            if (R == 4) launch_r<4, false>(id, S, store);
            else launch_r<8, false>(id, S, store);
        }
    }

    // the adjoint of a step: velocity nodes, then the source-side adjoint (it
    // needs v^ complete and sigma^ before the velocity update's transpose),
    // then the stress nodes, then the residual of the sampling of step t
    void launch_step(int kind, int S, const PointDev& q) override {
        if (kind != 2) {
            SsgBase::launch_step(kind, S, q);
            return;
        }
        launch_kernel(OWL_K_ADJ_P, S, false);
        launches++;
        if (q.src_adj) {
            launch_point_adj(q, S, 1, PA_SRC_NOW, stream);
            launches++;
        }
        launch_kernel(OWL_K_ADJ_V, S, false);
        launches++;
        if (nb_sct <= 4) {
            launch_point_adj(q, S, 1, PA_SCATTER | PA_TICK, stream);
            launches++;
        } else {
            launch_point_adj(q, S, nb_sct, PA_SCATTER, stream);
            launch_point_adj(q, S, 1, PA_TICK, stream);
            launches += 2;
        }
    }

    // compulsory bytes of one launch: each state / adjoint field read and
    // written once per shot, e terms written once and read once, materials once
    // per launch, PML memory and coefficients only inside the PML, gradient
    // accumulators (sum + compensation) once per shot group
    int n_store_p() const override { return 3; }

    double alg_bytes(int id, int S, int groups) const override {
        const bool fsf = desc.free_surface != 0;
        const double rows_s = NZp - (fsf ? P : 0), rows_v = rows_s;
        const double cs = (double)NXp * rows_s, cv = (double)NXp * rows_v;
        double np_ = 0;  // PML cells (either direction)
        for (int z = R + (fsf ? P : 0); z < R + NZp; ++z)
            for (int x = R; x < R + NXp; ++x)
                np_ += (x <= pr || x >= pr + nx || (!fsf && z <= pr) || z >= pr + nz) ? 1 : 0;
        switch (id) {
            case OWL_K_FWD_P: return S * (cs * (8.0 + 24.0) + np_ * 4 * 8.0) + cs * 16.0 + np_ * 2 * 16.0;
            case OWL_K_FWD_V: return S * (cv * (12.0 + 16.0) + np_ * 4 * 8.0) + cv * 8.0 + np_ * 2 * 16.0;
            case OWL_K_ADJ_P:
                return S * (cv * (16.0 + 16.0 + 16.0 + 8.0) + np_ * 4 * 8.0) + cv * 8.0 + np_ * 2 * 16.0 +
                       groups * cv * 2 * 16.0;
            case OWL_K_ADJ_V:
                return S * (cs * (16.0 + 24.0 + 16.0 + 12.0) + np_ * 4 * 8.0) + cs * 16.0 + np_ * 2 * 16.0 +
                       groups * cs * 4 * 16.0;
        }
        return 0;
    }

    void chain_rule(int S, int groups) override {
        El2dDev a = dev(S);
        const dim3 b(32, 8), g((nxq() + 31) / 32, (nzq() + 7) / 8);
        k_el2d_chain<<<g, b, 0, stream>>>(a, groups, c55p.p, rhop.p, vm.refined ? nullptr : jac.p, nparam,
                                          (long long)npad(), gpad.p, nxq(), nzq());
        OWL_LAUNCH_CHECK();
        launches++;
    }

    // refined mesh: the mesh cells' d J / d Cij to the regular rows and the
    // model parameters (k_el2d_zmap), then the fold of the padding
    void fold_out(float* grad, int mem) override {
        if (!vm.refined) {
            SsgBase::fold_out(grad, mem);
            return;
        }
        const int nzq_r = nz_model + 2 * P + 2;
        const size_t npr = (size_t)nxq() * nzq_r;
        gzmap.reserve((size_t)nparam * npr);
        const dim3 b(32, 8), g((nxq() + 31) / 32, (nzq_r + 7) / 8);
        k_el2d_zmap<<<g, b, 0, stream>>>(gpad.p, (long long)npad(), zptr.p, zrow.p, zw.p, jac.p, nparam,
                                         (long long)npr, gzmap.p, nxq(), nzq_r);
        OWL_LAUNCH_CHECK();
        launches++;
        const size_t nm = (size_t)nx * nz_model;
        seis_tmp.reserve((size_t)nparam * nm);
        for (int q = 0; q < nparam; ++q) {
            launch_fold(gzmap.p + (size_t)q * npr, nxq(), 1, P, nx, 1, nz_model, 2, seis_tmp.p + (size_t)q * nm,
                        stream);
            launches++;
        }
        copy_out(grad, seis_tmp.p, (size_t)nparam * nm * sizeof(float), mem);
    }
};

Engine* make_el2d_engine(const owl_ssg_desc& d) { return new El2dEngine(d); }

// refine_nz = ceiling(0.5 lambda / dz), lambda = sqrt(mean(c55 / rho over the
// padded surface row)) / f0_min (module_vars.f90:315-317)
int el2d_refine_rows(const owl_ssg_desc& d, int np, const float* const* f, float f0_min) {
    OWL_CHECK(np == el_nparam(d.aniso) && f, OWL_ERR_INVALID,
              "elastic 2D model needs " + std::to_string(el_nparam(d.aniso)) + " parameters for this parameterisation");
    for (int q = 0; q < np; ++q) OWL_CHECK(f[q], OWL_ERR_INVALID, "null model parameter");
    OWL_CHECK(d.nx >= 1 && d.nz >= 1 && d.pml >= 0 && d.dz > 0, OWL_ERR_INVALID, "bad grid");
    std::vector<float> p(np);
    float sum = 0.f;
    int cnt = 0;
    for (int i = -d.pml; i <= d.nx + d.pml + 1; ++i) {
        const int ii = std::min(std::max(i, 1), d.nx);
        for (int q = 0; q < np; ++q) p[q] = f[q][(size_t)(ii - 1) * d.nz];
        float a11, a13, a33, a55, r;
        cij_of<float>(d.aniso, p.data(), a11, a13, a33, a55, r);
        OWL_CHECK(r > 0 && a55 > 0, OWL_ERR_INVALID, "rho and c55 must be positive");
        sum += a55 / r;
        ++cnt;
    }
    const float lambda = std::sqrt(sum / (float)cnt) / f0_min;
    return (int)std::ceil(0.5f * lambda / d.dz);
}

}  // namespace owl
