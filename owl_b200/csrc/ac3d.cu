// ac3d.cu -- 3D isotropic acoustic SSG solver for B200 (sm_100a).
//
// Replaces update_wavefield / update_wavefield_free_surface / add_source of
// src/solver/acoustic_iso_3d/module_wavefield.f90:40-444 (single rank: the
// reference's MPI halo exchange, commute_array_group, is not needed because
// one B200 holds the whole model) and the gradient of
// submodule_fwi_gradient.f90 with the exact discrete adjoint.
//
// Layout in HBM. A field is (NZs, NYs, pitch) float32, x fastest, storage
// index = reference index + pml + R - 1 on every axis (the reference permutes
// (nz,ny,nx) to x fastest too, module_vars.f90:158). Per shot: p, vx, vy, vz
// as full fields, and the six CFS-PML memory variables as compact slabs that
// cover only their PML (x slab (NZp, NYp, 2P+1), y slab (NZp, 2P+1, NXp),
// z slab (2P+1, NYp, NXp)) -- the reference's _xmin/_xmax arrays, one slab.
//
// Kernels march along z (the slowest axis): a CTA owns a 32 x TY tile of one
// x-y plane and a chunk of z planes; x / y neighbours come from shared-memory
// tiles of the current plane (with the R halo), z neighbours from a register
// queue of 2R values that rotates as the CTA steps down.
#include <algorithm>
#include <cmath>

#include "ring.cuh"
#include "ssg_base.cuh"
#include "tma.cuh"

#ifndef OWL_AC3_ZCHUNK_MIN
#define OWL_AC3_ZCHUNK_MIN 16  // shortest z chunk of a forward CTA
#endif

namespace owl {

__constant__ float c_fd3[8];

struct Ac3dDev {
    int nx, ny, nz, P, R, pr, pitch, NXs, NYs, NZs, NXp, NYp, W;
    long long plane, fs, sst, sad;
    int x0, x1, y0, y1, z1, zp0, zvx0, zvz0, fsurf;
    float idx, idy, idz;
    int nshots, spt, zchunk;
    const float *dtbk, *dtbx, *dtby, *dtbz;
    const float *axi, *bxi, *axh, *bxh, *ayi, *byi, *ayh, *byh, *azi, *bzi, *azh, *bzh;
    // forward state (shot 0); memory slabs: m[0..2] for d(vx)/dx, d(vy)/dy, d(vz)/dz
    // (p update), m[3..5] for dp/dx, dp/dy, dp/dz (v updates)
    float *p, *vx, *vy, *vz, *m0, *m1, *m2, *m3, *m4, *m5;
    float *Sp, *Svx, *Svy, *Svz;
    long long sslot;
    int k;
    int* d_step;
    // adjoint state (shot 0)
    float *ap, *avx, *avy, *avz, *am0, *am1, *am2, *am3, *am4, *am5;
    float *aex, *aey, *aez, *aepx, *aepy, *aepz;
    float *Gbk, *Gbx, *Gby, *Gbz, *Cbk, *Cbx, *Cby, *Cbz;
    int* err;  // set by a TMA wait that gave up (OWL_ERR_TIMEOUT on the host)
};

// slab indices (only called for nodes inside the corresponding PML)
__device__ __forceinline__ int slab_i(int x, int R, int pr, int n, int P) { return x <= pr ? x - R : x - (pr + n) + P + 1; }
__device__ __forceinline__ long long xslab(const Ac3dDev& a, int x, int y, int z) {
    return ((long long)(z - a.R) * a.NYp + (y - a.R)) * a.W + slab_i(x, a.R, a.pr, a.nx, a.P);
}
__device__ __forceinline__ long long yslab(const Ac3dDev& a, int x, int y, int z) {
    return ((long long)(z - a.R) * a.W + slab_i(y, a.R, a.pr, a.ny, a.P)) * a.NXp + (x - a.R);
}
__device__ __forceinline__ long long zslab(const Ac3dDev& a, int x, int y, int z) {
    return ((long long)slab_i(z, a.R, a.pr, a.nz, a.P) * a.NYp + (y - a.R)) * a.NXp + (x - a.R);
}
__device__ __forceinline__ bool pin(int x, int pr, int n) { return x < pr || x >= pr + n; }   // integer node in PML
__device__ __forceinline__ bool phf(int x, int pr, int n) { return x <= pr || x >= pr + n; }  // half node in PML

// load a (TY x (32+2R)) tile of plane z (x halo) and a ((TY+2R) x 32) tile (y halo)
template <int R, int TY>
__device__ __forceinline__ void load_xy_tiles(float (*tx_)[32 + 2 * R], float (*ty_)[32], const float* fx, const float* fy,
                                              long long zoff, int bx0, int by0, const Ac3dDev& a, int xshift, int yshift) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
    constexpr int NT = 32 * TY, WX = 32 + 2 * R;
    for (int q = tid; q < TY * WX; q += NT) {
        int r = q / WX, c = q - r * WX;
        int xx = bx0 - R + xshift + c, yy = by0 + r;
        tx_[r][c] = (xx >= 0 && xx < a.NXs && yy < a.NYs) ? fx[zoff + (long long)yy * a.pitch + xx] : 0.f;
    }
    for (int q = tid; q < (TY + 2 * R) * 32; q += NT) {
        int r = q >> 5, c = q & 31;
        int xx = bx0 + c, yy = by0 - R + yshift + r;
        ty_[r][c] = (yy >= 0 && yy < a.NYs && xx < a.NXs) ? fy[zoff + (long long)yy * a.pitch + xx] : 0.f;
    }
}

// ------------------------------- forward ------------------------------------
#include "ac3d_fwd.cuh"
#include "ac3d_fwd_tma.cuh"

// One thread per cell, block 32 x 4 x 2, every neighbour an independent
// read-only load (served by L1 / L2): low register count, full occupancy and
// many loads in flight, at the price of re-reading halos from cache.
template <int R, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_p_n(Ac3dDev a) {
    const int x = a.x0 + blockIdx.x * 32 + threadIdx.x;
    const int y = a.y0 + blockIdx.y * 4 + threadIdx.y;
    const int nzb = (a.z1 - a.zp0 + 1) / 2;
    const int grp = blockIdx.z / nzb;
    const int z = a.zp0 + (blockIdx.z % nzb) * 2 + threadIdx.z;
    if (x >= a.x1 || y >= a.y1 || z >= a.z1) return;
    const int pt = a.pitch, pl = (int)a.plane;
    const int o = z * pl + y * pt + x;
    const float bk = __ldg(a.dtbk + o);
    const bool px = pin(x, a.pr, a.nx), py = pin(y, a.pr, a.ny);
    const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst;
        const float* __restrict__ vx = a.vx + so + o;
        const float* __restrict__ vy = a.vy + so + o;
        const float* __restrict__ vz = a.vz + so + o;
        float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) gx = gx + c_fd3[k - 1] * (__ldg(vx + k) - __ldg(vx + 1 - k));
#pragma unroll
        for (int k = 1; k <= R; ++k) gy = gy + c_fd3[k - 1] * (__ldg(vy + k * pt) - __ldg(vy + (1 - k) * pt));
#pragma unroll
        for (int k = 1; k <= R; ++k) gz = gz + c_fd3[k - 1] * (__ldg(vz + k * pl) - __ldg(vz + (1 - k) * pl));
        gx = a.idx * gx; gy = a.idy * gy; gz = a.idz * gz;
        if (px) {
            float* m = a.m0 + so + xslab(a, x, y, z);
            float mv = a.axi[x] * gx + a.bxi[x] * *m; *m = mv; gx = gx + mv;
        }
        if (py) {
            float* m = a.m1 + so + yslab(a, x, y, z);
            float mv = a.ayi[y] * gy + a.byi[y] * *m; *m = mv; gy = gy + mv;
        }
        if (pz) {
            float* m = a.m2 + so + zslab(a, x, y, z);
            float mv = a.azi[z] * gz + a.bzi[z] * *m; *m = mv; gz = gz + mv;
        }
        const float g = gx + gy + gz;
        float* pp = a.p + so + o;
        const float pn = *pp - bk * g;
        *pp = pn;
        if (a.fsurf && z <= a.pr + a.P) a.p[so + (2 * a.pr - z) * pl + y * pt + x] = -pn;
        if (STORE) a.Sp[slot + s * a.fs + o] = g;
    }
}

template <int R, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_v_n(Ac3dDev a) {
    const int zr0 = min(a.zvx0, a.zvz0);
    const int x = a.x0 + blockIdx.x * 32 + threadIdx.x;
    const int y = a.y0 + blockIdx.y * 4 + threadIdx.y;
    const int nzb = (a.z1 - zr0 + 1) / 2;
    const int grp = blockIdx.z / nzb;
    const int z = zr0 + (blockIdx.z % nzb) * 2 + threadIdx.z;
    if (x >= a.x1 || y >= a.y1 || z >= a.z1) return;
    const int pt = a.pitch, pl = (int)a.plane;
    const int o = z * pl + y * pt + x;
    const bool px = phf(x, a.pr, a.nx), py = phf(y, a.pr, a.ny);
    const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
    const float bxc = dox ? __ldg(a.dtbx + o) : 0.f, byc = dox ? __ldg(a.dtby + o) : 0.f;
    const float bzc = doz ? __ldg(a.dtbz + o) : 0.f;
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst;
        const float* __restrict__ p = a.p + so + o;
        if (dox) {
            float h = 0.f, hy = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (__ldg(p + k - 1) - __ldg(p - k));
#pragma unroll
            for (int k = 1; k <= R; ++k) hy = hy + c_fd3[k - 1] * (__ldg(p + (k - 1) * pt) - __ldg(p - k * pt));
            h = a.idx * h;
            hy = a.idy * hy;
            if (px) {
                float* m = a.m3 + so + xslab(a, x, y, z);
                float mv = a.axh[x] * h + a.bxh[x] * *m; *m = mv; h = h + mv;
            }
            if (py) {
                float* m = a.m4 + so + yslab(a, x, y, z);
                float mv = a.ayh[y] * hy + a.byh[y] * *m; *m = mv; hy = hy + mv;
            }
            a.vx[so + o] = a.vx[so + o] - bxc * h;
            a.vy[so + o] = a.vy[so + o] - byc * hy;
            if (STORE) { a.Svx[slot + s * a.fs + o] = h; a.Svy[slot + s * a.fs + o] = hy; }
        }
        if (doz) {
            float h = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (__ldg(p + (k - 1) * pl) - __ldg(p - k * pl));
            h = a.idz * h;
            if (pz) {
                float* m = a.m5 + so + zslab(a, x, y, z);
                float mv = a.azh[z] * h + a.bzh[z] * *m; *m = mv; h = h + mv;
            }
            a.vz[so + o] = a.vz[so + o] - bzc * h;
            if (STORE) a.Svz[slot + s * a.fs + o] = h;
        }
    }
}

// ------------------------------- adjoint ------------------------------------
// Same split as the 2D solver (ac2d.cu): k_ac3d_adj_p applies the transposed
// v-update stencils to the stored adjoint PML terms e_x, e_y, e_z of the
// velocity nodes, then forms the p-update terms e_px, e_py, e_pz of each cell;
// k_ac3d_adj_v applies the transposed p-update stencils to those and forms
// e_x, e_y, e_z for the step before. Kahan sums of v^ . S and p^ . S feed the
// coefficient gradients.
template <int R, int TY>
__global__ void __launch_bounds__(32 * TY) k_ac3d_adj_p(Ac3dDev a) {
    __shared__ float sx[TY][32 + 2 * R];
    __shared__ float sy[TY + 2 * R][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * TY;
    const int x = bx0 + tx, y = by0 + ty;
    const bool valid = x < a.x1 && y < a.y1;
    const int zr0 = min(min(a.zvx0, a.zvz0), a.zp0);
    const int nzc = (a.z1 - zr0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = zr0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool px = pin(x, a.pr, a.nx), py = pin(y, a.pr, a.ny);
    const float axi = px ? a.axi[x] : 0.f, bxi = px ? a.bxi[x] : 0.f;
    const float ayi = py ? a.ayi[y] : 0.f, byi = py ? a.byi[y] : 0.f;
    const long long oxy = (long long)y * a.pitch + x;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    for (int z = zb; z < ze; ++z) {
        const long long zo = (long long)z * a.plane, o = zo + oxy;
        const bool dop = z >= a.zp0, ownx = z >= a.zvx0, ownz = z >= a.zvz0;
        const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
        float gbk = 0.f, gbx = 0.f, gby = 0.f, gbz = 0.f;
        for (int s = s0; s < s1; ++s) {
            const long long sa = s * a.sad;
            load_xy_tiles<R, TY>(sx, sy, a.aex + sa, a.aey + sa, zo, bx0, by0, a, 0, 0);
            __syncthreads();
            if (valid) {
                const long long ss = slot + s * a.fs + o;
                if (ownx) {
                    gbx += a.avx[sa + o] * a.Svx[ss];
                    gby += a.avy[sa + o] * a.Svy[ss];
                }
                if (ownz) gbz += a.avz[sa + o] * a.Svz[ss];
                if (dop) {
                    const float* ez = a.aez + sa + oxy;
                    float sxv = 0.f, syv = 0.f, szv = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) sxv = sxv + c_fd3[k - 1] * (sx[ty][tx + R - k + 1] - sx[ty][tx + R + k]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) syv = syv + c_fd3[k - 1] * (sy[ty + R - k + 1][tx] - sy[ty + R + k][tx]);
#pragma unroll
                    for (int k = 1; k <= R; ++k)
                        szv = szv + c_fd3[k - 1] * (ez[(long long)(z - k + 1) * a.plane] - ez[(long long)(z + k) * a.plane]);
                    float dP = a.idx * sxv + a.idy * syv + a.idz * szv;
                    if (a.fsurf && z <= a.pr + a.P) {
                        const int zm = 2 * a.pr - z;
                        float sm = 0.f;
#pragma unroll
                        for (int k = 1; k <= R; ++k)
                            sm = sm + c_fd3[k - 1] * (ez[(long long)(zm - k + 1) * a.plane] - ez[(long long)(zm + k) * a.plane]);
                        dP = dP - a.idz * sm;
                    }
                    const float ph = a.ap[sa + o] + dP;
                    a.ap[sa + o] = ph;
                    gbk += ph * a.Sp[ss];
                    const float qv = -a.dtbk[o] * ph;
                    float ex = qv, ey = qv, ez2 = qv;
                    if (px) {
                        float* m = a.am0 + sa + xslab(a, x, y, z);
                        float u = qv + *m; *m = bxi * u; ex = qv + axi * u;
                    }
                    if (py) {
                        float* m = a.am1 + sa + yslab(a, x, y, z);
                        float u = qv + *m; *m = byi * u; ey = qv + ayi * u;
                    }
                    if (pz) {
                        float* m = a.am2 + sa + zslab(a, x, y, z);
                        float u = qv + *m; *m = a.bzi[z] * u; ez2 = qv + a.azi[z] * u;
                    }
                    a.aepx[sa + o] = ex;
                    a.aepy[sa + o] = ey;
                    a.aepz[sa + o] = ez2;
                }
            }
            __syncthreads();
        }
        if (valid) {
            const long long go = (long long)grp * a.fs + o;
            float sm, c;
            if (dop) { sm = a.Gbk[go]; c = a.Cbk[go]; kahan_add(sm, c, gbk); a.Gbk[go] = sm; a.Cbk[go] = c; }
            if (ownx) {
                sm = a.Gbx[go]; c = a.Cbx[go]; kahan_add(sm, c, gbx); a.Gbx[go] = sm; a.Cbx[go] = c;
                sm = a.Gby[go]; c = a.Cby[go]; kahan_add(sm, c, gby); a.Gby[go] = sm; a.Cby[go] = c;
            }
            if (ownz) { sm = a.Gbz[go]; c = a.Cbz[go]; kahan_add(sm, c, gbz); a.Gbz[go] = sm; a.Cbz[go] = c; }
        }
    }
}

template <int R, int TY>
__global__ void __launch_bounds__(32 * TY) k_ac3d_adj_v(Ac3dDev a) {
    __shared__ float sx[TY][32 + 2 * R];
    __shared__ float sy[TY + 2 * R][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * TY;
    const int x = bx0 + tx, y = by0 + ty;
    const bool valid = x < a.x1 && y < a.y1;
    const int zr0 = min(a.zvx0, a.zvz0);
    const int nzc = (a.z1 - zr0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = zr0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool px = phf(x, a.pr, a.nx), py = phf(y, a.pr, a.ny);
    const float axh = px ? a.axh[x] : 0.f, bxh = px ? a.bxh[x] : 0.f;
    const float ayh = py ? a.ayh[y] : 0.f, byh = py ? a.byh[y] : 0.f;
    const long long oxy = (long long)y * a.pitch + x;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad;
        const float* epz = a.aepz + sa + oxy;
        float q[2 * R];  // q[j] = e_pz(z - R + j)
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) q[j] = valid ? epz[(long long)(zb - R + j) * a.plane] : 0.f;
        for (int z = zb; z < ze; ++z) {
            const long long zo = (long long)z * a.plane, o = zo + oxy;
            // e_px with x halo shifted by -1 (nodes need cells m-R .. m+R-1)
            load_xy_tiles<R, TY>(sx, sy, a.aepx + sa, a.aepy + sa, zo, bx0, by0, a, -1, -1);
            __syncthreads();
            if (valid) {
                // the cell's own values are read ahead of its stores (the arrays
                // share one allocation: no plain read could move above a store);
                // what this launch does not write goes through the read-only path
                const bool ox = z >= a.zvx0, oz = z >= a.zvz0;
                const bool pzz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
                const float vx0 = ox ? a.avx[sa + o] : 0.f, vy0 = ox ? a.avy[sa + o] : 0.f;
                const float vz0 = oz ? a.avz[sa + o] : 0.f;
                float* m3p = a.am3 + sa + xslab(a, x, y, z);
                float* m4p = a.am4 + sa + yslab(a, x, y, z);
                float* m5p = a.am5 + sa + zslab(a, x, y, z);
                const float m3 = ox && px ? *m3p : 0.f, m4 = ox && py ? *m4p : 0.f, m5 = oz && pzz ? *m5p : 0.f;
                if (ox) {
                    float h = 0.f, hy = 0.f;
                    // sx col c <-> cell bx0 - R - 1 + c; node x needs cells x-k (col tx+R+1-k) and x+k-1 (col tx+R+k)
#pragma unroll
                    for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (sx[ty][tx + R + 1 - k] - sx[ty][tx + R + k]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) hy = hy + c_fd3[k - 1] * (sy[ty + R + 1 - k][tx] - sy[ty + R + k][tx]);
                    const float xh = vx0 + a.idx * h;
                    const float yh = vy0 + a.idy * hy;
                    a.avx[sa + o] = xh;
                    a.avy[sa + o] = yh;
                    float qx = -__ldg(a.dtbx + o) * xh, qy = -__ldg(a.dtby + o) * yh;
                    float ex = qx, ey = qy;
                    if (px) {
                        float u = qx + m3; *m3p = bxh * u; ex = qx + axh * u;
                    }
                    if (py) {
                        float u = qy + m4; *m4p = byh * u; ey = qy + ayh * u;
                    }
                    a.aex[sa + o] = ex;
                    a.aey[sa + o] = ey;
                }
                if (oz) {
                    float h = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (q[R - k] - q[R + k - 1]);
                    const float zh = vz0 + a.idz * h;
                    a.avz[sa + o] = zh;
                    float qz = -__ldg(a.dtbz + o) * zh, ez = qz;
                    if (pzz) {
                        float u = qz + m5; *m5p = a.bzh[z] * u; ez = qz + a.azh[z] * u;
                    }
                    a.aez[sa + o] = ez;
                }
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) q[j] = q[j + 1];
            q[2 * R - 1] = (valid && z + R < a.NZs) ? __ldg(epz + (long long)(z + R) * a.plane) : 0.f;
            __syncthreads();
        }
    }
}

#include "ac3d_adj_ring.cuh"

// ------------------------- FP64 chain rule ---------------------------------
__global__ void k_ac3d_chain(Ac3dDev a, int ngroups, const float* __restrict__ vpp, const float* __restrict__ rhop,
                             double dt, double* __restrict__ gvp, double* __restrict__ grho, int nxq, int nyq, int nzq) {
    const long long n = (long long)nxq * nyq * nzq;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(q % nxq);
        const long long r = q / nxq;
        const int iy = (int)(r % nyq), iz = (int)(r / nyq);
        const int x = a.R - 1 + ix, y = a.R - 1 + iy, z = a.R - 1 + iz;
        const long long o = (long long)z * a.plane + (long long)y * a.pitch + x;
        auto sumG = [&](const float* G, const float* C, long long oo) {
            double v = 0;
            for (int g = 0; g < ngroups; ++g) v += (double)G[g * a.fs + oo] - (double)C[g * a.fs + oo];
            return v;
        };
        const bool inx = x >= a.x0 && x < a.x1, iny = y >= a.y0 && y < a.y1;
        double vp = vpp[o], rho = rhop[o];
        double dv = 0, dr = 0;
        if (inx && iny && z >= a.zp0 && z < a.z1) {
            double gbk = sumG(a.Gbk, a.Cbk, o);
            dv += -gbk * dt * 2.0 * rho * vp;
            dr += -gbk * dt * vp * vp;
        }
        for (int d = 0; d <= 1; ++d) {
            int m = x + d;
            if (m >= a.x0 && m < a.x1 && iny && z >= a.zvx0 && z < a.z1) {
                long long om = o + d;
                double re = 0.5 * ((double)rhop[om] + (double)rhop[om - 1]);
                dr += sumG(a.Gbx, a.Cbx, om) * 0.5 * dt / (re * re);
            }
            int my = y + d;
            if (inx && my >= a.y0 && my < a.y1 && z >= a.zvx0 && z < a.z1) {
                long long om = o + (long long)d * a.pitch;
                double re = 0.5 * ((double)rhop[om] + (double)rhop[om - a.pitch]);
                dr += sumG(a.Gby, a.Cby, om) * 0.5 * dt / (re * re);
            }
            int mz = z + d;
            if (inx && iny && mz >= a.zvz0 && mz < a.z1) {
                long long om = o + (long long)d * a.plane;
                double re = 0.5 * ((double)rhop[om] + (double)rhop[om - a.plane]);
                dr += sumG(a.Gbz, a.Cbz, om) * 0.5 * dt / (re * re);
            }
        }
        gvp[q] += dv;
        grho[q] += dr;
    }
}

// ============================================================================
// host engine
// ============================================================================
struct Ac3dEngine : SsgBase {
    float idx, idy, idz;
    int W;
    long long sx_n, sy_n, sz_n;  // floats of one x / y / z slab
    int zchunk = 64;
    DevBuf<float> dtbk, dtbx, dtby, dtbz, vpp, rhop, pml_x, pml_y, pml_z;

    explicit Ac3dEngine(const owl_ssg_desc& d) : SsgBase(d, 3) {
        idx = (float)(1.0 / (double)d.dx);
        idy = (float)(1.0 / (double)d.dy);
        idz = (float)(1.0 / (double)d.dz);
        OWL_CUDA(cudaMemcpyToSymbol(c_fd3, fd_coefs(R), sizeof(float) * R));
        W = 2 * P + 1;
        sx_n = (long long)NZp * NYp * W;
        sy_n = (long long)NZp * W * NXp;
        sz_n = (long long)W * NYp * NXp;
        // state: p, vx, vy, vz, then slabs m0 (x), m1 (y), m2 (z), m3 (x), m4 (y), m5 (z)
        // shot strides rounded to 64 floats: every field of every shot starts 16-byte aligned
        sst = (4 * fs + 2 * (sx_n + sy_n + sz_n) + 63) / 64 * 64;
        // adjoint: p^, vx^, vy^, vz^, 6 memory slabs, e_x, e_y, e_z, e_px, e_py, e_pz; the
        // slabs rounded to 64 floats so that the e arrays start 16-byte aligned too
        sad = (10 * fs + slab_span() + 63) / 64 * 64;
        nS = 4;
        ngrad = 4;
        nparam = 2;
        ncomp = 1;
        for (int f = 0; f < 4; ++f) st_segments.push_back({f * fs, fs});
        long long off = 4 * fs;
        for (int r = 0; r < 2; ++r)
            for (long long n : {sx_n, sy_n, sz_n}) { st_segments.push_back({off, n}); off += n; }
    }

    long long st_off(int f) const {
        if (f < 4) return f * fs;
        const long long sl[6] = {sx_n, sy_n, sz_n, sx_n, sy_n, sz_n};
        long long off = 4 * fs;
        for (int i = 0; i < f - 4; ++i) off += sl[i];
        return off;
    }
    long long slab_span() const { return (2 * (sx_n + sy_n + sz_n) + 63) / 64 * 64; }
    long long ad_off(int f) const {  // 0..3 fields, 4..9 slabs, 10..15 e arrays
        if (f < 4) return f * fs;
        if (f < 10) return st_off(f);
        return 4 * fs + slab_span() + (long long)(f - 10) * fs;
    }
    float* st_field(int f) const override { return f < 4 ? st.p + st_off(f) : nullptr; }
    float* ad_field(int f) const override { return f < 4 ? ad.p + ad_off(f) : nullptr; }
    int rho_param() const override { return 1; }

    void set_model(int nparam_, const float* const* f) override {
        OWL_CHECK(nparam_ == 2 && f && f[0] && f[1], OWL_ERR_INVALID, "acoustic model needs vp and rho");
        const float* vp = f[0];
        const float* rho = f[1];
        std::vector<float> hvp(fs, 0.f), hrho(fs, 0.f), hbk(fs, 0.f);
        float maxv = -1e30f;
        for (int k = -P; k <= nz + P + 1; ++k)
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i) {
                    int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), ny),
                        kk = std::min(std::max(k, 1), nz);
                    size_t src = ((size_t)(ii - 1) * ny + (jj - 1)) * nz + (kk - 1);
                    float v = vp[src], r = rho[src];
                    OWL_CHECK(std::isfinite(v) && std::isfinite(r) && v > 0 && r > 0, OWL_ERR_INVALID,
                              "vp and rho must be finite and positive");
                    long long o = soff(i, j, k);
                    hvp[o] = v; hrho[o] = r;
                    hbk[o] = dt * (r * v * v);
                    maxv = std::max(maxv, v);
                }
        // dtb at velocity nodes (rho_eff_x/y/z, module_wavefield.f90:30-32)
        std::vector<float> hb(fs, 0.f);
        auto dtb = [&](int di, int dj, int dk, DevBuf<float>& out) {
            std::fill(hb.begin(), hb.end(), 0.f);
            for (int k = -P + 1; k <= nz + P; ++k)
                for (int j = -P + 1; j <= ny + P; ++j)
                    for (int i = -P + 1; i <= nx + P; ++i) {
                        float re = 0.5f * (hrho[soff(i, j, k)] + hrho[soff(i - di, j - dj, k - dk)]);
                        hb[soff(i, j, k)] = dt / re;
                    }
            out.upload(hb.data(), fs, stream);
            OWL_CUDA(cudaStreamSynchronize(stream));
        };
        dtb(1, 0, 0, dtbx);
        dtb(0, 1, 0, dtby);
        dtb(0, 0, 1, dtbz);
        const float* c = fd_coefs(R);
        float temp = 0.f;
        for (int q = 0; q < R; ++q) temp += std::fabs(c[q]);
        dt_stable_ = 1.0f / (temp * maxv * std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (desc.dy * desc.dy) +
                                                     1.0f / (desc.dz * desc.dz)));
        if (dt > dt_stable_ && !desc.allow_dt_adjust)
            throw OwlError(OWL_ERR_UNSTABLE, "dt = " + std::to_string(dt) + " exceeds the stable dt " +
                                                 std::to_string(dt_stable_));
        // pmlvp = max vp over the six model faces (module_vars.f90:162-164)
        float pmlvp = -1e30f;
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= ny; ++j) pmlvp = std::max({pmlvp, hvp[soff(1, j, k)], hvp[soff(nx, j, k)]});
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, hvp[soff(i, 1, k)], hvp[soff(i, ny, k)]});
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) pmlvp = std::max({pmlvp, hvp[soff(i, j, 1)], hvp[soff(i, j, nz)]});
        float alphamax = (float)(1.0 * (double)desc.f0_max * 3.14159265358979323846);
        auto pack = [&](int n, int len, float d, DevBuf<float>& out) {
            Pml1DHost h = build_pml_1d(n, P, R, len, d, dt, pmlvp, alphamax);
            std::vector<float> v(4 * len);
            std::copy(h.ai.begin(), h.ai.end(), v.begin());
            std::copy(h.bi.begin(), h.bi.end(), v.begin() + len);
            std::copy(h.ah.begin(), h.ah.end(), v.begin() + 2 * len);
            std::copy(h.bh.begin(), h.bh.end(), v.begin() + 3 * len);
            out.upload(v.data(), v.size(), stream);
            OWL_CUDA(cudaStreamSynchronize(stream));
        };
        pack(nx, pitch, desc.dx, pml_x);
        pack(ny, NYs, desc.dy, pml_y);
        pack(nz, NZs, desc.dz, pml_z);
        dtbk.upload(hbk.data(), fs, stream);
        vpp.upload(hvp.data(), fs, stream);
        rhop.upload(hrho.data(), fs, stream);
        OWL_CUDA(cudaStreamSynchronize(stream));
        h_rhop = std::move(hrho);
        model_set = true;
        invalidate_graphs();
    }

    // ---- sources / receivers (module_wavefield.f90:322-444)
    int src_ncomp(const owl_source& q) const override {
        OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION || q.mechanism == OWL_SRC_FORCE, OWL_ERR_UNSUPPORTED,
                  "acoustic media support explosion and force sources");
        return q.mechanism == OWL_SRC_FORCE ? 3 : 1;
    }
    void src_taps(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rc, float& rv) const override {
        const bool fsf = desc.free_surface != 0;
        float dir = 1.f;
        if (q.mechanism == OWL_SRC_FORCE) {
            // 3D force: one rho at the integer node (gx, gy, gz)
            OWL_CHECK(in_wavefield(q.gx, q.gy, q.gz), OWL_ERR_INVALID, "force source outside the grid");
            rv = h_rhop[soff(q.gx, q.gy, q.gz)];
            rc = pad_index(q.gx, q.gy, q.gz);
            dir = comp == 0 ? std::sin(q.polar) * std::cos(q.azimuth)
                            : comp == 1 ? std::sin(q.polar) * std::sin(q.azimuth) : std::cos(q.polar);
        }
        for (int irz = -4; irz <= 4; ++irz)
            for (int iry = -4; iry <= 4; ++iry)
                for (int irx = -4; irx <= 4; ++irx) {
                    TapPt t;
                    if (q.mechanism == OWL_SRC_EXPLOSION) {
                        t = TapPt{0, q.gx + irx, q.gy + iry, q.gz + irz,
                                  q.interp_ix[irx + 4] * q.interp_iy[iry + 4] * q.interp_iz[irz + 4]};
                    } else if (comp == 0) {
                        t = TapPt{1, q.hx + irx, q.gy + iry, q.gz + irz,
                                  dir / rv * q.interp_hx[irx + 4] * q.interp_iy[iry + 4] * q.interp_iz[irz + 4]};
                    } else if (comp == 1) {
                        t = TapPt{2, q.gx + irx, q.hy + iry, q.gz + irz,
                                  dir / rv * q.interp_ix[irx + 4] * q.interp_hy[iry + 4] * q.interp_iz[irz + 4]};
                    } else {
                        t = TapPt{3, q.gx + irx, q.gy + iry, q.hz + irz,
                                  dir / rv * q.interp_ix[irx + 4] * q.interp_iy[iry + 4] * q.interp_hz[irz + 4]};
                    }
                    if (fsf && t.k < 2) continue;
                    taps.push_back(t);
                }
    }
    // taps with a zero factor are dropped here (the table keeps none of them)
    void rec_taps(const owl_receiver& q, int, std::vector<TapPt>& taps) const override {
        for (int irz = -4; irz <= 4; ++irz) {
            if (q.interp_iz[irz + 4] == 0.f) continue;
            for (int iry = -4; iry <= 4; ++iry) {
                if (q.interp_iy[iry + 4] == 0.f) continue;
                for (int irx = -4; irx <= 4; ++irx)
                    if (q.interp_ix[irx + 4] != 0.f)
                        taps.push_back(TapPt{0, q.gx + irx, q.gy + iry, q.gz + irz,
                                             q.interp_ix[irx + 4] * q.interp_iy[iry + 4] * q.interp_iz[irz + 4] * q.weight});
            }
        }
    }
    void scatter_map(const TapPt& t, std::vector<TapPt>& out) const override {
        if (!desc.free_surface) { out.push_back(t); return; }
        if (t.k <= 0) out.push_back(TapPt{t.field, t.i, t.j, 2 - t.k, -t.w});
        else if (t.k >= 2) out.push_back(t);
    }

    Ac3dDev dev(int S) const {
        Ac3dDev a{};
        a.nx = nx; a.ny = ny; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch;
        a.NXs = NXs; a.NYs = NYs; a.NZs = NZs; a.NXp = NXp; a.NYp = NYp; a.W = W;
        a.plane = plane; a.fs = fs; a.sst = sst; a.sad = sad;
        a.x0 = R; a.x1 = R + NXp; a.y0 = R; a.y1 = R + NYp; a.z1 = R + NZp;
        a.fsurf = desc.free_surface != 0;
        a.zp0 = a.fsurf ? pr + 1 : R;
        a.zvx0 = a.fsurf ? pr : R;
        a.zvz0 = a.fsurf ? pr + 1 : R;
        a.idx = idx; a.idy = idy; a.idz = idz;
        a.nshots = S;
        a.zchunk = zchunk;
        a.dtbk = dtbk.p; a.dtbx = dtbx.p; a.dtby = dtby.p; a.dtbz = dtbz.p;
        a.axi = pml_x.p; a.bxi = pml_x.p + pitch; a.axh = pml_x.p + 2 * pitch; a.bxh = pml_x.p + 3 * pitch;
        a.ayi = pml_y.p; a.byi = pml_y.p + NYs; a.ayh = pml_y.p + 2 * NYs; a.byh = pml_y.p + 3 * NYs;
        a.azi = pml_z.p; a.bzi = pml_z.p + NZs; a.azh = pml_z.p + 2 * NZs; a.bzh = pml_z.p + 3 * NZs;
        float* s0 = st.p;
        a.p = s0; a.vx = s0 + fs; a.vy = s0 + 2 * fs; a.vz = s0 + 3 * fs;
        a.m0 = s0 + st_off(4); a.m1 = s0 + st_off(5); a.m2 = s0 + st_off(6);
        a.m3 = s0 + st_off(7); a.m4 = s0 + st_off(8); a.m5 = s0 + st_off(9);
        a.k = std::max(1, cur_k);
        a.d_step = ctr.p;
        a.err = ctr.p + 3;
        const long long F = (long long)S * fs;
        if (Sbuf.p && Sbuf.n >= (size_t)4 * a.k * F) {
            a.sslot = F;
            a.Sp = Sbuf.p; a.Svx = Sbuf.p + (long long)a.k * F; a.Svy = Sbuf.p + 2LL * a.k * F;
            a.Svz = Sbuf.p + 3LL * a.k * F;
        }
        if (ad.p && ad.n >= (size_t)sad * S) {
            float* b = ad.p;
            a.ap = b; a.avx = b + fs; a.avy = b + 2 * fs; a.avz = b + 3 * fs;
            a.am0 = b + ad_off(4); a.am1 = b + ad_off(5); a.am2 = b + ad_off(6);
            a.am3 = b + ad_off(7); a.am4 = b + ad_off(8); a.am5 = b + ad_off(9);
            a.aex = b + ad_off(10); a.aey = b + ad_off(11); a.aez = b + ad_off(12);
            a.aepx = b + ad_off(13); a.aepy = b + ad_off(14); a.aepz = b + ad_off(15);
        }
        if (G.p) {
            const long long gg = (long long)((S + spt_a - 1) / spt_a) * fs;
            a.Gbk = G.p; a.Gbx = G.p + gg; a.Gby = G.p + 2 * gg; a.Gbz = G.p + 3 * gg;
            a.Cbk = G.p + 4 * gg; a.Cbx = G.p + 5 * gg; a.Cby = G.p + 6 * gg; a.Cbz = G.p + 7 * gg;
        }
        return a;
    }

    dim3 grid3(int rows, int S, int spt, int tyo) const {
        const int nzc = (rows + zchunk - 1) / zchunk;
        return dim3((NXp + 31) / 32, (NYp + tyo - 1) / tyo, nzc * ((S + spt - 1) / spt));
    }

    // z chunk so that the grid holds about 128 CTAs per SM (chunks of at least
    // 16 planes): many short chunks keep enough copies in flight to approach
    // the HBM bound, at the price of re-reading 2R planes at each chunk start
    void pick_zchunk(int tyo) {
        const long long xy = (long long)((NXp + 31) / 32) * ((NYp + tyo - 1) / tyo);
        long long want = std::max<long long>(1, (148LL * 128 + xy - 1) / xy);
        zchunk = (int)std::max<long long>(OWL_AC3_ZCHUNK_MIN, (NZp + want - 1) / want);
    }

    template <int RR, int RY>
    void launch_fwd(int id, int S, bool store) {
        Ac3dDev a = dev(S);
        a.spt = spt_f;
        pick_zchunk(8 * RY);
        a.zchunk = zchunk;
        const int rows_p = a.z1 - a.zp0, rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        dim3 b(32, 8);
        if (id == OWL_K_FWD_P) {
            constexpr int sm = ring_bytes_p<RR, RY>();
            auto k = store ? k_ac3d_fwd_p<RR, RY, true> : k_ac3d_fwd_p<RR, RY, false>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<grid3(rows_p, S, spt_f, 8 * RY), b, sm, stream>>>(a);
        } else {
            constexpr int sm = ring_bytes_v<RR, RY>();
            auto k = store ? k_ac3d_fwd_v<RR, RY, true> : k_ac3d_fwd_v<RR, RY, false>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<grid3(rows_v, S, spt_f, 8 * RY), b, sm, stream>>>(a);
        }
    }

    // tensor maps of the TMA forward kernels: the state as (x, y, z, field, shot)
    // with one box per tile shape, the coefficients as (x, y, z)
    Ac3Maps tma_maps(int RY, int S) const {
        Ac3Maps m;
        const uint32_t TYO = 8 * RY, WX = 32 + 2 * R, HY = TYO + 2 * R;
        const uint64_t sd[5] = {(uint64_t)pitch, (uint64_t)NYs, (uint64_t)NZs, 4, (uint64_t)S};
        const uint64_t ss[4] = {(uint64_t)pitch * 4, (uint64_t)plane * 4, (uint64_t)fs * 4, (uint64_t)sst * 4};
        auto st5 = [&](uint32_t bx, uint32_t by) {
            const uint32_t b[5] = {bx, by, 1, 1, 1};
            return make_tensor_map_f32(st.p, 5, sd, ss, b);
        };
        m.sA = st5(WX, TYO);
        m.sB = st5(32, HY);
        m.sC = st5(32, TYO);
        m.sD = st5(WX, HY);
        const uint64_t md[3] = {(uint64_t)pitch, (uint64_t)NYs, (uint64_t)NZs};
        const uint64_t ms[2] = {(uint64_t)pitch * 4, (uint64_t)plane * 4};
        const uint32_t bc[3] = {32, TYO, 1};
        m.mk = make_tensor_map_f32(dtbk.p, 3, md, ms, bc);
        m.mx = make_tensor_map_f32(dtbx.p, 3, md, ms, bc);
        m.my = make_tensor_map_f32(dtby.p, 3, md, ms, bc);
        m.mz = make_tensor_map_f32(dtbz.p, 3, md, ms, bc);
        return m;
    }

    template <int RR, int RY>
    void launch_fwd_tma(int id, int S, bool store) {
        Ac3dDev a = dev(S);
        a.spt = spt_f;
        pick_zchunk(8 * RY);
        a.zchunk = zchunk;
        OWL_CHECK(sst % 4 == 0 && fs % 4 == 0 && pitch % 4 == 0 && ((uintptr_t)st.p & 15) == 0, OWL_ERR_UNSUPPORTED,
                  "TMA operands not 16-byte aligned");
        const Ac3Maps mp = tma_maps(RY, S);
        const int rows_p = a.z1 - a.zp0, rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        dim3 b(32, 8);
        if (id == OWL_K_FWD_P) {
            constexpr int sm = tma_bytes_p<RR, RY>();
            auto k = store ? k_ac3d_fwd_p_tma<RR, RY, true> : k_ac3d_fwd_p_tma<RR, RY, false>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<grid3(rows_p, S, spt_f, 8 * RY), b, sm, stream>>>(a, mp);
        } else {
            constexpr int sm = tma_bytes_v<RR, RY>();
            auto k = store ? k_ac3d_fwd_v_tma<RR, RY, true> : k_ac3d_fwd_v_tma<RR, RY, false>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<grid3(rows_v, S, spt_f, 8 * RY), b, sm, stream>>>(a, mp);
        }
    }

    // the ring adjoint kernels (tile_z 1 of the adjoint pass)
    template <int RR>
    void launch_adj_ring(int id, int S) {
        Ac3dDev a = dev(S);
        a.spt = spt_a;
        pick_zchunk(8);
        a.zchunk = zchunk;
        auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
        OWL_CHECK(al(a.aex) && al(a.aey) && al(a.aez) && al(a.aepx) && al(a.aepy) && al(a.aepz) && al(a.ap) &&
                      al(a.Sp) && al(a.Svx) && al(a.Svy) && al(a.Svz) && sad % 4 == 0 && a.sslot % 4 == 0 &&
                      fs % 4 == 0 && pitch % 4 == 0,
                  OWL_ERR_UNSUPPORTED, "ring adjoint operands not 16-byte aligned");
        const int rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        const int rows_a = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
        dim3 b(32, 8);
        if (id == OWL_K_ADJ_P) {
            constexpr int sm = ring_bytes_ap<RR>();
            OWL_CUDA(cudaFuncSetAttribute(k_ac3d_adj_p_ring<RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k_ac3d_adj_p_ring<RR><<<grid3(rows_a, S, spt_a, 8), b, sm, stream>>>(a);
        } else {
            constexpr int sm = ring_bytes_av<RR>();
            OWL_CUDA(cudaFuncSetAttribute(k_ac3d_adj_v_ring<RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k_ac3d_adj_v_ring<RR><<<grid3(rows_v, S, spt_a, 8), b, sm, stream>>>(a);
        }
    }

    template <int RR, int TY>
    void launch_adj(int id, int S) {
        Ac3dDev a = dev(S);
        a.spt = spt_a;
        pick_zchunk(TY);
        a.zchunk = zchunk;
        const int rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        const int rows_a = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
        dim3 b(32, TY);
        if (id == OWL_K_ADJ_P) k_ac3d_adj_p<RR, TY><<<grid3(rows_a, S, spt_a, TY), b, 0, stream>>>(a);
        else k_ac3d_adj_v<RR, TY><<<grid3(rows_v, S, spt_a, TY), b, 0, stream>>>(a);
    }

    template <int RR>
    void launch_naive(int id, int S, bool store) {
        Ac3dDev a = dev(S);
        a.spt = spt_f;
        const int zr0 = id == OWL_K_FWD_P ? a.zp0 : std::min(a.zvx0, a.zvz0);
        const int nzb = (a.z1 - zr0 + 1) / 2;
        dim3 b(32, 4, 2), g((NXp + 31) / 32, (NYp + 3) / 4, nzb * ((S + spt_f - 1) / spt_f));
        if (id == OWL_K_FWD_P) {
            if (store) k_ac3d_fwd_p_n<RR, true><<<g, b, 0, stream>>>(a);
            else k_ac3d_fwd_p_n<RR, false><<<g, b, 0, stream>>>(a);
        } else {
            if (store) k_ac3d_fwd_v_n<RR, true><<<g, b, 0, stream>>>(a);
            else k_ac3d_fwd_v_n<RR, false><<<g, b, 0, stream>>>(a);
        }
    }

    // rows per thread of the forward kernels, tuned for each kernel on its own
    // (the shared autotuner times the pair together); -1 = use tz_f
    int tz_fp = -1, tz_fv = -1;
    std::map<int, std::pair<int, int>> tz_split_cache;
    void tune_extra(int S, int k, bool) override {
        (void)k;
        auto it = tz_split_cache.find(S);
        if (it != tz_split_cache.end()) {
            tz_fp = it->second.first;
            tz_fv = it->second.second;
            return;
        }
        int best[2] = {tz_f, tz_f};
        for (int kid : {OWL_K_FWD_P, OWL_K_FWD_V}) {
            float bms = 1e30f;
            for (int tz : {0, 1, 2, 4, 11, 12, 14}) {
                (kid == OWL_K_FWD_P ? tz_fp : tz_fv) = tz;
                launch_kernel(kid, S, false);
                OWL_LAUNCH_CHECK();
                EventTimer tm(stream);
                for (int i = 0; i < 3; ++i) launch_kernel(kid, S, false);
                const float ms = (float)tm.stop_ms();
                launches += 4;
                if (ms < bms) { bms = ms; best[kid] = tz; }
            }
        }
        tz_fp = best[0];
        tz_fv = best[1];
        tz_split_cache[S] = {tz_fp, tz_fv};
    }
    void launch_params(const owl_run_opts& o) override {
        SsgBase::launch_params(o);
        tz_fp = tz_fv = -1;
    }

    template <int RR>
    void launch_r(int id, int S, bool store) {
        if (id <= OWL_K_FWD_V) {
            const int sel = id == OWL_K_FWD_P ? tz_fp : tz_fv;
            const int tz = sel >= 0 ? sel : tz_f;
            // 0: per cell; 1, 2, 4: cp.async ring with that many rows per thread;
            // 11, 12, 14: the TMA ring with 1, 2, 4 rows per thread
            if (tz == 0) launch_naive<RR>(id, S, store);
            else if (tz == 2) launch_fwd<RR, 2>(id, S, store);
            else if (tz == 1) launch_fwd<RR, 1>(id, S, store);
            else if (tz == 4) launch_fwd<RR, 4>(id, S, store);
            else if (tz == 11) launch_fwd_tma<RR, 1>(id, S, store);
            else if (tz == 12) launch_fwd_tma<RR, 2>(id, S, store);
            else launch_fwd_tma<RR, 4>(id, S, store);
        } else {
            if (tz_a == 1) launch_adj_ring<RR>(id, S);
            else if (tz_a == 2) launch_adj<RR, 2>(id, S);
            else if (tz_a == 8) launch_adj<RR, 8>(id, S);
            else launch_adj<RR, 4>(id, S);
        }
    }
    void launch_kernel(int id, int S, bool store) override {
        if (R == 4) launch_r<4>(id, S, store);
        else launch_r<8>(id, S, store);
    }

    double alg_bytes(int id, int S, int groups) const override {
        const double cells = (double)NXp * NYp * NZp;
        const double pml_i = 2.0 * P * ((double)NYp * NZp + (double)NXp * NZp + (double)NXp * NYp);
        const double pml_h = (2.0 * P + 1) * ((double)NYp * NZp + (double)NXp * NZp + (double)NXp * NYp);
        switch (id) {
            case OWL_K_FWD_P: return S * (cells * 20.0 + pml_i * 8.0) + cells * 4.0;
            case OWL_K_FWD_V: return S * (cells * 28.0 + pml_h * 8.0) + cells * 12.0;
            case OWL_K_ADJ_P: return S * (cells * 60.0 + pml_i * 8.0) + cells * 4.0 + groups * cells * 64.0;
            case OWL_K_ADJ_V: return S * (cells * 48.0 + pml_h * 8.0) + cells * 12.0;
        }
        return 0;
    }

    void chain_rule(int S, int groups) override {
        Ac3dDev a = dev(S);
        k_ac3d_chain<<<148 * 8, 256, 0, stream>>>(a, groups, vpp.p, rhop.p, (double)dt, gpad.p, gpad.p + npad(), nxq(),
                                                  nyq(), nzq());
        OWL_LAUNCH_CHECK();
        launches++;
    }
};

Engine* make_ac3d_engine(const owl_ssg_desc& d) { return new Ac3dEngine(d); }

}  // namespace owl
