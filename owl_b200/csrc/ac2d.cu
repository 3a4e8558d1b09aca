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
// One time step is two launches over all shots of a batch:
//   k_ac2d_fwd_p : the explosion sources of step t-1 added by the owner of each
//                  tap node (deferred from the end of step t-1, where the
//                  reference adds them after the velocity update), then
//                  p -= dtbk * (dx vx + dz vz), CFS-PML memory fused
//   k_ac2d_fwd_v : vx -= dtbx * dx p ; vz -= dtbz * dz p, CFS-PML memory fused,
//                  force sources of step t added by the tap nodes' owners; extra
//                  CTAs record the receivers of step t+1 from p plus the pending
//                  explosion taps; the last CTA advances the step counter
// The values are those of the reference's order (update, add_source, sample)
// to the bit. A batch whose taps fall outside the nodes a kernel updates keeps
// the separate point kernel of ssg_base.cu (three launches per step).
#include <algorithm>
#include <cstdlib>
#include <cmath>

#include "ssg_base.cuh"
#include "vec4.cuh"

namespace owl {

__constant__ float c_fd2[8];

// point work fused into the stencil kernels (FZ_* modes of ssg_base.cuh)
struct Ac2dPt {
    const int* item_ptr;  // injection items of shot s: [item_ptr[s], item_ptr[s + 1])
    const int4* box;      // per item: field, x0, -, z0 (storage coordinates of its 9 x 9 box)
    const float* bw;      // per item: 81 weights [z][x]
    const float* amp;     // per item: nt amplitudes (stf * amp * dt)
    int nt, rtot, nb, mode;
    int rows_pt;          // leading grid rows of point-work CTAs (0: none); the stencil rows follow
    int fmask;            // fields the batch's sources inject into (bit 0 p, 1 vx, 2 vz)
    const int4* bbox;     // per shot: bounding box (x0, x1, z0, z1) of its p taps, then of its vx / vz taps
    const int* rec_ptr;   // receivers (traces) of shot s: [rec_ptr[s], rec_ptr[s + 1])
    CSRView smp;
    float* rec;
    const int* sct_shot_ptr;  // scatter targets of shot s
    CSRView sct;
    const float* res;
    int* d_done;
};

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
    Ac2dPt pt;
};

__device__ __forceinline__ bool pml_int(int x, int pr, int n) { return x < pr || x >= pr + n; }
__device__ __forceinline__ bool pml_half(int x, int pr, int n) { return x <= pr || x >= pr + n; }
// this CTA's row of stencil tiles: the grid's leading rows are point-work CTAs
// (receiver sampling, residual scatter), so that they run beside the stencil
// CTAs instead of after them
__device__ __forceinline__ int ac2d_row(const Ac2dDev& a) { return (int)blockIdx.y - a.pt.rows_pt; }

// v + the injection of step index ti (0-based) of shot s's sources on field f
// at storage node (x, z), items in order as add_source loops them; taps of
// weight 0 are not taps
// (not inlined: it runs only in the CTAs around a source, and inlined it
// raised the registers of every CTA of the stencil kernels)
__device__ __noinline__ float ac2d_inj_taps(const int* __restrict__ item_ptr, const int4* __restrict__ box,
                                            const float* __restrict__ bw, const float* __restrict__ amp, int nt, int s,
                                            int f, int x, int z, int ti, float v) {
    if ((unsigned)ti >= (unsigned)nt) return v;
    const int i1 = item_ptr[s + 1];
    for (int it = item_ptr[s]; it < i1; ++it) {
        const int4 b = box[it];
        const unsigned dx = (unsigned)(x - b.y), dz = (unsigned)(z - b.w);
        if (b.x == f && dx < (unsigned)BOX_W && dz < (unsigned)BOX_W) {
            const float A = amp[(size_t)it * nt + ti];
            const float w = bw[(size_t)it * (BOX_W * BOX_W) + dz * BOX_W + dx];
            if (A != 0.f && w != 0.f) v = v + A * w;
        }
    }
    return v;
}
__device__ __forceinline__ float ac2d_inj(const Ac2dPt& q, int s, int f, int x, int z, int ti, float v) {
    return ac2d_inj_taps(q.item_ptr, q.box, q.bw, q.amp, q.nt, s, f, x, z, ti, v);
}
// the same for the four cells x .. x + 3 (the first n) of one row: one pass
// over the shot's items, each cell's taps added in item order as above
__device__ __noinline__ float4 ac2d_inj4_taps(const int* __restrict__ item_ptr, const int4* __restrict__ box,
                                              const float* __restrict__ bw, const float* __restrict__ amp, int nt,
                                              int s, int f, int x, int z, int ti, float4 v, int n) {
    if ((unsigned)ti >= (unsigned)nt) return v;
    float r[4] = {v.x, v.y, v.z, v.w};
    const int i1 = item_ptr[s + 1];
    for (int it = item_ptr[s]; it < i1; ++it) {
        const int4 b = box[it];
        const unsigned dz = (unsigned)(z - b.w);
        if (b.x != f || dz >= (unsigned)BOX_W) continue;
        const float A = amp[(size_t)it * nt + ti];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const unsigned dx = (unsigned)(x + q - b.y);
            if (q < n && dx < (unsigned)BOX_W) {
                const float w = bw[(size_t)it * (BOX_W * BOX_W) + dz * BOX_W + dx];
                if (A != 0.f && w != 0.f) r[q] = r[q] + A * w;
            }
        }
    }
    return make_float4(r[0], r[1], r[2], r[3]);
}
__device__ __forceinline__ float4 ac2d_inj4(const Ac2dPt& q, int s, int f, int x, int z, int ti, float4 v, int n) {
    return ac2d_inj4_taps(q.item_ptr, q.box, q.bw, q.amp, q.nt, s, f, x, z, ti, v, n);
}

// whether shot s has a tap on p (fmask 1) or on vx / vz (fmask 2 or 4) in
// columns [x0, x1) x rows [z0, z1) (storage): one read-only load of the shot's
// bounding box, independent of the stencil loads, and the same answer for every
// thread of a CTA, so the per-node lookups run only in the CTAs around sources
__device__ __forceinline__ bool ac2d_inj_near(const Ac2dPt& q, int s, int fmask, int x0, int x1, int z0, int z1) {
    if (!(q.fmask & fmask)) return false;
    const int4 b = __ldg(q.bbox + 2 * s + (fmask == 1 ? 0 : 1));
    return b.x < x1 && b.y > x0 && b.z < z1 && b.w > z0;
}

// ------------------------------- forward ------------------------------------
template <int R, bool STORE, bool FUSE>
__global__ void __launch_bounds__(512) k_ac2d_fwd_p(Ac2dDev a) {
    pdl_prologue();
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = a.zp0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const int cur = FUSE ? *a.d_step : 0;
    const int cx0 = a.x0 + blockIdx.x * blockDim.x, cz0 = a.zp0 + blockIdx.y * blockDim.y;  // the CTA's tile
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
        float p0 = a.p[so];
        const float m1 = px ? a.m1[so] : 0.f, m2 = pz ? a.m2[so] : 0.f;
        // whether this CTA holds explosion taps of shot s (its load overlaps the stencil's)
        const bool inj = FUSE && (a.pt.mode & FZ_INJ) &&
                         ac2d_inj_near(a.pt, s, 1, cx0, cx0 + blockDim.x, cz0, cz0 + blockDim.y);
        float sx = 0.f, sz = 0.f;
#pragma unroll
        for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (__ldg(vx + k) - __ldg(vx + 1 - k));
#pragma unroll
        for (int k = 1; k <= R; ++k) sz = sz + c_fd2[k - 1] * (__ldg(vz + k * pt) - __ldg(vz + (1 - k) * pt));
        // explosion sources of step t-1 (cur), added where add_source would have
        if (inj) p0 = ac2d_inj(a.pt, s, 0, x, z, cur - 1, p0);
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
        if (STORE) __stcs(a.Sp + slot + s * a.fs + o, g);  // streaming: see st4n_cs
    }
}

// receivers of step t+1 (cur + 2) of shot s from p and the pending explosion
// taps of step t (cur), each trace a sequential sum over its taps (the
// sampling of submodule_forward_modeling.f90:58-79 after add_source)
__device__ __noinline__ void ac2d_sample_cta(const Ac2dDev& a, int cta, int cur) {
    const Ac2dPt& q = a.pt;
    const int s = cta / q.nb, part = cta % q.nb, tr = cur + 2;
    if (s >= a.nshots || tr > q.nt) return;
    const int nthr = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
    const float* p = a.p + s * a.sst;
    for (int r = q.rec_ptr[s] + part * nthr + tid; r < q.rec_ptr[s + 1]; r += q.nb * nthr) {
        float acc = 0.f;
        for (int j = q.smp.ptr[r]; j < q.smp.ptr[r + 1]; ++j) {
            const long long off = q.smp.off[j];
            const int zz = (int)(off / a.pitch), xx = (int)(off - (long long)zz * a.pitch);
            acc = acc + ac2d_inj(q, s, 0, xx, zz, cur, p[off]) * q.smp.w[j];
        }
        q.rec[(size_t)(tr - 1) * q.rtot + r] = acc;
    }
}
// the launch's sampling CTAs: the leading grid rows of shot group 0
__device__ __forceinline__ void ac2d_sample(const Ac2dDev& a, int cur) {
    if (blockIdx.z == 0) ac2d_sample_cta(a, blockIdx.y * gridDim.x + blockIdx.x, cur);
}

template <int R, bool STORE, bool FUSE>
__device__ __forceinline__ void ac2d_fwd_v_cells(const Ac2dDev& a, int cur) {
    const int zr0 = min(a.zvx0, a.zvz0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + ac2d_row(a) * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const int cx0 = a.x0 + blockIdx.x * blockDim.x, cz0 = zr0 + ac2d_row(a) * blockDim.y;  // the CTA's tile
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
            float vn = vx0 - bxc * h;
            // force sources of step t
            if (FUSE && (a.pt.mode & FZ_INJ) && ac2d_inj_near(a.pt, s, 2, cx0, cx0 + blockDim.x, cz0, cz0 + blockDim.y))
                vn = ac2d_inj(a.pt, s, 1, x, z, cur, vn);
            a.vx[so] = vn;
            if (STORE) __stcs(a.Svx + slot + s * a.fs + o, h);
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
            float vn = vz0 - bzc * h;
            if (FUSE && (a.pt.mode & FZ_INJ) && ac2d_inj_near(a.pt, s, 4, cx0, cx0 + blockDim.x, cz0, cz0 + blockDim.y))
                vn = ac2d_inj(a.pt, s, 2, x, z, cur, vn);
            a.vz[so] = vn;
            if (STORE) __stcs(a.Svz + slot + s * a.fs + o, h);
        }
    }
}

// the fused instance is held to 32 registers (4 CTAs of 512 per SM), the
// occupancy of the plain kernel: the step is latency bound
template <int R, bool STORE>
__global__ void __launch_bounds__(512) k_ac2d_fwd_v(Ac2dDev a) {
    pdl_prologue();
    ac2d_fwd_v_cells<R, STORE, false>(a, 0);
}

// with the fused point work (VINJ: the batch has force sources, injected by
// the velocity kernel); held to 64 registers (2 CTAs of 512 per SM): at 40
// the injection call and the sampling branch spill
template <int R, bool STORE, bool VINJ>
__global__ void __launch_bounds__(512, 2) k_ac2d_fwd_vf(const __grid_constant__ Ac2dDev a) {
    pdl_prologue();
    const int cur = *a.d_step;
    if ((int)blockIdx.y < a.pt.rows_pt) {
        if (a.pt.mode & FZ_SMP) ac2d_sample(a, cur);
    } else {
        ac2d_fwd_v_cells<R, STORE, VINJ>(a, cur);
    }
    if (a.pt.mode & FZ_TICK) tick_last_block(a.d_step, a.pt.d_done, 1);
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
//
// PF: the next shot's cell values are loaded before this shot's stores (they
// cannot alias: each shot owns its own slices), so two shots' loads are in
// flight per thread instead of one
template <int R, bool PF>
__device__ __forceinline__ void ac2d_adj_p_cells(const Ac2dDev& a) {
    const int zr0 = min(min(a.zvx0, a.zvz0), a.zp0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + ac2d_row(a) * blockDim.y + threadIdx.y;
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
    // every read of a shot's cell is issued ahead of its stores: the arrays
    // share one allocation, so no plain read could move above a store and each
    // would cost its own round trip. Arrays that no thread of this launch
    // writes (the e terms of the neighbours, the stored stencil terms) are read
    // through the read-only path, which the compiler may schedule freely.
    struct Cell {
        float vx, svx, vz, svz, p0, sp, m1, m2;
    };
    auto load = [&](int s, Cell& L) {
        const long long sa = s * a.sad + o, ss = slot + s * a.fs + o;
        L.vx = ownx ? a.avx[sa] : 0.f;
        L.svx = ownx ? __ldcs(a.Svx + ss) : 0.f;
        L.vz = ownz ? a.avz[sa] : 0.f;
        L.svz = ownz ? __ldcs(a.Svz + ss) : 0.f;
        L.p0 = dop ? a.ap[sa] : 0.f;
        L.sp = dop ? __ldcs(a.Sp + ss) : 0.f;
        L.m1 = dop && px ? a.am1[sa] : 0.f;
        L.m2 = dop && pz ? a.am2[sa] : 0.f;
    };
    Cell nx_;
    if (PF && s0 < s1) load(s0, nx_);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad + o;
        Cell c_;
        if (PF) {
            c_ = nx_;
            if (s + 1 < s1) load(s + 1, nx_);
        } else {
            load(s, c_);
        }
        const float vx = c_.vx, svx = c_.svx, vz = c_.vz, svz = c_.svz, p0 = c_.p0, sp = c_.sp, m1 = c_.m1, m2 = c_.m2;
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
__global__ void __launch_bounds__(512) k_ac2d_adj_p(Ac2dDev a) {
    pdl_prologue();
    ac2d_adj_p_cells<R, false>(a);
}
template <int R>
__global__ void __launch_bounds__(512) k_ac2d_adj_p_pf(Ac2dDev a) {
    pdl_prologue();
    ac2d_adj_p_cells<R, true>(a);
}

// adjoint of the sampling of step t: the residual of step t into p^ at the
// receivers' tap nodes, one thread per target node, its contributions summed in
// a fixed order (k_point_adj's scatter phase)
__device__ __noinline__ void ac2d_scatter(const Ac2dDev& a, int t) {
    const Ac2dPt& q = a.pt;
    const int cta = blockIdx.y * gridDim.x + blockIdx.x;
    const int s = cta / q.nb, part = cta % q.nb;
    if (blockIdx.z != 0 || s >= a.nshots || t < 1) return;
    const int nthr = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int it = q.sct_shot_ptr[s] + part * nthr + tid; it < q.sct_shot_ptr[s + 1]; it += q.nb * nthr) {
        float acc = 0.f;
        const int j0 = q.sct.ptr[it], j1 = q.sct.ptr[it + 1];
        for (int j = j0; j < j1; ++j) acc = acc + q.res[(size_t)(t - 1) * q.rtot + q.sct.item[j]] * q.sct.w[j];
        float* f = a.ap + s * a.sad + q.sct.off[j0];
        *f = *f + acc;
    }
}

template <int R>
__device__ __forceinline__ void ac2d_adj_v_cells(const Ac2dDev& a) {
    const int zr0 = min(a.zvx0, a.zvz0);
    int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    int z = zr0 + ac2d_row(a) * blockDim.y + threadIdx.y;
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

template <int R, bool FUSE>
__global__ void __launch_bounds__(512) k_ac2d_adj_v(const __grid_constant__ Ac2dDev a) {
    pdl_prologue();
    if (FUSE && (int)blockIdx.y < a.pt.rows_pt) {
        if (a.pt.mode & FZ_SCT) ac2d_scatter(a, *a.d_step);
    } else {
        ac2d_adj_v_cells<R>(a);
    }
    if (FUSE && (a.pt.mode & FZ_TICK)) tick_last_block(a.d_step, a.pt.d_done, -1);
}

#include "ac2d_vec.cuh"

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

    // injection, sampling and the residual scatter run inside the stencil
    // kernels when every source tap lies on a node its kernel updates and the
    // receivers sample p
    bool fuse_supported() const override { return true; }
    bool fuse_tap_ok(int field, int x, int, int z, bool sampling) const override {
        const bool fsf = desc.free_surface != 0;
        if (sampling) return field == 0;
        const int x0 = R, x1 = R + NXp, z1 = R + NZp;
        const int z0 = field == 0 ? (fsf ? pr + 1 : R) : field == 1 ? (fsf ? pr : R) : (fsf ? pr + 1 : R);
        return field >= 0 && field <= 2 && x >= x0 && x < x1 && z >= z0 && z < z1;
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
        Ac2dPt& q = a.pt;
        q.item_ptr = inj_shot_ptr.p; q.box = inj_box.p; q.bw = inj_bw.p; q.amp = amp.p;
        q.nt = desc.nt; q.rtot = rtot; q.nb = 1; q.mode = fz_mode; q.rows_pt = 0; q.fmask = inj_fmask;
        q.bbox = inj_bbox.p;
        q.rec_ptr = rec_shot_ptr.p; q.smp = view(smp); q.rec = rec.p;
        q.sct_shot_ptr = sct_shot_ptr.p; q.sct = view(sct); q.res = res.p;
        q.d_done = ctr.p + 1;
        return a;
    }

    // tile heights of the autotuner: 4, 8, 16 rows of one-cell threads (32 x
    // tz), or 100 + 2, 4, 8 rows of four-cell threads (k_ac2d_*4, 32 x tz
    // threads covering 128 x tz cells); adjoint pass also 200 + 2, 4, 8 and
    // 300 + 4, 8: the four-cell / one-cell tiles with the adjoint p kernel
    // loading each thread's next shot ahead (when a CTA takes several shots).
    // The same for the forward and adjoint velocity-node kernels measured
    // slower: not built.
    std::vector<int> tune_tz(int pass) const override {
        if (pass == 1) return {4, 8, 16, 304, 308, 102, 104, 108, 202, 204, 208};
        return {4, 8, 16, 102, 104, 108};
    }
    void launch_params(const owl_run_opts& o) override {
        const bool code = o.tile_z >= 100;
        owl_run_opts q = o;
        if (code) q.tile_z = o.tile_z % 100;
        SsgBase::launch_params(q);
        if (code) {
            OWL_CHECK(o.tile_z < 400 && (o.tile_z >= 300 || (tile_x == 32 && q.tile_z >= 1 && q.tile_z <= 8)),
                      OWL_ERR_INVALID,
                      "tile_z: rows, 100 + (1 .. 8) or 200 + (1 .. 8) with tile_x 32, or 300 + rows");
            tz_f = tz_a = o.tile_z;
        }
    }

    template <int RR>
    void launch_r(int id, int S, bool store) {
        const int tzv = (id == OWL_K_FWD_P || id == OWL_K_FWD_V) ? tz_f : tz_a;
        if (tzv >= 100 && tzv < 300) {
            launch_v4<RR>(id, S, store, tzv - 100);
            return;
        }
        // codes 300 + h: the one-cell tiles of h rows, the adjoint p kernel loading each thread's next shot ahead
        const bool pf = tzv >= 300;
        Ac2dDev a = dev(S);
        const int rows_p = a.z1 - a.zp0, rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        const int rows_a = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
        const bool fz = fz_mode != 0;
        // extra CTA rows after the stencil rows for the sampling / scatter work, nb CTAs per shot
        auto add_point_rows = [&](dim3& g, int nb) {
            a.pt.rows_pt = (S * nb + (int)g.x - 1) / (int)g.x;
            a.pt.nb = nb;
            g.y += a.pt.rows_pt;
        };
        if (id == OWL_K_FWD_P || id == OWL_K_FWD_V) {
            a.spt = spt_f;
            const int ty = tz_f % 100;
            dim3 b(tile_x, ty);
            if (id == OWL_K_FWD_P) {
                dim3 g = grid_for(rows_p, S, spt_f, ty);
                if (store) {
                    if (fz) launch_pdl(k_ac2d_fwd_p<RR, true, true>, g, b, 0, stream, a);
                    else launch_pdl(k_ac2d_fwd_p<RR, true, false>, g, b, 0, stream, a);
                } else {
                    if (fz) launch_pdl(k_ac2d_fwd_p<RR, false, true>, g, b, 0, stream, a);
                    else launch_pdl(k_ac2d_fwd_p<RR, false, false>, g, b, 0, stream, a);
                }
            } else {
                dim3 g = grid_for(rows_v, S, spt_f, ty);
                if (fz && (fz_mode & FZ_SMP)) add_point_rows(g, nb_rec);
                const bool vinj = (inj_fmask & 6) != 0;
                if (store) {
                    if (fz) launch_pdl(vinj ? k_ac2d_fwd_vf<RR, true, true> : k_ac2d_fwd_vf<RR, true, false>, g, b, 0,
                                       stream, a);
                    else launch_pdl(k_ac2d_fwd_v<RR, true>, g, b, 0, stream, a);
                } else {
                    if (fz) launch_pdl(vinj ? k_ac2d_fwd_vf<RR, false, true> : k_ac2d_fwd_vf<RR, false, false>, g, b, 0,
                                       stream, a);
                    else launch_pdl(k_ac2d_fwd_v<RR, false>, g, b, 0, stream, a);
                }
            }
        } else {
            a.spt = spt_a;
            const int ty = tz_a % 100;
            dim3 b(tile_x, ty);
            if (id == OWL_K_ADJ_P) {
                if (pf && spt_a > 1) launch_pdl(k_ac2d_adj_p_pf<RR>, grid_for(rows_a, S, spt_a, ty), b, 0, stream, a);
                else launch_pdl(k_ac2d_adj_p<RR>, grid_for(rows_a, S, spt_a, ty), b, 0, stream, a);
            } else {
                dim3 g = grid_for(rows_v, S, spt_a, ty);
                if (fz && (fz_mode & FZ_SCT)) add_point_rows(g, nb_sct);
                if (fz) launch_pdl(k_ac2d_adj_v<RR, true>, g, b, 0, stream, a);
                else launch_pdl(k_ac2d_adj_v<RR, false>, g, b, 0, stream, a);
            }
        }
    }
    // the four-cell kernels: 32 x ty threads over 128 x ty cells
    template <int RR>
    void launch_v4(int id, int S, bool store, int ty) {
        // tile codes 200 + ty: the same tiles, the adjoint p kernel loading each thread's next shot ahead
        const bool pf = ty >= 100;
        ty %= 100;
        Ac2dDev a = dev(S);
        const int rows_p = a.z1 - a.zp0, rows_v = a.z1 - std::min(a.zvx0, a.zvz0);
        const int rows_a = a.z1 - std::min(std::min(a.zvx0, a.zvz0), a.zp0);
        const bool fz = fz_mode != 0;
        auto grid = [&](int rows, int spt) {
            return dim3((NXp + 127) / 128, (rows + ty - 1) / ty, (S + spt - 1) / spt);
        };
        auto add_point_rows = [&](dim3& g, int nb) {
            a.pt.rows_pt = (S * nb + (int)g.x - 1) / (int)g.x;
            a.pt.nb = nb;
            g.y += a.pt.rows_pt;
        };
        const dim3 b(32, ty);
        if (id == OWL_K_FWD_P) {
            a.spt = spt_f;
            const dim3 g = grid(rows_p, spt_f);
            if (store) {
                if (fz) launch_pdl(k_ac2d_fwd_p4<RR, true, true>, g, b, 0, stream, a);
                else launch_pdl(k_ac2d_fwd_p4<RR, true, false>, g, b, 0, stream, a);
            } else {
                if (fz) launch_pdl(k_ac2d_fwd_p4<RR, false, true>, g, b, 0, stream, a);
                else launch_pdl(k_ac2d_fwd_p4<RR, false, false>, g, b, 0, stream, a);
            }
        } else if (id == OWL_K_FWD_V) {
            a.spt = spt_f;
            dim3 g = grid(rows_v, spt_f);
            if (fz && (fz_mode & FZ_SMP)) add_point_rows(g, nb_rec);
            const bool vinj = (inj_fmask & 6) != 0;
            if (store) {
                if (fz) launch_pdl(vinj ? k_ac2d_fwd_v4<RR, true, true, true> : k_ac2d_fwd_v4<RR, true, true, false>, g, b,
                                   0, stream, a);
                else launch_pdl(k_ac2d_fwd_v4<RR, true, false, false>, g, b, 0, stream, a);
            } else {
                if (fz) launch_pdl(vinj ? k_ac2d_fwd_v4<RR, false, true, true> : k_ac2d_fwd_v4<RR, false, true, false>, g,
                                   b, 0, stream, a);
                else launch_pdl(k_ac2d_fwd_v4<RR, false, false, false>, g, b, 0, stream, a);
            }
        } else if (id == OWL_K_ADJ_P) {
            a.spt = spt_a;
            if (pf && spt_a > 1) launch_pdl(k_ac2d_adj_p4_pf<RR>, grid(rows_a, spt_a), b, 0, stream, a);
            else launch_pdl(k_ac2d_adj_p4<RR>, grid(rows_a, spt_a), b, 0, stream, a);
        } else {
            a.spt = spt_a;
            dim3 g = grid(rows_v, spt_a);
            if (fz && (fz_mode & FZ_SCT)) add_point_rows(g, nb_sct);
            if (fz) launch_pdl(k_ac2d_adj_v4<RR, true>, g, b, 0, stream, a);
            else launch_pdl(k_ac2d_adj_v4<RR, false>, g, b, 0, stream, a);
        }
    }
    void launch_kernel(int id, int S, bool store) override {
        if (R == 4) launch_r<4>(id, S, store);
        else launch_r<8>(id, S, store);
    }

    // persistent forward segments (OWL_PERSIST=1): one cooperative launch per
    // segment of the four-cell forward with the fused point work
    DevBuf<unsigned> pbar;  // the grid barrier's arrival count and generation
    int num_sms = 0;
    bool run_steps_persistent(int kind, int n, int S) override {
        const char* e = std::getenv("OWL_PERSIST");
        if (!(e && e[0] == '1' && e[1] == 0) || kind == 2 || !fuse_fwd || tz_f < 100 || tz_f >= 200) return false;
        if (R == 4) return persist_r<4>(kind, n, S);
        return persist_r<8>(kind, n, S);
    }
    template <int RR>
    bool persist_r(int kind, int n, int S) {
        Ac2dDev a = dev(S);
        a.spt = spt_f;
        a.pt.mode = FZ_INJ | (kind == 1 ? 0 : FZ_SMP);
        a.pt.rows_pt = 0;
        a.pt.nb = nb_rec;
        const int ty = tz_f - 100;
        Ac2dPersist p{};
        p.n = n;
        p.gx = (NXp + 127) / 128;
        p.gy_p = (a.z1 - a.zp0 + ty - 1) / ty;
        p.gy_v = (a.z1 - std::min(a.zvx0, a.zvz0) + ty - 1) / ty;
        p.gz = (S + spt_f - 1) / spt_f;
        p.nsmp = kind == 1 ? 0 : S * nb_rec;
        if (!pbar.p) pbar.reserve(2);
        OWL_CUDA(cudaMemsetAsync(pbar.p, 0, 2 * sizeof(unsigned), stream));
        // failure-detection test: OWL_PERSIST_STALL=1 starts the arrival count
        // past the block count, so no block is ever the last to arrive and
        // every barrier wait runs out (the call reports OWL_ERR_TIMEOUT)
        if (const char* st = std::getenv("OWL_PERSIST_STALL"))
            if (st[0] == '1' && st[1] == 0) OWL_CUDA(cudaMemsetAsync(pbar.p, 0x40, sizeof(unsigned), stream));
        p.bar = pbar.p;
        p.err = ctr.p + 3;
        const bool store = kind == 1 || kind == 3, vinj = (inj_fmask & 6) != 0;
        void (*k)(Ac2dDev, Ac2dPersist) =
            store ? (vinj ? k_ac2d_fwd_persist<RR, true, true> : k_ac2d_fwd_persist<RR, true, false>)
                  : (vinj ? k_ac2d_fwd_persist<RR, false, true> : k_ac2d_fwd_persist<RR, false, false>);
        if (!num_sms) {
            int d = 0;
            OWL_CUDA(cudaGetDevice(&d));
            OWL_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, d));
        }
        int per_sm = 0;
        OWL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * ty, 0));
        const int np = p.gx * p.gy_p * p.gz, nv = p.nsmp + p.gx * p.gy_v * p.gz;
        // every block resident at once (the cooperative launch checks it)
        const int nblocks = std::max(1, std::min(per_sm * num_sms, std::max(np, nv)));
        void* args[] = {&a, &p};
        OWL_CUDA(cudaLaunchCooperativeKernel((void*)k, dim3(nblocks), dim3(32, ty), args, 0, stream));
        launches += 1;
        return true;
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
