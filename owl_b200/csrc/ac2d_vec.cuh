// ac2d_vec.cuh -- the 2D acoustic stencil kernels with four consecutive x
// cells per thread (included by ac2d.cu after the one-cell kernels, inside
// namespace owl).
//
// Same arithmetic, per cell and in the same order, as k_ac2d_fwd_p / _fwd_v /
// _adj_p / _adj_v, with the fused point work of those kernels. A thread owns
// cells x .. x + 3 of one row (x - x0 a multiple of 4, so every row access is a
// 16-byte float4): the x arms of its four stencils come from one window of
// 2R + 4 values, f[x - R .. x + R + 3], read as R / 2 + 1 float4 loads, the z
// arms from one float4 per row, and the cell's own values and coefficients
// from one float4 each -- about a fifth of the load instructions of four
// one-cell threads, for the same bytes. The row pitch leaves at least four
// floats after the last stored column (ssg_base.cu), so a window never
// leaves its row. The thread at the right edge of the compute region may own
// fewer than four cells (n < 4): it stores those cells one by one.
#pragma once

// (vec4.cuh is included by ac2d.cu, outside the namespace)
template <int R>
__device__ __forceinline__ void ac2d_win(const float* f, float* w) { win4<R>(f, w); }
// COH: plain (coherent) loads, for fields that the same launch writes (the
// persistent segment kernel); otherwise the read-only path
template <int R, bool COH>
__device__ __forceinline__ void ac2d_winc(const float* f, float* w) {
    if (!COH) {
        win4<R>(f, w);
        return;
    }
#pragma unroll
    for (int q = 0; q < R / 2 + 1; ++q) {
        const float4 t = ld4(f - R + 4 * q);
        w[4 * q] = t.x; w[4 * q + 1] = t.y; w[4 * q + 2] = t.z; w[4 * q + 3] = t.w;
    }
}
template <bool COH>
__device__ __forceinline__ float4 ldc4(const float* p) { return COH ? ld4(p) : ldg4(p); }

struct Ac2dV4 {  // the thread's four cells
    int x, z, n;
    long long o;
};
// the thread's cells in tile (b.x, b.y) of 32 x blockDim.y four-cell threads
__device__ __forceinline__ bool ac2d_v4t(const Ac2dDev& a, int zr0, uint3 b, Ac2dV4& c) {
    c.x = a.x0 + 4 * (b.x * blockDim.x + threadIdx.x);
    c.z = zr0 + b.y * blockDim.y + threadIdx.y;
    c.n = min(4, a.x1 - c.x);
    c.o = (long long)c.z * a.pitch + c.x;
    return c.x < a.x1 && c.z < a.z1;
}
// the launch's own tile: blockIdx, past the leading point-work rows
__device__ __forceinline__ uint3 ac2d_tile(const Ac2dDev& a) {
    return make_uint3(blockIdx.x, (unsigned)ac2d_row(a), blockIdx.z);
}
__device__ __forceinline__ bool ac2d_v4(const Ac2dDev& a, int zr0, Ac2dV4& c) { return ac2d_v4t(a, zr0, ac2d_tile(a), c); }

// tile b of the pressure update of step cur (the device step counter's value)
template <int R, bool STORE, bool FUSE, bool COH = false>
__device__ __forceinline__ void ac2d_fwd_p4_tile(const Ac2dDev& a, uint3 b, int cur) {
    Ac2dV4 c;
    if (!ac2d_v4t(a, a.zp0, b, c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const int cx0 = a.x0 + 4 * b.x * blockDim.x, cz0 = a.zp0 + b.y * blockDim.y;  // the tile's cells
    const float4 dtbk = ldg4(a.dtbk + o);
    bool px[4];
    float ax[4], bx[4];
    bool anyx = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        px[q] = q < n && pml_int(x + q, a.pr, a.nx);
        ax[q] = px[q] ? a.axi[x + q] : 0.f;
        bx[q] = px[q] ? a.bxi[x + q] : 0.f;
        anyx |= px[q];
    }
    const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const float az = pz ? a.azi[z] : 0.f, bz = pz ? a.bzi[z] : 0.f;
    const bool mirror = a.fsurf && z <= a.pr + a.P;
    const long long omir = (long long)(2 * a.pr - z) * a.pitch + x;
    const int s0 = b.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(cur % a.k) * a.sslot : 0;
    const int pt = a.pitch;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst + o;
        const float* vx = a.vx + so;
        const float* vz = a.vz + so;
        // the cells' own values ahead of their stores (see k_ac2d_fwd_p)
        float4 p0 = ld4(a.p + so);
        float4 m1 = anyx ? ld4(a.m1 + so) : zero, m2 = pz ? ld4(a.m2 + so) : zero;
        // whether this CTA holds explosion taps of shot s (its load overlaps the stencil's)
        const bool inj = FUSE && (a.pt.mode & FZ_INJ) &&
                         ac2d_inj_near(a.pt, s, 1, cx0, cx0 + 4 * blockDim.x, cz0, cz0 + blockDim.y);
        float w[2 * R + 4];
        ac2d_winc<R, COH>(vx, w);
        float sx[4] = {0.f, 0.f, 0.f, 0.f}, sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int k = 1; k <= R; ++k) sx[q] = sx[q] + c_fd2[k - 1] * (w[R + q + k] - w[R + q + 1 - k]);
#pragma unroll
        for (int k = 1; k <= R; ++k) {
            const float4 up = ldc4<COH>(vz + k * pt), dn = ldc4<COH>(vz + (1 - k) * pt);
#pragma unroll
            for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fd2[k - 1] * (f4at(up, q) - f4at(dn, q));
        }
        // explosion sources of step t-1 (cur), added where add_source would have
        if (inj) p0 = ac2d_inj4(a.pt, s, 0, x, z, cur - 1, p0, n);
        float4 pn = p0, gS = zero;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float gx = a.idx * sx[q], gz = a.idz * sz[q];
            if (px[q]) {
                const float m = ax[q] * gx + bx[q] * f4at(m1, q);
                f4set(m1, q, m);
                gx = gx + m;
            }
            if (pz) {
                const float m = az * gz + bz * f4at(m2, q);
                f4set(m2, q, m);
                gz = gz + m;
            }
            const float g = gx + gz;
            f4set(pn, q, f4at(p0, q) - f4at(dtbk, q) * g);
            f4set(gS, q, g);
        }
        st4n(a.p + so, pn, n);
        if (anyx) st4n(a.m1 + so, m1, n);
        if (pz) st4n(a.m2 + so, m2, n);
        if (mirror) st4n(a.p + s * a.sst + omir, make_float4(-pn.x, -pn.y, -pn.z, -pn.w), n);
        if (STORE) st4n_cs(a.Sp + slot + s * a.fs + o, gS, n);
    }
}

template <int R, bool STORE, bool FUSE>
__global__ void __launch_bounds__(256) k_ac2d_fwd_p4(Ac2dDev a) {
    pdl_prologue();
    ac2d_fwd_p4_tile<R, STORE, FUSE>(a, ac2d_tile(a), (FUSE || STORE) ? *a.d_step : 0);
}

// tile b of the velocity update of step cur
template <int R, bool STORE, bool FUSE, bool COH = false>
__device__ __forceinline__ void ac2d_fwd_v4_tile(const Ac2dDev& a, uint3 b, int cur) {
    Ac2dV4 c;
    if (!ac2d_v4t(a, min(a.zvx0, a.zvz0), b, c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const int cx0 = a.x0 + 4 * b.x * blockDim.x, cz0 = min(a.zvx0, a.zvz0) + b.y * blockDim.y;
    const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
    const float4 bxc = ldg4(a.dtbx + o), bzc = ldg4(a.dtbz + o);
    bool px[4];
    float ax[4], bx[4];
    bool anyx = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        px[q] = q < n && pml_half(x + q, a.pr, a.nx);
        ax[q] = px[q] ? a.axh[x + q] : 0.f;
        bx[q] = px[q] ? a.bxh[x + q] : 0.f;
        anyx |= px[q];
    }
    const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float az = pz ? a.azh[z] : 0.f, bz = pz ? a.bzh[z] : 0.f;
    const int s0 = b.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(cur % a.k) * a.sslot : 0;
    const int pt = a.pitch;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst + o;
        const float* p = a.p + so;
        const bool inj = FUSE && (a.pt.mode & FZ_INJ);
        const int cx1 = cx0 + 4 * blockDim.x, cz1 = cz0 + blockDim.y;
        const bool injx = inj && ac2d_inj_near(a.pt, s, 2, cx0, cx1, cz0, cz1);
        const bool injz = inj && ac2d_inj_near(a.pt, s, 4, cx0, cx1, cz0, cz1);
        float4 vx0 = dox ? ld4(a.vx + so) : zero, m3 = dox && anyx ? ld4(a.m3 + so) : zero;
        float4 vz0 = doz ? ld4(a.vz + so) : zero, m4 = doz && pz ? ld4(a.m4 + so) : zero;
        if (dox) {
            float w[2 * R + 4];
            ac2d_winc<R, COH>(p, w);
            float4 vn = vx0, hS = zero;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float sx = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (w[R + q + k - 1] - w[R + q - k]);
                float h = a.idx * sx;
                if (px[q]) {
                    const float m = ax[q] * h + bx[q] * f4at(m3, q);
                    f4set(m3, q, m);
                    h = h + m;
                }
                f4set(vn, q, f4at(vx0, q) - f4at(bxc, q) * h);
                f4set(hS, q, h);
            }
            if (anyx) st4n(a.m3 + so, m3, n);
            if (STORE) st4n_cs(a.Svx + slot + s * a.fs + o, hS, n);
            // force sources of step t, added to the updated cells (out of the
            // loop above, so that the calls hold no stencil values live)
            if (FUSE && injx) vn = ac2d_inj4(a.pt, s, 1, x, z, cur, vn, n);
            st4n(a.vx + so, vn, n);
        }
        if (doz) {
            float sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 up = ldc4<COH>(p + (k - 1) * pt), dn = ldc4<COH>(p - k * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fd2[k - 1] * (f4at(up, q) - f4at(dn, q));
            }
            float4 vn = vz0, hS = zero;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float h = a.idz * sz[q];
                if (pz) {
                    const float m = az * h + bz * f4at(m4, q);
                    f4set(m4, q, m);
                    h = h + m;
                }
                f4set(vn, q, f4at(vz0, q) - f4at(bzc, q) * h);
                f4set(hS, q, h);
            }
            if (pz) st4n(a.m4 + so, m4, n);
            if (STORE) st4n_cs(a.Svz + slot + s * a.fs + o, hS, n);
            if (FUSE && injz) vn = ac2d_inj4(a.pt, s, 2, x, z, cur, vn, n);
            st4n(a.vz + so, vn, n);
        }
    }
}

// FUSE: the sampling CTAs; VINJ: also the force sources of the batch
template <int R, bool STORE, bool FUSE, bool VINJ>
__global__ void __launch_bounds__(256) k_ac2d_fwd_v4(const __grid_constant__ Ac2dDev a) {
    pdl_prologue();
    const int cur = (FUSE || STORE) ? *a.d_step : 0;
    if (FUSE && (int)blockIdx.y < a.pt.rows_pt) {
        if (a.pt.mode & FZ_SMP) ac2d_sample(a, cur);
    } else {
        ac2d_fwd_v4_tile<R, STORE, VINJ>(a, ac2d_tile(a), cur);
    }
    if (FUSE && (a.pt.mode & FZ_TICK)) tick_last_block(a.d_step, a.pt.d_done, 1);
}

// PF: the next shot's cell values are loaded before this shot's stores (they
// cannot alias: each shot owns its own slices), so two shots' loads are in
// flight per thread instead of one
template <int R, bool PF>
__device__ __forceinline__ void ac2d_adj_p4_cells(const Ac2dDev& a) {
    Ac2dV4 c;
    if (!ac2d_v4(a, min(min(a.zvx0, a.zvz0), a.zp0), c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool dop = z >= a.zp0, ownx = z >= a.zvx0, ownz = z >= a.zvz0;
    bool px[4];
    float ax[4], bx[4];
    bool anyx = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        px[q] = q < n && pml_int(x + q, a.pr, a.nx);
        ax[q] = px[q] ? a.axi[x + q] : 0.f;
        bx[q] = px[q] ? a.bxi[x + q] : 0.f;
        anyx |= px[q];
    }
    const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const float4 bk = ldg4(a.dtbk + o);
    const float azi = pz ? a.azi[z] : 0.f, bzi = pz ? a.bzi[z] : 0.f;
    const bool mirror = a.fsurf && z <= a.pr + a.P;
    const long long om = (long long)(2 * a.pr - z) * a.pitch + x;
    const int pt = a.pitch;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float gbk[4] = {0.f, 0.f, 0.f, 0.f}, gbx[4] = {0.f, 0.f, 0.f, 0.f}, gbz[4] = {0.f, 0.f, 0.f, 0.f};
    // every read of a shot's cells ahead of its stores (see k_ac2d_adj_p)
    struct Cell {
        float4 vx, svx, vz, svz, p0, sp, m1, m2;
    };
    auto load = [&](int s, Cell& L) {
        const long long sa = s * a.sad + o, ss = slot + s * a.fs + o;
        L.vx = ownx ? ld4(a.avx + sa) : zero;
        L.svx = ownx ? ldcs4(a.Svx + ss) : zero;
        L.vz = ownz ? ld4(a.avz + sa) : zero;
        L.svz = ownz ? ldcs4(a.Svz + ss) : zero;
        L.p0 = dop ? ld4(a.ap + sa) : zero;
        L.sp = dop ? ldcs4(a.Sp + ss) : zero;
        L.m1 = dop && anyx ? ld4(a.am1 + sa) : zero;
        L.m2 = dop && pz ? ld4(a.am2 + sa) : zero;
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
        const float4 vx = c_.vx, svx = c_.svx, vz = c_.vz, svz = c_.svz, p0 = c_.p0, sp = c_.sp, m1 = c_.m1, m2 = c_.m2;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (ownx) gbx[q] += f4at(vx, q) * f4at(svx, q);
            if (ownz) gbz[q] += f4at(vz, q) * f4at(svz, q);
        }
        if (!dop) continue;
        float w[2 * R + 4];
        ac2d_win<R>(a.aex + sa, w);
        float sx[4] = {0.f, 0.f, 0.f, 0.f}, sz[4] = {0.f, 0.f, 0.f, 0.f}, sm[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int k = 1; k <= R; ++k) sx[q] = sx[q] + c_fd2[k - 1] * (w[R + q + 1 - k] - w[R + q + k]);
        const float* ez = a.aez + sa;
#pragma unroll
        for (int k = 1; k <= R; ++k) {
            const float4 lo = ldg4(ez + (1 - k) * pt), hi = ldg4(ez + k * pt);
#pragma unroll
            for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fd2[k - 1] * (f4at(lo, q) - f4at(hi, q));
        }
        if (mirror) {
            // p(i, 2-j) = -p(i, j), j <= 0: the adjoint landing on the mirror row folds back with a minus
            const float* em = a.aez + s * a.sad + om;
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 lo = ldg4(em + (1 - k) * pt), hi = ldg4(em + k * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sm[q] = sm[q] + c_fd2[k - 1] * (f4at(lo, q) - f4at(hi, q));
            }
        }
        float4 ph4 = zero, mn1 = m1, mn2 = m2, epx4 = zero, epz4 = zero;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float dP = a.idx * sx[q] + a.idz * sz[q];
            if (mirror) dP = dP - a.idz * sm[q];
            const float ph = f4at(p0, q) + dP;
            f4set(ph4, q, ph);
            gbk[q] += ph * f4at(sp, q);
            const float qq = -f4at(bk, q) * ph;
            float epx = qq, epz = qq;
            if (px[q]) {
                const float u = qq + f4at(m1, q);
                f4set(mn1, q, bx[q] * u);
                epx = qq + ax[q] * u;
            }
            if (pz) {
                const float u = qq + f4at(m2, q);
                f4set(mn2, q, bzi * u);
                epz = qq + azi * u;
            }
            f4set(epx4, q, epx);
            f4set(epz4, q, epz);
        }
        st4n(a.ap + sa, ph4, n);
        if (anyx) st4n(a.am1 + sa, mn1, n);
        if (pz) st4n(a.am2 + sa, mn2, n);
        st4n(a.aepx + sa, epx4, n);
        st4n(a.aepz + sa, epz4, n);
    }
    const long long go = (long long)blockIdx.z * a.fs + o;
    auto kahan4 = [&](float* G, float* C, const float* g) {
        float4 sm = ld4(G + go), cc = ld4(C + go);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float s_ = f4at(sm, q), c_ = f4at(cc, q);
            kahan_add(s_, c_, g[q]);
            f4set(sm, q, s_);
            f4set(cc, q, c_);
        }
        st4n(G + go, sm, n);
        st4n(C + go, cc, n);
    };
    if (dop) kahan4(a.Gbk, a.Cbk, gbk);
    if (ownx) kahan4(a.Gbx, a.Cbx, gbx);
    if (ownz) kahan4(a.Gbz, a.Cbz, gbz);
}

template <int R>
__global__ void __launch_bounds__(256) k_ac2d_adj_p4(Ac2dDev a) {
    pdl_prologue();
    ac2d_adj_p4_cells<R, false>(a);
}
// the pipelined form, held to 128 registers (two CTAs of 256 per SM)
template <int R>
__global__ void __launch_bounds__(256, 2) k_ac2d_adj_p4_pf(Ac2dDev a) {
    pdl_prologue();
    ac2d_adj_p4_cells<R, true>(a);
}

template <int R>
__device__ __forceinline__ void ac2d_adj_v4_cells(const Ac2dDev& a) {
    Ac2dV4 c;
    if (!ac2d_v4(a, min(a.zvx0, a.zvz0), c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
    bool px[4];
    float ax[4], bx[4];
    bool anyx = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        px[q] = q < n && pml_half(x + q, a.pr, a.nx);
        ax[q] = px[q] ? a.axh[x + q] : 0.f;
        bx[q] = px[q] ? a.bxh[x + q] : 0.f;
        anyx |= px[q];
    }
    const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    const float4 bxc = ldg4(a.dtbx + o), bzc = ldg4(a.dtbz + o);
    const float azh = pz ? a.azh[z] : 0.f, bzh = pz ? a.bzh[z] : 0.f;
    const int pt = a.pitch;
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad + o;
        const float4 vx = dox ? ld4(a.avx + sa) : zero, m3 = dox && anyx ? ld4(a.am3 + sa) : zero;
        const float4 vz = doz ? ld4(a.avz + sa) : zero, m4 = doz && pz ? ld4(a.am4 + sa) : zero;
        if (dox) {
            float w[2 * R + 4];
            ac2d_win<R>(a.aepx + sa, w);
            float4 xh4 = zero, mn = m3, e4 = zero;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float sx = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) sx = sx + c_fd2[k - 1] * (w[R + q - k] - w[R + q + k - 1]);
                const float xh = f4at(vx, q) + a.idx * sx;
                f4set(xh4, q, xh);
                const float qq = -f4at(bxc, q) * xh;
                float e = qq;
                if (px[q]) {
                    const float u = qq + f4at(m3, q);
                    f4set(mn, q, bx[q] * u);
                    e = qq + ax[q] * u;
                }
                f4set(e4, q, e);
            }
            st4n(a.avx + sa, xh4, n);
            if (anyx) st4n(a.am3 + sa, mn, n);
            st4n(a.aex + sa, e4, n);
        }
        if (doz) {
            const float* ep = a.aepz + sa;
            float sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 lo = ldg4(ep - k * pt), hi = ldg4(ep + (k - 1) * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fd2[k - 1] * (f4at(lo, q) - f4at(hi, q));
            }
            float4 zh4 = zero, mn = m4, e4 = zero;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float zh = f4at(vz, q) + a.idz * sz[q];
                f4set(zh4, q, zh);
                const float qq = -f4at(bzc, q) * zh;
                float e = qq;
                if (pz) {
                    const float u = qq + f4at(m4, q);
                    f4set(mn, q, bzh * u);
                    e = qq + azh * u;
                }
                f4set(e4, q, e);
            }
            st4n(a.avz + sa, zh4, n);
            if (pz) st4n(a.am4 + sa, mn, n);
            st4n(a.aez + sa, e4, n);
        }
    }
}

template <int R, bool FUSE>
__global__ void __launch_bounds__(256) k_ac2d_adj_v4(const __grid_constant__ Ac2dDev a) {
    pdl_prologue();
    if (FUSE && (int)blockIdx.y < a.pt.rows_pt) {
        if (a.pt.mode & FZ_SCT) ac2d_scatter(a, *a.d_step);
    } else {
        ac2d_adj_v4_cells<R>(a);
    }
    if (FUSE && (a.pt.mode & FZ_TICK)) tick_last_block(a.d_step, a.pt.d_done, -1);
}

// ------------------------- persistent forward segment -------------------------
// All n steps of a forward segment in one cooperative launch: each block loops
// over the pressure tiles of a step, a grid barrier, the sampling CTAs' work
// and the velocity tiles, a barrier, the next step. Injection, sampling and
// the arithmetic are those of the fused step kernels (same tile functions);
// the fields that the launch itself writes are read with plain (coherent)
// loads, not through the read-only path, whose cache a barrier does not
// invalidate.

// bounded barrier of a cooperative launch: bar[0] counts arrivals, bar[1] is
// the generation. The last block to arrive resets the count and advances the
// generation; the others poll it (with a pause between polls). A wait that
// outlasts PERSIST_SPIN_LIMIT polls, or sees another block's failure, records
// it in *err (the host reports OWL_ERR_TIMEOUT) and returns false, and the
// block leaves the kernel.
constexpr unsigned PERSIST_SPIN_LIMIT = 1u << 21;  // polls (about a second at most)
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        int ok = 1;
        volatile unsigned* vgen = bar + 1;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
        if (atomicAdd(bar, 1u) == nb - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned i = 0;
            while (*vgen == g) {
                if (++i > PERSIST_SPIN_LIMIT || *(volatile int*)err) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

struct Ac2dPersist {
    int n;                   // steps of the segment
    int gx, gy_p, gy_v, gz;  // pressure / velocity tiles: x, rows, shot groups
    int nsmp;                // sampling work items (shots x CTAs per shot; 0: none)
    unsigned* bar;
    int* err;
};

template <int R, bool STORE, bool VINJ>
__global__ void __launch_bounds__(256) k_ac2d_fwd_persist(const __grid_constant__ Ac2dDev a, Ac2dPersist p) {
    // the step counter as the segment starts; no block writes it before every
    // block has passed the last barrier
    const int cur0 = *a.d_step;
    const int np = p.gx * p.gy_p * p.gz, nv = p.nsmp + p.gx * p.gy_v * p.gz;
    for (int i = 0; i < p.n; ++i) {
        const int cur = cur0 + i;
        for (int t = blockIdx.x; t < np; t += gridDim.x) {
            const uint3 b = make_uint3(t % p.gx, (t / p.gx) % p.gy_p, t / (p.gx * p.gy_p));
            ac2d_fwd_p4_tile<R, STORE, true, true>(a, b, cur);
        }
        if (!grid_barrier(p.bar, p.err)) return;
        for (int t = blockIdx.x; t < nv; t += gridDim.x) {
            if (t < p.nsmp) {
                ac2d_sample_cta(a, t, cur);
            } else {
                const int u = t - p.nsmp;
                const uint3 b = make_uint3(u % p.gx, (u / p.gx) % p.gy_v, u / (p.gx * p.gy_v));
                ac2d_fwd_v4_tile<R, STORE, VINJ, true>(a, b, cur);
            }
        }
        if (!grid_barrier(p.bar, p.err)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) *a.d_step = cur0 + p.n;
}
