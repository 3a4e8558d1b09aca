// ac3d_fwd_tma.cuh -- the 3D acoustic forward ring kernels with their tiles
// brought in by TMA (included by ac3d.cu after ac3d_fwd.cuh, inside namespace
// owl).
//
// Same tiles, ring stages, z register queues and arithmetic as k_ac3d_fwd_p /
// k_ac3d_fwd_v (ac3d_fwd.cuh); only the copies differ: per plane, one thread
// issues one tiled cp.async.bulk.tensor per tile (the neighbour tiles with their
// R halo, the ahead plane, the cell's own values, the coefficients) into the
// stage and arms the stage's mbarrier with the stage's bytes; every thread
// waits on the stage's phase (bounded, tma.cuh). No per-thread copy slots, no
// per-thread copy instructions. Tensor maps: the forward state as a 5D array
// (x, y, z, field p / vx / vy / vz, shot), one per tile shape, and the
// coefficients as 3D arrays. Out-of-range rows and columns load as zero, as the
// cp.async kernels' zero-filled chunks.
#pragma once

constexpr int AC3_FP = 0, AC3_FVX = 1, AC3_FVY = 2, AC3_FVZ = 3;  // fields of the state map

struct Ac3Maps {
    CUtensorMap sA;  // state, box (32 + 2R) x TYO: a tile with its x halo
    CUtensorMap sB;  // state, box 32 x (TYO + 2R): a tile with its y halo
    CUtensorMap sC;  // state, box 32 x TYO
    CUtensorMap sD;  // state, box (32 + 2R) x (TYO + 2R): both halos
    CUtensorMap mk, mx, my, mz;  // dtbk, dtbx, dtby, dtbz, box 32 x TYO
};

// the ring starts at the first 1024-byte boundary of the dynamic shared memory
// (TMA destinations stay 128-byte aligned: every tile offset is a multiple of
// 128 bytes); its barriers live after the NS stages
__device__ __forceinline__ float* ac3_ring(float* raw) {
    return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~(uintptr_t)1023);
}
template <int STAGE>
__device__ __forceinline__ uint64_t* ac3_bars(float* ring) {
    return reinterpret_cast<uint64_t*>(ring + AC3_NS * STAGE);
}

// waits (bounded, by thread 0) for the planes [from, to) issued into the ring
__device__ __forceinline__ void ac3_drain(uint64_t* bar, unsigned from, unsigned to) {
    for (unsigned j = from; j < to; ++j) (void)mbar_wait(&bar[j % AC3_NS], (j / AC3_NS) & 1u, nullptr);
}

// p -= dtbk (dx vx + dy vy + dz vz), PML memory fused (module_wavefield.f90:66-102)
template <int R, int RY, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_p_tma(Ac3dDev a, const __grid_constant__ Ac3Maps mp) {
    using T = RingP<R, RY>;
    extern __shared__ __align__(128) float ring_raw[];
    float* ring = ac3_ring(ring_raw);
    uint64_t* bar = ac3_bars<T::STAGE>(ring);
    static_assert((T::OY * 4) % 128 == 0 && (T::OZ * 4) % 128 == 0 && (T::OP * 4) % 128 == 0 &&
                      (T::OB * 4) % 128 == 0 && (T::STAGE * 4) % 128 == 0, "tile offsets must stay 128-byte aligned");
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * T::TYO;
    const int x = bx0 + tx;
    const int nzc = (a.z1 - a.zp0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = a.zp0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool px = pin(x, a.pr, a.nx);
    const float ax = px ? a.axi[x] : 0.f, bx = px ? a.bxi[x] : 0.f;
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const int pl = (int)a.plane;
    bool valid[RY];
    int oxy[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = by0 + ty + 8 * r;
        valid[r] = x < a.x1 && y < a.y1;
        oxy[r] = y * a.pitch + x;
    }
    if (tid == 0) {
        for (int i = 0; i < AC3_NS; ++i) mbar_init(&bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned g = 0, issued = 0;  // planes consumed / issued by this CTA
    bool ok = true;
    for (int s = s0; s < s1 && ok; ++s) {
        const long long so = s * a.sst;
        const float* vz = a.vz + so;
        auto issue = [&](int z, unsigned pos) {
            float* st = ring + (pos % AC3_NS) * T::STAGE;
            uint64_t* b = &bar[pos % AC3_NS];
            fence_proxy_async();
            mbar_expect_tx(b, T::STAGE * 4);
            tma_load_5d(st + T::OX, &mp.sA, bx0 - R, by0, z, AC3_FVX, s, b);
            tma_load_5d(st + T::OY, &mp.sB, bx0, by0 - R, z, AC3_FVY, s, b);
            tma_load_5d(st + T::OZ, &mp.sC, bx0, by0, min(z + 1 + R, a.NZs - 1), AC3_FVZ, s, b);
            tma_load_5d(st + T::OP, &mp.sC, bx0, by0, z, AC3_FP, s, b);
            tma_load_3d(st + T::OB, &mp.mk, bx0, by0, z, b);
        };
        float q[RY][2 * R];  // q[r][j] = vz(z - R + 1 + j)
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
            for (int j = 0; j < 2 * R; ++j) q[r][j] = valid[r] ? vz[(zb - R + 1 + j) * pl + oxy[r]] : 0.f;
        if (tid == 0)
            for (int j = 0; j < AC3_NS - 1 && zb + j < ze; ++j) issue(zb + j, issued++);
        for (int z = zb; z < ze; ++z, ++g) {
            if (tid == 0 && z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, issued++);
            const bool w = mbar_wait(&bar[g % AC3_NS], (g / AC3_NS) & 1u, a.err);
            if (!__syncthreads_and(w)) { ok = false; break; }
            const float* st = ring + (g % AC3_NS) * T::STAGE;
            const int zo = z * pl;
            const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                const int lr = ty + 8 * r;
                if (valid[r]) {
                    const int y = by0 + lr;
                    const float* sx = st + T::OX + lr * T::WX + tx + R;
                    const float* sy = st + T::OY + (lr + R) * 32 + tx;
                    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) gx = gx + c_fd3[k - 1] * (sx[k] - sx[1 - k]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) gy = gy + c_fd3[k - 1] * (sy[k * 32] - sy[(1 - k) * 32]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) gz = gz + c_fd3[k - 1] * (q[r][R - 1 + k] - q[r][R - k]);
                    gx = a.idx * gx; gy = a.idy * gy; gz = a.idz * gz;
                    if (px) {
                        float* m = a.m0 + so + xslab(a, x, y, z);
                        float mv = ax * gx + bx * *m; *m = mv; gx = gx + mv;
                    }
                    if (pin(y, a.pr, a.ny)) {
                        float* m = a.m1 + so + yslab(a, x, y, z);
                        float mv = a.ayi[y] * gy + a.byi[y] * *m; *m = mv; gy = gy + mv;
                    }
                    if (pz) {
                        float* m = a.m2 + so + zslab(a, x, y, z);
                        float mv = a.azi[z] * gz + a.bzi[z] * *m; *m = mv; gz = gz + mv;
                    }
                    const float gs = gx + gy + gz;
                    const int o = zo + oxy[r];
                    const float pn = st[T::OP + lr * 32 + tx] - st[T::OB + lr * 32 + tx] * gs;
                    a.p[so + o] = pn;
                    if (a.fsurf && z <= a.pr + a.P) a.p[so + (2 * a.pr - z) * pl + oxy[r]] = -pn;
                    if (STORE) a.Sp[slot + s * a.fs + o] = gs;
                }
#pragma unroll
                for (int j = 0; j < 2 * R - 1; ++j) q[r][j] = q[r][j + 1];
                q[r][2 * R - 1] = st[T::OZ + lr * 32 + tx];
            }
            __syncthreads();  // the stage is free for the plane issued next
        }
    }
    if (!ok && tid == 0) ac3_drain(bar, g, issued);
}

// vx -= dtbx dx p, vy -= dtby dy p, vz -= dtbz dz p, PML memory fused (module_wavefield.f90:106-170)
template <int R, int RY, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_v_tma(Ac3dDev a, const __grid_constant__ Ac3Maps mp) {
    using T = RingV<R, RY>;
    extern __shared__ __align__(128) float ring_raw[];
    float* ring = ac3_ring(ring_raw);
    uint64_t* bar = ac3_bars<T::STAGE>(ring);
    static_assert((T::OQ * 4) % 128 == 0 && (T::OV * 4) % 128 == 0 && (T::TYO * 32 * 4) % 128 == 0 &&
                      (T::STAGE * 4) % 128 == 0, "tile offsets must stay 128-byte aligned");
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * T::TYO;
    const int x = bx0 + tx;
    const int zr0 = min(a.zvx0, a.zvz0);
    const int nzc = (a.z1 - zr0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = zr0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool px = phf(x, a.pr, a.nx);
    const float ax = px ? a.axh[x] : 0.f, bx = px ? a.bxh[x] : 0.f;
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const int pl = (int)a.plane;
    bool valid[RY];
    int oxy[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int y = by0 + ty + 8 * r;
        valid[r] = x < a.x1 && y < a.y1;
        oxy[r] = y * a.pitch + x;
    }
    if (tid == 0) {
        for (int i = 0; i < AC3_NS; ++i) mbar_init(&bar[i], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned g = 0, issued = 0;
    bool ok = true;
    constexpr int TT = T::TYO * 32;
    for (int s = s0; s < s1 && ok; ++s) {
        const long long so = s * a.sst;
        const float* p = a.p + so;
        auto issue = [&](int z, unsigned pos) {
            float* st = ring + (pos % AC3_NS) * T::STAGE;
            uint64_t* b = &bar[pos % AC3_NS];
            fence_proxy_async();
            mbar_expect_tx(b, T::STAGE * 4);
            tma_load_5d(st + T::OP, &mp.sD, bx0 - R, by0 - R, z, AC3_FP, s, b);
            tma_load_5d(st + T::OQ, &mp.sC, bx0, by0, min(z + R, a.NZs - 1), AC3_FP, s, b);
            tma_load_5d(st + T::OV, &mp.sC, bx0, by0, z, AC3_FVX, s, b);
            tma_load_5d(st + T::OV + TT, &mp.sC, bx0, by0, z, AC3_FVY, s, b);
            tma_load_5d(st + T::OV + 2 * TT, &mp.sC, bx0, by0, z, AC3_FVZ, s, b);
            tma_load_3d(st + T::OV + 3 * TT, &mp.mx, bx0, by0, z, b);
            tma_load_3d(st + T::OV + 4 * TT, &mp.my, bx0, by0, z, b);
            tma_load_3d(st + T::OV + 5 * TT, &mp.mz, bx0, by0, z, b);
        };
        float q[RY][2 * R];  // q[r][j] = p(z - R + j)
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
            for (int j = 0; j < 2 * R; ++j) q[r][j] = valid[r] ? p[(zb - R + j) * pl + oxy[r]] : 0.f;
        if (tid == 0)
            for (int j = 0; j < AC3_NS - 1 && zb + j < ze; ++j) issue(zb + j, issued++);
        for (int z = zb; z < ze; ++z, ++g) {
            if (tid == 0 && z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, issued++);
            const bool w = mbar_wait(&bar[g % AC3_NS], (g / AC3_NS) & 1u, a.err);
            if (!__syncthreads_and(w)) { ok = false; break; }
            const float* st = ring + (g % AC3_NS) * T::STAGE;
            const int zo = z * pl;
            const bool dox = z >= a.zvx0, doz = z >= a.zvz0;
            const bool pz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                const int lr = ty + 8 * r;
                if (valid[r]) {
                    const int y = by0 + lr;
                    const int o = zo + oxy[r];
                    const float* sp = st + T::OP + (lr + R) * T::WX + tx + R;
                    const float* ov = st + T::OV + lr * 32 + tx;
                    if (dox) {
                        float h = 0.f, hy = 0.f;
#pragma unroll
                        for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (sp[k - 1] - sp[-k]);
#pragma unroll
                        for (int k = 1; k <= R; ++k) hy = hy + c_fd3[k - 1] * (sp[(k - 1) * T::WX] - sp[-k * T::WX]);
                        h = a.idx * h;
                        hy = a.idy * hy;
                        if (px) {
                            float* m = a.m3 + so + xslab(a, x, y, z);
                            float mv = ax * h + bx * *m; *m = mv; h = h + mv;
                        }
                        if (phf(y, a.pr, a.ny)) {
                            float* m = a.m4 + so + yslab(a, x, y, z);
                            float mv = a.ayh[y] * hy + a.byh[y] * *m; *m = mv; hy = hy + mv;
                        }
                        a.vx[so + o] = ov[0] - ov[3 * TT] * h;
                        a.vy[so + o] = ov[TT] - ov[4 * TT] * hy;
                        if (STORE) { a.Svx[slot + s * a.fs + o] = h; a.Svy[slot + s * a.fs + o] = hy; }
                    }
                    if (doz) {
                        float h = 0.f;
#pragma unroll
                        for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (q[r][R + k - 1] - q[r][R - k]);
                        h = a.idz * h;
                        if (pz) {
                            float* m = a.m5 + so + zslab(a, x, y, z);
                            float mv = a.azh[z] * h + a.bzh[z] * *m; *m = mv; h = h + mv;
                        }
                        a.vz[so + o] = ov[2 * TT] - ov[5 * TT] * h;
                        if (STORE) a.Svz[slot + s * a.fs + o] = h;
                    }
                }
#pragma unroll
                for (int j = 0; j < 2 * R - 1; ++j) q[r][j] = q[r][j + 1];
                q[r][2 * R - 1] = st[T::OQ + lr * 32 + tx];
            }
            __syncthreads();
        }
    }
    if (!ok && tid == 0) ac3_drain(bar, g, issued);
}

template <int R, int RY>
constexpr int tma_bytes_p() { return 1024 + AC3_NS * RingP<R, RY>::STAGE * 4 + AC3_NS * 8; }
template <int R, int RY>
constexpr int tma_bytes_v() { return 1024 + AC3_NS * RingV<R, RY>::STAGE * 4 + AC3_NS * 8; }
