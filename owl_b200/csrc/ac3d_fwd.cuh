// ac3d_fwd.cuh -- 3D acoustic forward kernels with an asynchronous copy ring
// (included by ac3d.cu after Ac3dDev and the slab helpers).
//
// Block 32 x 8 threads, tile 32 (x) x TYO = 8*RY (y) outputs, each thread owns
// RY rows (y = ty + 8 r); the CTA marches a chunk of z planes. Every operand of
// a plane -- the neighbour tiles with their R halo and the cell's own values --
// is brought into a NS-stage shared-memory ring by 16-byte cp.async copies
// issued NS-1 planes ahead, so HBM loads overlap the arithmetic without holding
// registers. z neighbours come from a register queue of 2R values per row.
#pragma once
// (no namespace block: ac3d.cu includes this inside namespace owl)

#ifndef OWL_AC3_STAGES
#define OWL_AC3_STAGES 4
#endif
constexpr int AC3_NS = OWL_AC3_STAGES;  // ring stages

// cp16 / cp_commit / cp_wait / TileSlots: ring.cuh

template <int R, int RY>
struct RingP {
    static constexpr int TYO = 8 * RY, WX = 32 + 2 * R, CHX = WX / 4;
    // per stage: vx (TYO x WX), vy (TYO+2R x 32), vz ahead (TYO x 32), p (TYO x 32), dtbk (TYO x 32)
    static constexpr int OX = 0, OY = OX + TYO * WX, OZ = OY + (TYO + 2 * R) * 32, OP = OZ + TYO * 32,
                         OB = OP + TYO * 32, STAGE = OB + TYO * 32;
};

// p -= dtbk (dx vx + dy vy + dz vz), PML memory fused (module_wavefield.f90:66-102)
template <int R, int RY, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_p(Ac3dDev a) {
    using T = RingP<R, RY>;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
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
    TileSlots<T::TYO, T::CHX> sx_;
    TileSlots<T::TYO + 2 * R, 8> sy_;
    TileSlots<T::TYO, 8> sc_;
    sx_.init(bx0 - R, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst;
        const float* vx = a.vx + so;
        const float* vy = a.vy + so;
        const float* vz = a.vz + so;
        const float* pp = a.p + so;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OX, vx + zo);
            sy_.copy(st + T::OY, vy + zo);
            const long long za = (long long)min(z + 1 + R, a.NZs - 1) * pl;
            sc_.copy(st + T::OZ, vz + za);
            sc_.copy(st + T::OP, pp + zo);
            sc_.copy(st + T::OB, a.dtbk + zo);
        };
        float q[RY][2 * R];  // q[r][j] = vz(z - R + 1 + j)
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
            for (int j = 0; j < 2 * R; ++j) q[r][j] = valid[r] ? vz[(zb - R + 1 + j) * pl + oxy[r]] : 0.f;
#pragma unroll
        for (int j = 0; j < AC3_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            if (z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, (i + AC3_NS - 1) % AC3_NS);
            cp_commit();
            cp_wait<AC3_NS - 1>();
            __syncthreads();
            const float* st = ring + (i % AC3_NS) * T::STAGE;
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
                    const float g = gx + gy + gz;
                    const int o = zo + oxy[r];
                    const float pn = st[T::OP + lr * 32 + tx] - st[T::OB + lr * 32 + tx] * g;
                    a.p[so + o] = pn;
                    if (a.fsurf && z <= a.pr + a.P) a.p[so + (2 * a.pr - z) * pl + oxy[r]] = -pn;
                    if (STORE) a.Sp[slot + s * a.fs + o] = g;
                }
#pragma unroll
                for (int j = 0; j < 2 * R - 1; ++j) q[r][j] = q[r][j + 1];
                q[r][2 * R - 1] = st[T::OZ + lr * 32 + tx];
            }
            __syncthreads();
        }
        cp_wait<0>();
        __syncthreads();
    }
}

template <int R, int RY>
struct RingV {
    static constexpr int TYO = 8 * RY, WX = 32 + 2 * R, CHX = WX / 4, HY = TYO + 2 * R;
    // per stage: p (HY x WX, both halos), p ahead (TYO x 32), vx, vy, vz, dtbx, dtby, dtbz (TYO x 32 each)
    static constexpr int OP = 0, OQ = HY * WX, OV = OQ + TYO * 32, STAGE = OV + 6 * TYO * 32;
};

// vx -= dtbx dx p, vy -= dtby dy p, vz -= dtbz dz p, PML memory fused (module_wavefield.f90:106-170)
template <int R, int RY, bool STORE>
__global__ void __launch_bounds__(256) k_ac3d_fwd_v(Ac3dDev a) {
    using T = RingV<R, RY>;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
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
    TileSlots<T::HY, T::CHX> sp_;
    TileSlots<T::TYO, 8> sc_;
    sp_.init(bx0 - R, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    for (int s = s0; s < s1; ++s) {
        const long long so = s * a.sst;
        const float* p = a.p + so;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sp_.copy(st + T::OP, p + zo);
            sc_.copy(st + T::OQ, p + (long long)min(z + R, a.NZs - 1) * pl);
            sc_.copy(st + T::OV, a.vx + so + zo);
            sc_.copy(st + T::OV + T::TYO * 32, a.vy + so + zo);
            sc_.copy(st + T::OV + 2 * T::TYO * 32, a.vz + so + zo);
            sc_.copy(st + T::OV + 3 * T::TYO * 32, a.dtbx + zo);
            sc_.copy(st + T::OV + 4 * T::TYO * 32, a.dtby + zo);
            sc_.copy(st + T::OV + 5 * T::TYO * 32, a.dtbz + zo);
        };
        float q[RY][2 * R];  // q[r][j] = p(z - R + j)
#pragma unroll
        for (int r = 0; r < RY; ++r)
#pragma unroll
            for (int j = 0; j < 2 * R; ++j) q[r][j] = valid[r] ? p[(zb - R + j) * pl + oxy[r]] : 0.f;
#pragma unroll
        for (int j = 0; j < AC3_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            if (z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, (i + AC3_NS - 1) % AC3_NS);
            cp_commit();
            cp_wait<AC3_NS - 1>();
            __syncthreads();
            const float* st = ring + (i % AC3_NS) * T::STAGE;
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
                        a.vx[so + o] = ov[0] - ov[3 * T::TYO * 32] * h;
                        a.vy[so + o] = ov[T::TYO * 32] - ov[4 * T::TYO * 32] * hy;
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
                        a.vz[so + o] = ov[2 * T::TYO * 32] - ov[5 * T::TYO * 32] * h;
                        if (STORE) a.Svz[slot + s * a.fs + o] = h;
                    }
                }
#pragma unroll
                for (int j = 0; j < 2 * R - 1; ++j) q[r][j] = q[r][j + 1];
                q[r][2 * R - 1] = st[T::OQ + lr * 32 + tx];
            }
            __syncthreads();
        }
        cp_wait<0>();
        __syncthreads();
    }
}

template <int R, int RY>
constexpr int ring_bytes_p() { return AC3_NS * RingP<R, RY>::STAGE * 4; }
template <int R, int RY>
constexpr int ring_bytes_v() { return AC3_NS * RingV<R, RY>::STAGE * 4; }

