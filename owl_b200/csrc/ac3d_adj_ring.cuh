// ac3d_adj_ring.cuh -- z-marching adjoint kernels of the 3D acoustic solver with
// an asynchronous copy ring (included by ac3d.cu inside namespace owl, after the
// tiled adjoint kernels).
//
// Block 32 x 8 threads, one row per thread; the CTA marches a chunk of z planes
// per shot. Per plane the e planes that the transposed stencils read along x and
// y arrive with their halos, the "ahead" plane of the z queue, and the cell's
// own adjoint fields, stored stencil terms and coefficients, all through 16-byte
// cp.async copies issued NS-1 planes ahead into an NS-stage shared-memory ring.
// The CPML memories and the Kahan gradient sums are read before the ring wait;
// the gradient sums take one Kahan update per shot. The arithmetic is that of
// k_ac3d_adj_p / k_ac3d_adj_v.
#pragma once

template <int R>
struct RingAP {
    static constexpr int WX = 32 + 2 * R, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // e_x (x halo), e_y (y halo), e_z at z + R + 1; p^, vx^, vy^, vz^, Sp, Svx, Svy, Svz, dtbk
    static constexpr int OX = 0, OY = 8 * WX, OA = OY + HY * 32, OO = OA + T, STAGE = OO + 9 * T;
};

template <int R>
struct RingAV {
    // e_px tile from x = bx0 - R - 4 (aligned), wide enough for the shifted stencil
    static constexpr int WX = 32 + 2 * R + 4, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // e_px (x halo), e_py (y halo, from row by0 - R - 1), e_pz at z + R; vx^, vy^, vz^, dtbx, dtby, dtbz
    static constexpr int OX = 0, OY = 8 * WX, OA = OY + HY * 32, OO = OA + T, STAGE = OO + 6 * T;
};

template <int R>
constexpr int ring_bytes_ap() { return AC3_NS * RingAP<R>::STAGE * 4; }
template <int R>
constexpr int ring_bytes_av() { return AC3_NS * RingAV<R>::STAGE * 4; }

__device__ __forceinline__ void kahan_rmw(float* G, float* C, long long go, float g, float c, float v) {
    kahan_add(g, c, v);
    G[go] = g;
    C[go] = c;
}

template <int R>
__global__ void __launch_bounds__(256) k_ac3d_adj_p_ring(Ac3dDev a) {
    using T = RingAP<R>;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * 8;
    const int x = bx0 + tx, y = by0 + ty;
    const bool valid = x < a.x1 && y < a.y1;
    const int zr0 = min(min(a.zvx0, a.zvz0), a.zp0);
    const int nzc = (a.z1 - zr0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = zr0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool px = pin(x, a.pr, a.nx), py = pin(y, a.pr, a.ny);
    const float axi = valid && px ? a.axi[x] : 0.f, bxi = valid && px ? a.bxi[x] : 0.f;
    const float ayi = valid && py ? a.ayi[y] : 0.f, byi = valid && py ? a.byi[y] : 0.f;
    const long long pl = a.plane;
    const long long oxy = (long long)y * a.pitch + x;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const int lo = ty * 32 + tx;
    TileSlots<8, T::CHX> sx_;
    TileSlots<T::HY, 8> sy_;
    TileSlots<8, 8> sc_;
    sx_.init(bx0 - R, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad, sS = slot + s * a.fs;
        const float* ez = a.aez + sa;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OX, a.aex + sa + zo);
            sy_.copy(st + T::OY, a.aey + sa + zo);
            sc_.copy(st + T::OA, ez + (long long)min(z + R + 1, a.NZs - 1) * pl);
            sc_.copy(st + T::OO, a.ap + sa + zo);
            sc_.copy(st + T::OO + T::T, a.avx + sa + zo);
            sc_.copy(st + T::OO + 2 * T::T, a.avy + sa + zo);
            sc_.copy(st + T::OO + 3 * T::T, a.avz + sa + zo);
            sc_.copy(st + T::OO + 4 * T::T, a.Sp + sS + zo);
            sc_.copy(st + T::OO + 5 * T::T, a.Svx + sS + zo);
            sc_.copy(st + T::OO + 6 * T::T, a.Svy + sS + zo);
            sc_.copy(st + T::OO + 7 * T::T, a.Svz + sS + zo);
            sc_.copy(st + T::OO + 8 * T::T, a.dtbk + zo);
        };
        // z queue of e_z: planes z-R+1 .. z+R
        float q[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) q[j] = valid ? ez[(long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
#pragma unroll
        for (int j = 0; j < AC3_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            const long long o = (long long)z * pl + oxy, go = (long long)grp * a.fs + o;
            const bool dop = z >= a.zp0, ownx = z >= a.zvx0, ownz = z >= a.zvz0;
            const bool pz = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
            // CPML memories and gradient sums of the cell, before the ring wait
            float* m0p = a.am0 + sa + xslab(a, x, y, z);
            float* m1p = a.am1 + sa + yslab(a, x, y, z);
            float* m2p = a.am2 + sa + zslab(a, x, y, z);
            const bool u0 = valid && dop && px, u1 = valid && dop && py, u2 = valid && dop && pz;
            const float m0 = u0 ? *m0p : 0.f, m1 = u1 ? *m1p : 0.f, m2 = u2 ? *m2p : 0.f;
            const bool gk = valid && dop, gx = valid && ownx, gz = valid && ownz;
            const float Gk = gk ? a.Gbk[go] : 0.f, Ck = gk ? a.Cbk[go] : 0.f;
            const float Gx = gx ? a.Gbx[go] : 0.f, Cx = gx ? a.Cbx[go] : 0.f;
            const float Gy = gx ? a.Gby[go] : 0.f, Cy = gx ? a.Cby[go] : 0.f;
            const float Gz = gz ? a.Gbz[go] : 0.f, Cz = gz ? a.Cbz[go] : 0.f;
            cp_wait<AC3_NS - 2>();
            __syncthreads();
            if (z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, (i + AC3_NS - 1) % AC3_NS);
            cp_commit();
            const float* st = ring + (i % AC3_NS) * T::STAGE;
            if (valid) {
                const float* own = st + T::OO + lo;
                if (ownx) {
                    kahan_rmw(a.Gbx, a.Cbx, go, Gx, Cx, own[T::T] * own[5 * T::T]);
                    kahan_rmw(a.Gby, a.Cby, go, Gy, Cy, own[2 * T::T] * own[6 * T::T]);
                }
                if (ownz) kahan_rmw(a.Gbz, a.Cbz, go, Gz, Cz, own[3 * T::T] * own[7 * T::T]);
                if (dop) {
                    const float* sx = st + T::OX + ty * T::WX + tx + R;
                    const float* sy = st + T::OY + (ty + R) * 32 + tx;
                    float sxv = 0.f, syv = 0.f, szv = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) sxv = sxv + c_fd3[k - 1] * (sx[1 - k] - sx[k]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) syv = syv + c_fd3[k - 1] * (sy[(1 - k) * 32] - sy[k * 32]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) szv = szv + c_fd3[k - 1] * (q[R - k] - q[R - 1 + k]);
                    float dP = a.idx * sxv + a.idy * syv + a.idz * szv;
                    if (a.fsurf && z <= a.pr + a.P) {
                        const int zm = 2 * a.pr - z;
                        const float* em = ez + oxy;
                        float sm = 0.f;
#pragma unroll
                        for (int k = 1; k <= R; ++k)
                            sm = sm + c_fd3[k - 1] * (__ldg(em + (long long)(zm - k + 1) * pl) - __ldg(em + (long long)(zm + k) * pl));
                        dP = dP - a.idz * sm;
                    }
                    const float ph = own[0] + dP;
                    a.ap[sa + o] = ph;
                    kahan_rmw(a.Gbk, a.Cbk, go, Gk, Ck, ph * own[4 * T::T]);
                    const float qv = -own[8 * T::T] * ph;
                    float ex = qv, ey = qv, ez2 = qv;
                    if (px) { const float u = qv + m0; *m0p = bxi * u; ex = qv + axi * u; }
                    if (py) { const float u = qv + m1; *m1p = byi * u; ey = qv + ayi * u; }
                    if (pz) { const float u = qv + m2; *m2p = a.bzi[z] * u; ez2 = qv + a.azi[z] * u; }
                    a.aepx[sa + o] = ex;
                    a.aepy[sa + o] = ey;
                    a.aepz[sa + o] = ez2;
                }
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) q[j] = q[j + 1];
            q[2 * R - 1] = st[T::OA + lo];
        }
        cp_wait<0>();
        __syncthreads();
    }
}

template <int R>
__global__ void __launch_bounds__(256) k_ac3d_adj_v_ring(Ac3dDev a) {
    using T = RingAV<R>;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * 8;
    const int x = bx0 + tx, y = by0 + ty;
    const bool valid = x < a.x1 && y < a.y1;
    const int zr0 = min(a.zvx0, a.zvz0);
    const int nzc = (a.z1 - zr0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = zr0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool px = phf(x, a.pr, a.nx), py = phf(y, a.pr, a.ny);
    const float axh = valid && px ? a.axh[x] : 0.f, bxh = valid && px ? a.bxh[x] : 0.f;
    const float ayh = valid && py ? a.ayh[y] : 0.f, byh = valid && py ? a.byh[y] : 0.f;
    const long long pl = a.plane;
    const long long oxy = (long long)y * a.pitch + x;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const int lo = ty * 32 + tx;
    TileSlots<8, T::CHX> sx_;
    TileSlots<T::HY, 8> sy_;
    TileSlots<8, 8> sc_;
    sx_.init(bx0 - R - 4, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R - 1, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    for (int s = s0; s < s1; ++s) {
        const long long sa = s * a.sad;
        const float* epz = a.aepz + sa;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OX, a.aepx + sa + zo);
            sy_.copy(st + T::OY, a.aepy + sa + zo);
            sc_.copy(st + T::OA, epz + (long long)min(z + R, a.NZs - 1) * pl);
            sc_.copy(st + T::OO, a.avx + sa + zo);
            sc_.copy(st + T::OO + T::T, a.avy + sa + zo);
            sc_.copy(st + T::OO + 2 * T::T, a.avz + sa + zo);
            sc_.copy(st + T::OO + 3 * T::T, a.dtbx + zo);
            sc_.copy(st + T::OO + 4 * T::T, a.dtby + zo);
            sc_.copy(st + T::OO + 5 * T::T, a.dtbz + zo);
        };
        // z queue of e_pz: planes z-R .. z+R-1
        float q[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) q[j] = valid ? epz[(long long)(zb - R + j) * pl + oxy] : 0.f;
#pragma unroll
        for (int j = 0; j < AC3_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            const long long o = (long long)z * pl + oxy;
            const bool ox = z >= a.zvx0, oz = z >= a.zvz0;
            const bool pzz = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
            float* m3p = a.am3 + sa + xslab(a, x, y, z);
            float* m4p = a.am4 + sa + yslab(a, x, y, z);
            float* m5p = a.am5 + sa + zslab(a, x, y, z);
            const float m3 = valid && ox && px ? *m3p : 0.f, m4 = valid && ox && py ? *m4p : 0.f;
            const float m5 = valid && oz && pzz ? *m5p : 0.f;
            cp_wait<AC3_NS - 2>();
            __syncthreads();
            if (z + AC3_NS - 1 < ze) issue(z + AC3_NS - 1, (i + AC3_NS - 1) % AC3_NS);
            cp_commit();
            const float* st = ring + (i % AC3_NS) * T::STAGE;
            if (valid) {
                const float* own = st + T::OO + lo;
                if (ox) {
                    // tile column c holds cell bx0 - R - 4 + c; row r holds cell by0 - R - 1 + r
                    const float* sx = st + T::OX + ty * T::WX + tx + R + 4;
                    const float* sy = st + T::OY + (ty + R + 1) * 32 + tx;
                    float h = 0.f, hy = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (sx[-k] - sx[k - 1]);
#pragma unroll
                    for (int k = 1; k <= R; ++k) hy = hy + c_fd3[k - 1] * (sy[-k * 32] - sy[(k - 1) * 32]);
                    const float xh = own[0] + a.idx * h;
                    const float yh = own[T::T] + a.idy * hy;
                    a.avx[sa + o] = xh;
                    a.avy[sa + o] = yh;
                    const float qx = -own[3 * T::T] * xh, qy = -own[4 * T::T] * yh;
                    float ex = qx, ey = qy;
                    if (px) { const float u = qx + m3; *m3p = bxh * u; ex = qx + axh * u; }
                    if (py) { const float u = qy + m4; *m4p = byh * u; ey = qy + ayh * u; }
                    a.aex[sa + o] = ex;
                    a.aey[sa + o] = ey;
                }
                if (oz) {
                    float h = 0.f;
#pragma unroll
                    for (int k = 1; k <= R; ++k) h = h + c_fd3[k - 1] * (q[R - k] - q[R + k - 1]);
                    const float zh = own[2 * T::T] + a.idz * h;
                    a.avz[sa + o] = zh;
                    const float qz = -own[5 * T::T] * zh;
                    float ez = qz;
                    if (pzz) { const float u = qz + m5; *m5p = a.bzh[z] * u; ez = qz + a.azh[z] * u; }
                    a.aez[sa + o] = ez;
                }
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) q[j] = q[j + 1];
            q[2 * R - 1] = st[T::OA + lo];
        }
        cp_wait<0>();
        __syncthreads();
    }
}
