// el3d_ring_adj.cuh -- z-marching adjoint kernels of the 3D elastic solver
// (included by el3d.cu inside namespace owl, after the per-cell adjoint kernels,
// e3_kahan and pml_adr). Half-width R, no free surface.
//
// The scheme of the forward ring kernels (el3d_ring.cuh): a 32 x 8 CTA marches a
// chunk of z planes per shot. Per plane, through 16-byte cp.async copies issued
// NS-1 planes ahead into an NS-stage shared-memory ring: the e-term planes the
// transposed stencils read along x and y (with their halos), the "ahead" planes
// of the z register queues, the buoyancies (moduli), and the cell's own adjoint
// fields and stored stencil terms. The CPML memories and the Kahan gradient sums
// of the cell are read before the ring wait, so that their latency overlaps it;
// the sums take one Kahan update per shot. The arithmetic is that of
// k_el3d_adj_v / k_el3d_adj_s.
#pragma once

constexpr int E3RA_NS_V = 4, E3RA_NS_S = 3;  // ring stages (the stress kernel's stage is larger)

template <int R>
struct RingA3V {
    static constexpr int WX = 32 + 2 * R, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // x-halo tiles e_xvx, e_xvy, e_xvz; y-halo tiles e_yvx, e_yvy, e_yvz; ahead tiles
    // e_zvx, e_zvy (plane z + R + 1), e_zvz (z + R); bx, by, bz; vx^, vy^, vz^; S6, S7, S8
    static constexpr int OX = 0, OY = 3 * 8 * WX, OA = OY + 3 * HY * 32, OB = OA + 3 * T, OV = OB + 3 * T,
                         OS = OV + 3 * T, STAGE = OS + 3 * T;
};

template <int R>
struct RingA3S {
    static constexpr int WX = 32 + 2 * R, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // x-halo tiles e_xxx, e_xxz, e_xxy; y-halo tiles e_yyy, e_yyz, e_yxy; ahead tiles
    // e_zzz (plane z + R + 1), e_zyz, e_zxz (z + R); nine moduli; six stress adjoints; S0..S5
    static constexpr int OX = 0, OY = 3 * 8 * WX, OA = OY + 3 * HY * 32, OM = OA + 3 * T, OV = OM + 9 * T,
                         OS = OV + 6 * T, STAGE = OS + 6 * T;
};

template <int R>
constexpr int e3ra_bytes_v() { return E3RA_NS_V * RingA3V<R>::STAGE * 4; }
template <int R>
constexpr int e3ra_bytes_s() { return E3RA_NS_S * RingA3S<R>::STAGE * 4; }

// Kahan update of correlation q with the sum / compensation read ahead
__device__ __forceinline__ void e3_kahan_rw(float* G, long long gg, long long go, int q, float sm, float c, float v) {
    kahan_add(sm, c, v);
    G[q * gg + go] = sm;
    G[(12 + q) * gg + go] = c;
}

// velocity nodes: v^ += D^T e (stress-derivative e terms), rho correlations,
// adjoint PML terms of the velocity derivatives
template <int R, bool MP>
__global__ void __launch_bounds__(256, 2) k_el3d_adj_v_ring(El3dDev a) {
    using T = RingA3V<R>;
    constexpr int NS = E3RA_NS_V;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * 8;
    const int x = bx0 + tx, y = by0 + ty;
    const int nzc = (a.z1 - a.z0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = a.z0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool valid = x < a.x1 && y < a.y1;
    const long long pl = a.plane, fs = a.fs;
    const int oxy = y * a.pitch + x;
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const float axi = valid ? a.axi[x] : 0.f, bxi = valid ? a.bxi[x] : 0.f;
    const float axh = valid ? a.axh[x] : 0.f, bxh = valid ? a.bxh[x] : 0.f;
    const float ayi = valid ? a.ayi[y] : 0.f, byi = valid ? a.byi[y] : 0.f;
    const float ayh = valid ? a.ayh[y] : 0.f, byh = valid ? a.byh[y] : 0.f;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    TileSlots<8, T::CHX> sx_;
    TileSlots<T::HY, 8> sy_;
    TileSlots<8, 8> sc_;
    sx_.init(bx0 - R, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    const int lo = ty * 32 + tx;
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        const float* e = ad + 27 * fs;
        float* ew = ad + 27 * fs;
        float* mh = ad + 9 * fs;
        const float* Ss = a.S + slot + s * fs;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OX, e + N_XVX * fs + zo);
            sx_.copy(st + T::OX + 8 * T::WX, e + N_XVY * fs + zo);
            sx_.copy(st + T::OX + 16 * T::WX, e + N_XVZ * fs + zo);
            sy_.copy(st + T::OY, e + N_YVX * fs + zo);
            sy_.copy(st + T::OY + T::HY * 32, e + N_YVY * fs + zo);
            sy_.copy(st + T::OY + 2 * T::HY * 32, e + N_YVZ * fs + zo);
            const long long z1 = (long long)min(z + R + 1, a.NZs - 1) * pl, z0 = (long long)min(z + R, a.NZs - 1) * pl;
            sc_.copy(st + T::OA, e + N_ZVX * fs + z1);
            sc_.copy(st + T::OA + T::T, e + N_ZVY * fs + z1);
            sc_.copy(st + T::OA + 2 * T::T, e + N_ZVZ * fs + z0);
            sc_.copy(st + T::OB, a.bx + zo);
            sc_.copy(st + T::OB + T::T, a.by + zo);
            sc_.copy(st + T::OB + 2 * T::T, a.bz + zo);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                sc_.copy(st + T::OV + q * T::T, ad + (E3_VX + q) * fs + zo);
                sc_.copy(st + T::OS + q * T::T, Ss + (6 + q) * a.sterm + zo);
            }
        };
        // z queues: e_zvx, e_zvy planes z-R+1 .. z+R (transposed M), e_zvz planes z-R .. z+R-1 (transposed P)
        float qx[2 * R], qy[2 * R], qz[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) {
            qx[j] = valid ? e[N_ZVX * fs + (long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
            qy[j] = valid ? e[N_ZVY * fs + (long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
            qz[j] = valid ? e[N_ZVZ * fs + (long long)(zb - R + j) * pl + oxy] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            // CPML memories and gradient sums of the cell, before the ring wait
            const long long o = (long long)z * pl + oxy, go = (long long)grp * fs + o;
            const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
            const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
            const bool sh_vx = valid && (oxh || oyi || ozi), sh_vy = valid && (oxi || oyh || ozi),
                       sh_vz = valid && (oxi || oyi || ozh);
            const bool p0 = sh_vx && (MP || axh != 0.f), p1 = sh_vx && (MP || ayi != 0.f), p2 = sh_vx && (MP || azi != 0.f);
            const bool p3 = sh_vy && (MP || axi != 0.f), p4 = sh_vy && (MP || ayh != 0.f), p5 = sh_vy && (MP || azi != 0.f);
            const bool p6 = sh_vz && (MP || axi != 0.f), p7 = sh_vz && (MP || ayi != 0.f), p8 = sh_vz && (MP || azh != 0.f);
            const float m0 = p0 ? mh[N_XXX * fs + o] : 0.f, m1 = p1 ? mh[N_YXY * fs + o] : 0.f;
            const float m2 = p2 ? mh[N_ZXZ * fs + o] : 0.f, m3 = p3 ? mh[N_XXY * fs + o] : 0.f;
            const float m4 = p4 ? mh[N_YYY * fs + o] : 0.f, m5 = p5 ? mh[N_ZYZ * fs + o] : 0.f;
            const float m6 = p6 ? mh[N_XXZ * fs + o] : 0.f, m7 = p7 ? mh[N_YYZ * fs + o] : 0.f;
            const float m8 = p8 ? mh[N_ZZZ * fs + o] : 0.f;
            float g[3], c[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                g[q] = valid ? a.G[(9 + q) * a.gg + go] : 0.f;
                c[q] = valid ? a.G[(21 + q) * a.gg + go] : 0.f;
            }
            cp_wait<NS - 2>();
            __syncthreads();
            if (z + NS - 1 < ze) issue(z + NS - 1, (i + NS - 1) % NS);
            cp_commit();
            const float* st = ring + (i % NS) * T::STAGE;
            if (valid) {
                const float* xa = st + T::OX + ty * T::WX + tx + R;  // e_xvx
                const float* xb = xa + 8 * T::WX;                    // e_xvy
                const float* xc = xb + 8 * T::WX;                    // e_xvz
                const float* ya = st + T::OY + (ty + R) * 32 + tx;   // e_yvx
                const float* yb = ya + T::HY * 32;                   // e_yvy
                const float* yc = yb + T::HY * 32;                   // e_yvz
                const float* ov = st + T::OV + lo;
                const float* os = st + T::OS + lo;
                const float* ob = st + T::OB + lo;
                float tpx = 0.f, tmx = 0.f, tmy = 0.f;
                // vx^ += Dx^T e_xvx (P) + Dz^T e_zvx (M) + Dy^T e_yvx (M)
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    tpx = tpx + c_fd3e[q - 1] * (xa[-q] - xa[q - 1]);
                    tmx = tmx + c_fd3e[q - 1] * (qx[R - q] - qx[R - 1 + q]);
                    tmy = tmy + c_fd3e[q - 1] * (ya[(1 - q) * 32] - ya[q * 32]);
                }
                float v = ov[0] + a.idx * tpx + a.idz * tmx + a.idy * tmy;
                ad[E3_VX * fs + o] = v;
                e3_kahan_rw(a.G, a.gg, go, 9, g[0], c[0], v * os[0]);
                float qq = ob[0] * v, e1 = qq, e2 = qq, e3 = qq;
                if (p0) e1 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 0) : axh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 0) : bxh, m0, mh + N_XXX * fs + o);
                if (p1) e2 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 1) : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 1) : byi, m1, mh + N_YXY * fs + o);
                if (p2) e3 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 2) : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 2) : bzi, m2, mh + N_ZXZ * fs + o);
                ew[N_XXX * fs + o] = e1; ew[N_YXY * fs + o] = e2; ew[N_ZXZ * fs + o] = e3;
                // vy^ += Dy^T e_yvy (P) + Dz^T e_zvy (M) + Dx^T e_xvy (M)
                tpx = 0.f; tmx = 0.f; tmy = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    tpx = tpx + c_fd3e[q - 1] * (yb[-q * 32] - yb[(q - 1) * 32]);
                    tmx = tmx + c_fd3e[q - 1] * (qy[R - q] - qy[R - 1 + q]);
                    tmy = tmy + c_fd3e[q - 1] * (xb[1 - q] - xb[q]);
                }
                v = ov[T::T] + a.idy * tpx + a.idz * tmx + a.idx * tmy;
                ad[E3_VY * fs + o] = v;
                e3_kahan_rw(a.G, a.gg, go, 10, g[1], c[1], v * os[T::T]);
                qq = ob[T::T] * v; e1 = qq; e2 = qq; e3 = qq;
                if (p3) e1 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 3) : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 3) : bxi, m3, mh + N_XXY * fs + o);
                if (p4) e2 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 4) : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 4) : byh, m4, mh + N_YYY * fs + o);
                if (p5) e3 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 5) : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 5) : bzi, m5, mh + N_ZYZ * fs + o);
                ew[N_XXY * fs + o] = e1; ew[N_YYY * fs + o] = e2; ew[N_ZYZ * fs + o] = e3;
                // vz^ += Dz^T e_zvz (P) + Dy^T e_yvz (M) + Dx^T e_xvz (M)
                tpx = 0.f; tmx = 0.f; tmy = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    tpx = tpx + c_fd3e[q - 1] * (qz[R - q] - qz[R + q - 1]);
                    tmx = tmx + c_fd3e[q - 1] * (yc[(1 - q) * 32] - yc[q * 32]);
                    tmy = tmy + c_fd3e[q - 1] * (xc[1 - q] - xc[q]);
                }
                v = ov[2 * T::T] + a.idz * tpx + a.idy * tmx + a.idx * tmy;
                ad[E3_VZ * fs + o] = v;
                e3_kahan_rw(a.G, a.gg, go, 11, g[2], c[2], v * os[2 * T::T]);
                qq = ob[2 * T::T] * v; e1 = qq; e2 = qq; e3 = qq;
                if (p6) e1 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 6) : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 6) : bxi, m6, mh + N_XXZ * fs + o);
                if (p7) e2 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 7) : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 7) : byi, m7, mh + N_YYZ * fs + o);
                if (p8) e3 = pml_adr(qq, MP ? e3_ca<E3_PERM_S>(a, o, 9, 8) : azh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 8) : bzh, m8, mh + N_ZZZ * fs + o);
                ew[N_XXZ * fs + o] = e1; ew[N_YYZ * fs + o] = e2; ew[N_ZZZ * fs + o] = e3;
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) {
                qx[j] = qx[j + 1];
                qy[j] = qy[j + 1];
                qz[j] = qz[j + 1];
            }
            qx[2 * R - 1] = st[T::OA + lo];
            qy[2 * R - 1] = st[T::OA + T::T + lo];
            qz[2 * R - 1] = st[T::OA + 2 * T::T + lo];
        }
        cp_wait<0>();
        __syncthreads();
    }
}

// stress nodes: sigma^ += D^T e (velocity-derivative e terms), Cij
// correlations, adjoint PML terms of the stress derivatives
template <int R, bool MP>
__global__ void __launch_bounds__(256, 2) k_el3d_adj_s_ring(El3dDev a) {
    using T = RingA3S<R>;
    constexpr int NS = E3RA_NS_S;
    extern __shared__ __align__(16) float ring[];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx0 = a.x0 + blockIdx.x * 32, by0 = a.y0 + blockIdx.y * 8;
    const int x = bx0 + tx, y = by0 + ty;
    const int nzc = (a.z1 - a.z0 + a.zchunk - 1) / a.zchunk;
    const int zc = blockIdx.z % nzc, grp = blockIdx.z / nzc;
    const int zb = a.z0 + zc * a.zchunk, ze = min(a.z1, zb + a.zchunk);
    const bool valid = x < a.x1 && y < a.y1;
    const long long pl = a.plane, fs = a.fs;
    const int oxy = y * a.pitch + x;
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const float axi = valid ? a.axi[x] : 0.f, bxi = valid ? a.bxi[x] : 0.f;
    const float axh = valid ? a.axh[x] : 0.f, bxh = valid ? a.bxh[x] : 0.f;
    const float ayi = valid ? a.ayi[y] : 0.f, byi = valid ? a.byi[y] : 0.f;
    const float ayh = valid ? a.ayh[y] : 0.f, byh = valid ? a.byh[y] : 0.f;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    TileSlots<8, T::CHX> sx_;
    TileSlots<T::HY, 8> sy_;
    TileSlots<8, 8> sc_;
    sx_.init(bx0 - R, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    const int lo = ty * 32 + tx;
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        const float* e = ad + 27 * fs;
        float* ew = ad + 27 * fs;
        float* mh = ad + 9 * fs;
        const float* Ss = a.S + slot + s * fs;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OX, e + N_XXX * fs + zo);
            sx_.copy(st + T::OX + 8 * T::WX, e + N_XXZ * fs + zo);
            sx_.copy(st + T::OX + 16 * T::WX, e + N_XXY * fs + zo);
            sy_.copy(st + T::OY, e + N_YYY * fs + zo);
            sy_.copy(st + T::OY + T::HY * 32, e + N_YYZ * fs + zo);
            sy_.copy(st + T::OY + 2 * T::HY * 32, e + N_YXY * fs + zo);
            const long long z1 = (long long)min(z + R + 1, a.NZs - 1) * pl, z0 = (long long)min(z + R, a.NZs - 1) * pl;
            sc_.copy(st + T::OA, e + N_ZZZ * fs + z1);
            sc_.copy(st + T::OA + T::T, e + N_ZYZ * fs + z0);
            sc_.copy(st + T::OA + 2 * T::T, e + N_ZXZ * fs + z0);
            sc_.copy(st + T::OM, a.c11 + zo);
            sc_.copy(st + T::OM + T::T, a.c12 + zo);
            sc_.copy(st + T::OM + 2 * T::T, a.c13 + zo);
            sc_.copy(st + T::OM + 3 * T::T, a.c22 + zo);
            sc_.copy(st + T::OM + 4 * T::T, a.c23 + zo);
            sc_.copy(st + T::OM + 5 * T::T, a.c33 + zo);
            sc_.copy(st + T::OM + 6 * T::T, a.c44e + zo);
            sc_.copy(st + T::OM + 7 * T::T, a.c55e + zo);
            sc_.copy(st + T::OM + 8 * T::T, a.c66e + zo);
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                sc_.copy(st + T::OV + q * T::T, ad + (E3_XX + q) * fs + zo);
                sc_.copy(st + T::OS + q * T::T, Ss + q * a.sterm + zo);
            }
        };
        // z queues: e_zzz planes z-R+1 .. z+R (transposed M); e_zyz, e_zxz planes z-R .. z+R-1 (transposed P)
        float qz[2 * R], qy[2 * R], qx[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) {
            qz[j] = valid ? e[N_ZZZ * fs + (long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
            qy[j] = valid ? e[N_ZYZ * fs + (long long)(zb - R + j) * pl + oxy] : 0.f;
            qx[j] = valid ? e[N_ZXZ * fs + (long long)(zb - R + j) * pl + oxy] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            const long long o = (long long)z * pl + oxy, go = (long long)grp * fs + o;
            const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
            const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
            const bool sh_n = valid && (oxi || oyi || ozi), sh_yz = valid && (oxi || oyh || ozh),
                       sh_xz = valid && (oxh || oyi || ozh), sh_xy = valid && (oxh || oyh || ozi);
            const bool p0 = sh_n && (MP || axi != 0.f), p1 = sh_n && (MP || ayi != 0.f), p2 = sh_n && (MP || azi != 0.f);
            const bool p3 = sh_yz && (MP || azh != 0.f), p4 = sh_yz && (MP || ayh != 0.f);
            const bool p5 = sh_xz && (MP || azh != 0.f), p6 = sh_xz && (MP || axh != 0.f);
            const bool p7 = sh_xy && (MP || ayh != 0.f), p8 = sh_xy && (MP || axh != 0.f);
            const float m0 = p0 ? mh[N_XVX * fs + o] : 0.f, m1 = p1 ? mh[N_YVY * fs + o] : 0.f;
            const float m2 = p2 ? mh[N_ZVZ * fs + o] : 0.f, m3 = p3 ? mh[N_ZVY * fs + o] : 0.f;
            const float m4 = p4 ? mh[N_YVZ * fs + o] : 0.f, m5 = p5 ? mh[N_ZVX * fs + o] : 0.f;
            const float m6 = p6 ? mh[N_XVZ * fs + o] : 0.f, m7 = p7 ? mh[N_YVX * fs + o] : 0.f;
            const float m8 = p8 ? mh[N_XVY * fs + o] : 0.f;
            float g[9], c[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                g[q] = valid ? a.G[q * a.gg + go] : 0.f;
                c[q] = valid ? a.G[(12 + q) * a.gg + go] : 0.f;
            }
            cp_wait<NS - 2>();
            __syncthreads();
            if (z + NS - 1 < ze) issue(z + NS - 1, (i + NS - 1) % NS);
            cp_commit();
            const float* st = ring + (i % NS) * T::STAGE;
            if (valid) {
                const float* xa = st + T::OX + ty * T::WX + tx + R;  // e_xxx
                const float* xb = xa + 8 * T::WX;                    // e_xxz
                const float* xc = xb + 8 * T::WX;                    // e_xxy
                const float* ya = st + T::OY + (ty + R) * 32 + tx;   // e_yyy
                const float* yb = ya + T::HY * 32;                   // e_yyz
                const float* yc = yb + T::HY * 32;                   // e_yxy
                const float* ov = st + T::OV + lo;
                const float* os = st + T::OS + lo;
                float sxx = 0.f, syy = 0.f, szz = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    sxx = sxx + c_fd3e[q - 1] * (xa[1 - q] - xa[q]);
                    syy = syy + c_fd3e[q - 1] * (ya[(1 - q) * 32] - ya[q * 32]);
                    szz = szz + c_fd3e[q - 1] * (qz[R - q] - qz[R - 1 + q]);
                }
                const float xh = ov[0] + a.idx * sxx;
                const float yh = ov[T::T] + a.idy * syy;
                const float zh = ov[2 * T::T] + a.idz * szz;
                float tz1 = 0.f, ty1 = 0.f, tz2 = 0.f, tx2 = 0.f, ty3 = 0.f, tx3 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    tz1 = tz1 + c_fd3e[q - 1] * (qy[R - q] - qy[R + q - 1]);
                    ty1 = ty1 + c_fd3e[q - 1] * (yb[-q * 32] - yb[(q - 1) * 32]);
                    tz2 = tz2 + c_fd3e[q - 1] * (qx[R - q] - qx[R + q - 1]);
                    tx2 = tx2 + c_fd3e[q - 1] * (xb[-q] - xb[q - 1]);
                    ty3 = ty3 + c_fd3e[q - 1] * (yc[-q * 32] - yc[(q - 1) * 32]);
                    tx3 = tx3 + c_fd3e[q - 1] * (xc[-q] - xc[q - 1]);
                }
                const float yzh = ov[3 * T::T] + (a.idz * tz1 + a.idy * ty1);
                const float xzh = ov[4 * T::T] + (a.idz * tz2 + a.idx * tx2);
                const float xyh = ov[5 * T::T] + a.idy * ty3 + a.idx * tx3;
                ad[E3_XX * fs + o] = xh; ad[E3_YY * fs + o] = yh; ad[E3_ZZ * fs + o] = zh;
                ad[E3_YZ * fs + o] = yzh; ad[E3_XZ * fs + o] = xzh; ad[E3_XY * fs + o] = xyh;
                const float dX = os[0], dY = os[T::T], dZ = os[2 * T::T];
                e3_kahan_rw(a.G, a.gg, go, 0, g[0], c[0], xh * dX);
                e3_kahan_rw(a.G, a.gg, go, 1, g[1], c[1], xh * dY + yh * dX);
                e3_kahan_rw(a.G, a.gg, go, 2, g[2], c[2], xh * dZ + zh * dX);
                e3_kahan_rw(a.G, a.gg, go, 3, g[3], c[3], yh * dY);
                e3_kahan_rw(a.G, a.gg, go, 4, g[4], c[4], yh * dZ + zh * dY);
                e3_kahan_rw(a.G, a.gg, go, 5, g[5], c[5], zh * dZ);
                e3_kahan_rw(a.G, a.gg, go, 6, g[6], c[6], yzh * os[3 * T::T]);
                e3_kahan_rw(a.G, a.gg, go, 7, g[7], c[7], xzh * os[4 * T::T]);
                e3_kahan_rw(a.G, a.gg, go, 8, g[8], c[8], xyh * os[5 * T::T]);
                const float* sm = st + T::OM + lo;
                const float c11 = sm[0], c12 = sm[T::T], c13 = sm[2 * T::T], c22 = sm[3 * T::T], c23 = sm[4 * T::T],
                            c33 = sm[5 * T::T];
                float qx_ = a.dt * (c11 * xh + c12 * yh + c13 * zh);
                float qy_ = a.dt * (c12 * xh + c22 * yh + c23 * zh);
                float qz_ = a.dt * (c13 * xh + c23 * yh + c33 * zh);
                if (p0) qx_ = pml_adr(qx_, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 0) : axi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 0) : bxi, m0, mh + N_XVX * fs + o);
                if (p1) qy_ = pml_adr(qy_, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 1) : ayi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 1) : byi, m1, mh + N_YVY * fs + o);
                if (p2) qz_ = pml_adr(qz_, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 2) : azi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 2) : bzi, m2, mh + N_ZVZ * fs + o);
                ew[N_XVX * fs + o] = qx_; ew[N_YVY * fs + o] = qy_; ew[N_ZVZ * fs + o] = qz_;
                float q = a.dt * sm[6 * T::T] * yzh, e1 = q, e2 = q;
                if (p3) e1 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 3) : azh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 3) : bzh, m3, mh + N_ZVY * fs + o);
                if (p4) e2 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 4) : ayh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 4) : byh, m4, mh + N_YVZ * fs + o);
                ew[N_ZVY * fs + o] = e1; ew[N_YVZ * fs + o] = e2;
                q = a.dt * sm[7 * T::T] * xzh; e1 = q; e2 = q;
                if (p5) e1 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 5) : azh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 5) : bzh, m5, mh + N_ZVX * fs + o);
                if (p6) e2 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 6) : axh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 6) : bxh, m6, mh + N_XVZ * fs + o);
                ew[N_ZVX * fs + o] = e1; ew[N_XVZ * fs + o] = e2;
                q = a.dt * sm[8 * T::T] * xyh; e1 = q; e2 = q;
                if (p7) e1 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 7) : ayh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 7) : byh, m7, mh + N_YVX * fs + o);
                if (p8) e2 = pml_adr(q, MP ? e3_ca<E3_PERM_AS>(a, o, 0, 8) : axh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 8) : bxh, m8, mh + N_XVY * fs + o);
                ew[N_YVX * fs + o] = e1; ew[N_XVY * fs + o] = e2;
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) {
                qz[j] = qz[j + 1];
                qy[j] = qy[j + 1];
                qx[j] = qx[j + 1];
            }
            qz[2 * R - 1] = st[T::OA + lo];
            qy[2 * R - 1] = st[T::OA + T::T + lo];
            qx[2 * R - 1] = st[T::OA + 2 * T::T + lo];
        }
        cp_wait<0>();
        __syncthreads();
    }
}
