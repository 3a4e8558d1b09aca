// el3d_ring.cuh -- z-marching forward kernels of the 3D elastic solver with an
// asynchronous copy ring (included by el3d.cu inside namespace owl, after
// El3dDev and the stencil helpers). Half-width R, no free surface.
//
// Block 32 x 8 threads, one output per thread and plane; the CTA marches a
// chunk of z planes. Every in-plane operand -- the neighbour tiles with their R
// halo, the cell's own fields and its moduli / buoyancies -- arrives in an
// NS-stage shared-memory ring by 16-byte cp.async copies issued NS-1 planes
// ahead (copy slots computed once per CTA, ring.cuh), right after the plane's
// one barrier. z derivatives come from a register queue of 2R values per field,
// fed from the ring's "ahead" tiles. The CPML memories of a cell are read
// before the ring wait and written back after the update.
// The arithmetic and its order are those of k_el3d_fwd_s / k_el3d_fwd_v.
#pragma once

constexpr int E3R_NS = 4;  // ring stages

template <int R>
struct RingE3S {
    static constexpr int WX = 32 + 2 * R, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // vx, vy, vz with both halos; vx, vy at z + R and vz at z + R + 1 (queue feeds);
    // the six stresses; the nine moduli
    static constexpr int OVX = 0, OVY = HY * WX, OVZ = 2 * HY * WX, OA = 3 * HY * WX, OS = OA + 3 * T,
                         OM = OS + 6 * T, STAGE = OM + 9 * T;
};

template <int R>
struct RingE3V {
    static constexpr int WX = 32 + 2 * R, HY = 8 + 2 * R, CHX = WX / 4, T = 8 * 32;
    // sxx (x halo), syy (y halo), sxy (both), sxz (x halo), syz (y halo);
    // sxz, syz at z + R + 1 and szz at z + R (queue feeds); vx, vy, vz; bx, by, bz
    static constexpr int OXX = 0, OYY = OXX + 8 * WX, OXY = OYY + HY * 32, OXZ = OXY + HY * WX, OYZ = OXZ + 8 * WX,
                         OA = OYZ + HY * 32, OV = OA + 3 * T, OB = OV + 3 * T, STAGE = OB + 3 * T;
};

template <int R>
constexpr int e3r_bytes_s() { return E3R_NS * RingE3S<R>::STAGE * 4; }
template <int R>
constexpr int e3r_bytes_v() { return E3R_NS * RingE3V<R>::STAGE * 4; }

template <int R, bool STORE, bool MP>
__global__ void __launch_bounds__(256, 2) k_el3d_fwd_s_ring(El3dDev a) {
    using T = RingE3S<R>;
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
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    TileSlots<T::HY, T::CHX> sh_;
    TileSlots<8, 8> sc_;
    sh_.init(bx0 - R, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    const int lo = ty * 32 + tx;  // this thread's element of a plain tile
    for (int s = s0; s < s1; ++s) {
        float* stp = a.st + s * a.sst;
        const float* vx = stp + E3_VX * fs;
        const float* vy = stp + E3_VY * fs;
        const float* vz = stp + E3_VZ * fs;
        float* m = stp + E3_M0 * fs;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sh_.copy(st + T::OVX, vx + zo);
            sh_.copy(st + T::OVY, vy + zo);
            sh_.copy(st + T::OVZ, vz + zo);
            const long long za = (long long)min(z + R, a.NZs - 1) * pl, zz = (long long)min(z + R + 1, a.NZs - 1) * pl;
            sc_.copy(st + T::OA, vx + za);
            sc_.copy(st + T::OA + T::T, vy + za);
            sc_.copy(st + T::OA + 2 * T::T, vz + zz);
#pragma unroll
            for (int q = 0; q < 6; ++q) sc_.copy(st + T::OS + q * T::T, stp + q * fs + zo);
            sc_.copy(st + T::OM, a.c11 + zo);
            sc_.copy(st + T::OM + T::T, a.c12 + zo);
            sc_.copy(st + T::OM + 2 * T::T, a.c13 + zo);
            sc_.copy(st + T::OM + 3 * T::T, a.c22 + zo);
            sc_.copy(st + T::OM + 4 * T::T, a.c23 + zo);
            sc_.copy(st + T::OM + 5 * T::T, a.c33 + zo);
            sc_.copy(st + T::OM + 6 * T::T, a.c44e + zo);
            sc_.copy(st + T::OM + 7 * T::T, a.c55e + zo);
            sc_.copy(st + T::OM + 8 * T::T, a.c66e + zo);
        };
        // z queues: qx, qy hold planes z-R .. z+R-1 (M stencils), qz planes z-R+1 .. z+R (P stencil)
        float qx[2 * R], qy[2 * R], qz[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) {
            qx[j] = valid ? vx[(long long)(zb - R + j) * pl + oxy] : 0.f;
            qy[j] = valid ? vy[(long long)(zb - R + j) * pl + oxy] : 0.f;
            qz[j] = valid ? vz[(long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < E3R_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            // the plane's z coefficients and the cell's CPML memories, loaded
            // before the ring wait so that their latency overlaps it
            const long long o = (long long)z * pl + oxy;
            float* mo = m + o;
            const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
            const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
            const bool sh_n = valid && (oxi || oyi || ozi), sh_yz = valid && (oxi || oyh || ozh),
                       sh_xz = valid && (oxh || oyi || ozh), sh_xy = valid && (oxh || oyh || ozi);
            const bool p0 = sh_n && (MP || axi != 0.f), p1 = sh_n && (MP || ayi != 0.f), p2 = sh_n && (MP || azi != 0.f);
            const bool p3 = sh_yz && (MP || ayh != 0.f), p4 = sh_yz && (MP || azh != 0.f);
            const bool p5 = sh_xz && (MP || axh != 0.f), p6 = sh_xz && (MP || azh != 0.f);
            const bool p7 = sh_xy && (MP || axh != 0.f), p8 = sh_xy && (MP || ayh != 0.f);
            const float m0 = p0 ? mo[N_XVX * fs] : 0.f, m1 = p1 ? mo[N_YVY * fs] : 0.f, m2 = p2 ? mo[N_ZVZ * fs] : 0.f;
            const float m3 = p3 ? mo[N_YVZ * fs] : 0.f, m4 = p4 ? mo[N_ZVY * fs] : 0.f;
            const float m5 = p5 ? mo[N_XVZ * fs] : 0.f, m6 = p6 ? mo[N_ZVX * fs] : 0.f;
            const float m7 = p7 ? mo[N_XVY * fs] : 0.f, m8 = p8 ? mo[N_YVX * fs] : 0.f;
            // plane z's group is complete once at most NS-2 later groups are pending; the
            // barrier also retires every read of the stage refilled next (plane z-1's)
            cp_wait<E3R_NS - 2>();
            __syncthreads();
            if (z + E3R_NS - 1 < ze) issue(z + E3R_NS - 1, (i + E3R_NS - 1) % E3R_NS);
            cp_commit();
            const float* st = ring + (i % E3R_NS) * T::STAGE;
            if (valid) {
                const float* tvx = st + T::OVX + (ty + R) * T::WX + tx + R;
                const float* tvy = st + T::OVY + (ty + R) * T::WX + tx + R;
                const float* tvz = st + T::OVZ + (ty + R) * T::WX + tx + R;
                const float* sm = st + T::OM + lo;
                const float c11 = sm[0], c12 = sm[T::T], c13 = sm[2 * T::T], c22 = sm[3 * T::T], c23 = sm[4 * T::T],
                            c33 = sm[5 * T::T];
                const float g44 = a.dt * sm[6 * T::T], g55 = a.dt * sm[7 * T::T], g66 = a.dt * sm[8 * T::T];
                float sX = 0.f, sY = 0.f, sZ = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    sX = sX + c_fd3e[q - 1] * (tvx[q] - tvx[1 - q]);
                    sY = sY + c_fd3e[q - 1] * (tvy[q * T::WX] - tvy[(1 - q) * T::WX]);
                    sZ = sZ + c_fd3e[q - 1] * (qz[R - 1 + q] - qz[R - q]);
                }
                float dX = a.idx * sX, dY = a.idy * sY, dZ = a.idz * sZ;
                if (p0) dX = pml_up(dX, MP ? e3_ca<E3_PERM_S>(a, o, 0, 0) : axi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 0) : bxi, m0, mo + N_XVX * fs);
                if (p1) dY = pml_up(dY, MP ? e3_ca<E3_PERM_S>(a, o, 0, 1) : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 1) : byi, m1, mo + N_YVY * fs);
                if (p2) dZ = pml_up(dZ, MP ? e3_ca<E3_PERM_S>(a, o, 0, 2) : azi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 2) : bzi, m2, mo + N_ZVZ * fs);
                const float* so = st + T::OS + lo;
                stp[E3_XX * fs + o] = so[0] + a.dt * (c11 * dX + c12 * dY + c13 * dZ);
                stp[E3_YY * fs + o] = so[T::T] + a.dt * (c12 * dX + c22 * dY + c23 * dZ);
                stp[E3_ZZ * fs + o] = so[2 * T::T] + a.dt * (c13 * dX + c23 * dY + c33 * dZ);
                // syz: dz vy + dy vz
                float a1 = 0.f, a2 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    a1 = a1 + c_fd3e[q - 1] * (qy[R + q - 1] - qy[R - q]);
                    a2 = a2 + c_fd3e[q - 1] * (tvz[(q - 1) * T::WX] - tvz[-q * T::WX]);
                }
                float dzvy = a.idz * a1, dyvz = a.idy * a2;
                if (p3) dyvz = pml_up(dyvz, MP ? e3_ca<E3_PERM_S>(a, o, 0, 3) : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 3) : byh, m3, mo + N_YVZ * fs);
                if (p4) dzvy = pml_up(dzvy, MP ? e3_ca<E3_PERM_S>(a, o, 0, 4) : azh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 4) : bzh, m4, mo + N_ZVY * fs);
                stp[E3_YZ * fs + o] = so[3 * T::T] + g44 * (dzvy + dyvz);
                // sxz: dz vx + dx vz
                a1 = 0.f; a2 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    a1 = a1 + c_fd3e[q - 1] * (qx[R + q - 1] - qx[R - q]);
                    a2 = a2 + c_fd3e[q - 1] * (tvz[q - 1] - tvz[-q]);
                }
                float dzvx = a.idz * a1, dxvz = a.idx * a2;
                if (p5) dxvz = pml_up(dxvz, MP ? e3_ca<E3_PERM_S>(a, o, 0, 5) : axh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 5) : bxh, m5, mo + N_XVZ * fs);
                if (p6) dzvx = pml_up(dzvx, MP ? e3_ca<E3_PERM_S>(a, o, 0, 6) : azh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 6) : bzh, m6, mo + N_ZVX * fs);
                stp[E3_XZ * fs + o] = so[4 * T::T] + g55 * (dzvx + dxvz);
                // sxy: dy vx + dx vy
                a1 = 0.f; a2 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    a1 = a1 + c_fd3e[q - 1] * (tvx[(q - 1) * T::WX] - tvx[-q * T::WX]);
                    a2 = a2 + c_fd3e[q - 1] * (tvy[q - 1] - tvy[-q]);
                }
                float dyvx = a.idy * a1, dxvy = a.idx * a2;
                if (p7) dxvy = pml_up(dxvy, MP ? e3_ca<E3_PERM_S>(a, o, 0, 7) : axh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 7) : bxh, m7, mo + N_XVY * fs);
                if (p8) dyvx = pml_up(dyvx, MP ? e3_ca<E3_PERM_S>(a, o, 0, 8) : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 8) : byh, m8, mo + N_YVX * fs);
                stp[E3_XY * fs + o] = so[5 * T::T] + g66 * (dyvx + dxvy);
                if (STORE) {
                    float* S = a.S + slot + s * fs + o;
                    S[0] = dX; S[a.sterm] = dY; S[2 * a.sterm] = dZ;
                    S[3 * a.sterm] = dzvy + dyvz; S[4 * a.sterm] = dzvx + dxvz; S[5 * a.sterm] = dyvx + dxvy;
                }
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

template <int R, bool STORE, bool MP>
__global__ void __launch_bounds__(256, 2) k_el3d_fwd_v_ring(El3dDev a) {
    using T = RingE3V<R>;
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
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    const int s0 = grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    TileSlots<8, T::CHX> sx_;
    TileSlots<T::HY, 8> sy_;
    TileSlots<T::HY, T::CHX> sxy_;
    TileSlots<8, 8> sc_;
    sx_.init(bx0 - R, by0, a.pitch, a.NYs);
    sy_.init(bx0, by0 - R, a.pitch, a.NYs);
    sxy_.init(bx0 - R, by0 - R, a.pitch, a.NYs);
    sc_.init(bx0, by0, a.pitch, a.NYs);
    const int lo = ty * 32 + tx;
    for (int s = s0; s < s1; ++s) {
        float* stp = a.st + s * a.sst;
        const float* sxx = stp + E3_XX * fs;
        const float* syy = stp + E3_YY * fs;
        const float* szz = stp + E3_ZZ * fs;
        const float* syz = stp + E3_YZ * fs;
        const float* sxz = stp + E3_XZ * fs;
        const float* sxy = stp + E3_XY * fs;
        float* m = stp + E3_M0 * fs;
        auto issue = [&](int z, int stage) {
            float* st = ring + stage * T::STAGE;
            const long long zo = (long long)z * pl;
            sx_.copy(st + T::OXX, sxx + zo);
            sy_.copy(st + T::OYY, syy + zo);
            sxy_.copy(st + T::OXY, sxy + zo);
            sx_.copy(st + T::OXZ, sxz + zo);
            sy_.copy(st + T::OYZ, syz + zo);
            const long long za = (long long)min(z + R, a.NZs - 1) * pl, zz = (long long)min(z + R + 1, a.NZs - 1) * pl;
            sc_.copy(st + T::OA, sxz + zz);
            sc_.copy(st + T::OA + T::T, syz + zz);
            sc_.copy(st + T::OA + 2 * T::T, szz + za);
#pragma unroll
            for (int q = 0; q < 3; ++q) sc_.copy(st + T::OV + q * T::T, stp + (E3_VX + q) * fs + zo);
            sc_.copy(st + T::OB, a.bx + zo);
            sc_.copy(st + T::OB + T::T, a.by + zo);
            sc_.copy(st + T::OB + 2 * T::T, a.bz + zo);
        };
        // z queues: sxz, syz planes z-R+1 .. z+R (P stencils), szz planes z-R .. z+R-1 (M stencil)
        float qxz[2 * R], qyz[2 * R], qzz[2 * R];
#pragma unroll
        for (int j = 0; j < 2 * R; ++j) {
            qxz[j] = valid ? sxz[(long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
            qyz[j] = valid ? syz[(long long)(zb - R + 1 + j) * pl + oxy] : 0.f;
            qzz[j] = valid ? szz[(long long)(zb - R + j) * pl + oxy] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < E3R_NS - 1; ++j) {
            if (zb + j < ze) issue(zb + j, j);
            cp_commit();
        }
        for (int z = zb, i = 0; z < ze; ++z, ++i) {
            // the plane's z coefficients and the cell's CPML memories, loaded
            // before the ring wait so that their latency overlaps it
            const long long o = (long long)z * pl + oxy;
            float* mo = m + o;
            const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
            const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
            const bool sh_vx = valid && (oxh || oyi || ozi), sh_vy = valid && (oxi || oyh || ozi),
                       sh_vz = valid && (oxi || oyi || ozh);
            const bool p0 = sh_vx && (MP || axh != 0.f), p1 = sh_vx && (MP || ayi != 0.f), p2 = sh_vx && (MP || azi != 0.f);
            const bool p3 = sh_vy && (MP || axi != 0.f), p4 = sh_vy && (MP || ayh != 0.f), p5 = sh_vy && (MP || azi != 0.f);
            const bool p6 = sh_vz && (MP || axi != 0.f), p7 = sh_vz && (MP || ayi != 0.f), p8 = sh_vz && (MP || azh != 0.f);
            const float m0 = p0 ? mo[N_XXX * fs] : 0.f, m1 = p1 ? mo[N_YXY * fs] : 0.f, m2 = p2 ? mo[N_ZXZ * fs] : 0.f;
            const float m3 = p3 ? mo[N_XXY * fs] : 0.f, m4 = p4 ? mo[N_YYY * fs] : 0.f, m5 = p5 ? mo[N_ZYZ * fs] : 0.f;
            const float m6 = p6 ? mo[N_XXZ * fs] : 0.f, m7 = p7 ? mo[N_YYZ * fs] : 0.f, m8 = p8 ? mo[N_ZZZ * fs] : 0.f;
            cp_wait<E3R_NS - 2>();
            __syncthreads();
            if (z + E3R_NS - 1 < ze) issue(z + E3R_NS - 1, (i + E3R_NS - 1) % E3R_NS);
            cp_commit();
            const float* st = ring + (i % E3R_NS) * T::STAGE;
            if (valid) {
                const float* txx = st + T::OXX + ty * T::WX + tx + R;
                const float* tyy = st + T::OYY + (ty + R) * 32 + tx;
                const float* txy = st + T::OXY + (ty + R) * T::WX + tx + R;
                const float* txz = st + T::OXZ + ty * T::WX + tx + R;
                const float* tyz = st + T::OYZ + (ty + R) * 32 + tx;
                // vx: dx sxx (M) + dy sxy (P) + dz sxz (P)
                float h1 = 0.f, h2 = 0.f, h3 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    h1 = h1 + c_fd3e[q - 1] * (txx[q - 1] - txx[-q]);
                    h2 = h2 + c_fd3e[q - 1] * (txy[q * T::WX] - txy[(1 - q) * T::WX]);
                    h3 = h3 + c_fd3e[q - 1] * (qxz[R - 1 + q] - qxz[R - q]);
                }
                h1 = a.idx * h1; h2 = a.idy * h2; h3 = a.idz * h3;
                if (p0) h1 = pml_up(h1, MP ? e3_ca<E3_PERM_S>(a, o, 9, 0) : axh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 0) : bxh, m0, mo + N_XXX * fs);
                if (p1) h2 = pml_up(h2, MP ? e3_ca<E3_PERM_S>(a, o, 9, 1) : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 1) : byi, m1, mo + N_YXY * fs);
                if (p2) h3 = pml_up(h3, MP ? e3_ca<E3_PERM_S>(a, o, 9, 2) : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 2) : bzi, m2, mo + N_ZXZ * fs);
                const float hx = h1 + h2 + h3;
                stp[E3_VX * fs + o] = st[T::OV + lo] + st[T::OB + lo] * hx;
                // vy: dx sxy (P) + dy syy (M) + dz syz (P)
                h1 = 0.f; h2 = 0.f; h3 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    h1 = h1 + c_fd3e[q - 1] * (txy[q] - txy[1 - q]);
                    h2 = h2 + c_fd3e[q - 1] * (tyy[(q - 1) * 32] - tyy[-q * 32]);
                    h3 = h3 + c_fd3e[q - 1] * (qyz[R - 1 + q] - qyz[R - q]);
                }
                h1 = a.idx * h1; h2 = a.idy * h2; h3 = a.idz * h3;
                if (p3) h1 = pml_up(h1, MP ? e3_ca<E3_PERM_S>(a, o, 9, 3) : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 3) : bxi, m3, mo + N_XXY * fs);
                if (p4) h2 = pml_up(h2, MP ? e3_ca<E3_PERM_S>(a, o, 9, 4) : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 4) : byh, m4, mo + N_YYY * fs);
                if (p5) h3 = pml_up(h3, MP ? e3_ca<E3_PERM_S>(a, o, 9, 5) : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 5) : bzi, m5, mo + N_ZYZ * fs);
                const float hy = h1 + h2 + h3;
                stp[E3_VY * fs + o] = st[T::OV + T::T + lo] + st[T::OB + T::T + lo] * hy;
                // vz: dx sxz (P) + dy syz (P) + dz szz (M)
                h1 = 0.f; h2 = 0.f; h3 = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    h1 = h1 + c_fd3e[q - 1] * (txz[q] - txz[1 - q]);
                    h2 = h2 + c_fd3e[q - 1] * (tyz[q * 32] - tyz[(1 - q) * 32]);
                    h3 = h3 + c_fd3e[q - 1] * (qzz[R + q - 1] - qzz[R - q]);
                }
                h1 = a.idx * h1; h2 = a.idy * h2; h3 = a.idz * h3;
                if (p6) h1 = pml_up(h1, MP ? e3_ca<E3_PERM_S>(a, o, 9, 6) : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 6) : bxi, m6, mo + N_XXZ * fs);
                if (p7) h2 = pml_up(h2, MP ? e3_ca<E3_PERM_S>(a, o, 9, 7) : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 7) : byi, m7, mo + N_YYZ * fs);
                if (p8) h3 = pml_up(h3, MP ? e3_ca<E3_PERM_S>(a, o, 9, 8) : azh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 8) : bzh, m8, mo + N_ZZZ * fs);
                const float hz = h1 + h2 + h3;
                stp[E3_VZ * fs + o] = st[T::OV + 2 * T::T + lo] + st[T::OB + 2 * T::T + lo] * hz;
                if (STORE) {
                    float* S = a.S + slot + s * fs + o;
                    S[6 * a.sterm] = hx; S[7 * a.sterm] = hy; S[8 * a.sterm] = hz;
                }
            }
#pragma unroll
            for (int j = 0; j < 2 * R - 1; ++j) {
                qxz[j] = qxz[j + 1];
                qyz[j] = qyz[j + 1];
                qzz[j] = qzz[j + 1];
            }
            qxz[2 * R - 1] = st[T::OA + lo];
            qyz[2 * R - 1] = st[T::OA + T::T + lo];
            qzz[2 * R - 1] = st[T::OA + 2 * T::T + lo];
        }
        cp_wait<0>();
        __syncthreads();
    }
}
