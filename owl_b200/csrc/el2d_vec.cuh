// el2d_vec.cuh -- the 2D elastic forward stencil kernels with four consecutive
// x cells per thread (included by el2d.cu after the one-cell kernels, inside
// namespace owl; vec4.cuh is included at file scope).
//
// Same arithmetic, per cell and in the same order, as k_el2d_fwd_s /
// k_el2d_fwd_v. A thread owns cells x .. x + 3 of one row (x - x0 a multiple
// of 4): the x arms of its stencils come from one window f[x - R .. x + R + 3]
// per field (win4), the z arms from one float4 per row, its own values,
// moduli and memories from one float4 each, the per-cell M-PML coefficient
// float4s only in the PML. Row conditions (free-surface row, images, which
// stresses exist) are the same for the four cells; the PML tests along x are
// per cell. A memory float4 is written back whole when any of its cells is in
// the PML: the other cells keep the value just read (this launch writes them
// nowhere else). The thread at the right edge may own fewer than four cells
// (n < 4): it stores those one by one.
#pragma once

struct El2dV4 {  // the thread's four cells
    int x, z, n;
    long long o;
};
__device__ __forceinline__ bool el2d_v4(const El2dDev& a, int zr0, El2dV4& c) {
    c.x = a.x0 + 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    c.z = zr0 + blockIdx.y * blockDim.y + threadIdx.y;
    c.n = min(4, a.x1 - c.x);
    c.o = (long long)c.z * a.pitch + c.x;
    return c.x < a.x1 && c.z < a.z1;
}

// (256, 3): 80 registers, three CTAs per SM instead of two (a few bytes
// spilled); ZR as in k_el2d_fwd_s
template <int R, bool STORE, bool ZR>
__global__ void __launch_bounds__(256, 3) k_el2d_fwd_s4(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    El2dV4 c;
    if (!el2d_v4(a, a.zs0, c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const int pt = a.pitch;
    const bool row1 = a.fsurf && z == a.pr;
    const bool dxz = z >= a.zxz0;
    const bool pz_i = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool pz_h = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    // per-cell PML tests; the M-PML coefficients and the moduli are read where
    // they are used (read-only path), which holds fewer registers across the
    // shot loop
    bool px_i[4], pii[4], phh[4];
    bool any_i = false, any_h = false;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        px_i[q] = q < n && el_pml_int(x + q, a.pr, a.nx);
        pii[q] = q < n && (px_i[q] || pz_i);
        phh[q] = q < n && (el_pml_half(x + q, a.pr, a.nx) || pz_h);
        any_i |= (row1 ? px_i[q] : pii[q]);
        any_h |= phh[q];
    }
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
        // the cells' own stresses and memories ahead of their stores (see k_el2d_fwd_s)
        const float4 xx0 = ld4(sxx), zz0 = row1 ? zero : ld4(szz), xz0 = dxz ? ld4(sxzp) : zero;
        float4 mxv = any_i ? ld4(mem + M_DXVX * a.fs) : zero;
        float4 mzv = !row1 && any_i ? ld4(mem + M_DZVZ * a.fs) : zero;
        float4 mxz = dxz && any_h ? ld4(mem + M_DXVZ * a.fs) : zero, mzx = dxz && any_h ? ld4(mem + M_DZVX * a.fs) : zero;
        float w[2 * R + 4];
        win4<R>(vx, w);
        float dxv[4], dzv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float sx = 0.f;
#pragma unroll
            for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (w[R + q + k] - w[R + q + 1 - k]);
            dxv[q] = a.idx * sx;
        }
        if (row1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (px_i[q]) {
                    const float4 ci = __ldg(a.pii + o + q);
                    const float m = ci.x * dxv[q] + ci.y * f4at(mxv, q);
                    f4set(mxv, q, m);
                    dxv[q] = dxv[q] + m;
                }
                dzv[q] = -(__ldg(a.c13 + o + q) / __ldg(a.c33 + o + q) * dxv[q]);
            }
        } else {
            float sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 up = ldg4(vz + k * pt), dn = ldg4(vz + (1 - k) * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fde[k - 1] * (f4at(up, q) - f4at(dn, q));
            }
            const float zsi = ZR ? a.idz * __ldg(a.zfi + z) : a.idz;  // 1/dz times the row's dz scaling
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                dzv[q] = zsi * sz[q];
                if (pii[q]) {
                    const float4 ci = __ldg(a.pii + o + q);
                    const float m1 = ci.x * dxv[q] + ci.y * f4at(mxv, q);
                    f4set(mxv, q, m1);
                    dxv[q] = dxv[q] + m1;
                    const float m2 = ci.z * dzv[q] + ci.w * f4at(mzv, q);
                    f4set(mzv, q, m2);
                    dzv[q] = dzv[q] + m2;
                }
            }
        }
        if (any_i) st4n(mem + M_DXVX * a.fs, mxv, n);
        if (!row1 && any_i) st4n(mem + M_DZVZ * a.fs, mzv, n);
        float4 xxn, zzn;
        const float4 c11 = ldg4(a.c11 + o), c13 = ldg4(a.c13 + o), c33 = ldg4(a.c33 + o);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            f4set(xxn, q, f4at(xx0, q) + a.dt * (f4at(c11, q) * dxv[q] + f4at(c13, q) * dzv[q]));
            f4set(zzn, q, f4at(zz0, q) + a.dt * (f4at(c13, q) * dxv[q] + f4at(c33, q) * dzv[q]));
        }
        st4n(sxx, xxn, n);
        if (row1) {
            st4n(szz, zero, n);
        } else {
            st4n(szz, zzn, n);
            if (mir) st4n(st + EL_SZZ * a.fs + (long long)(2 * a.pr - z) * pt + x,
                          make_float4(-zzn.x, -zzn.y, -zzn.z, -zzn.w), n);
        }
        if (STORE) {
            st4n(a.S + slot + s * a.fs + o, make_float4(dxv[0], dxv[1], dxv[2], dxv[3]), n);
            st4n(a.S + a.sterm + slot + s * a.fs + o, make_float4(dzv[0], dzv[1], dzv[2], dzv[3]), n);
        }
        // sigma_xz
        if (dxz) {
            float sxz[4] = {0.f, 0.f, 0.f, 0.f};
            win4<R>(vz, w);
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int k = 1; k <= R; ++k) sxz[q] = sxz[q] + c_fde[k - 1] * (w[R + q + k - 1] - w[R + q - k]);
            float szx[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 up = ldg4(vx + (k - 1) * pt), dn = ldg4(vx - k * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) szx[q] = szx[q] + c_fde[k - 1] * (f4at(up, q) - f4at(dn, q));
            }
            float4 xzn, gS;
            const float4 c55 = ldg4(a.c55e + o);
            const float zsh = ZR ? a.idz * __ldg(a.zfh + z) : a.idz;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float dzvx = zsh * szx[q], dxvz = a.idx * sxz[q];
                if (phh[q]) {
                    const float4 ch = __ldg(a.phh + o + q);
                    const float m3 = ch.x * dxvz + ch.y * f4at(mxz, q);
                    f4set(mxz, q, m3);
                    dxvz = dxvz + m3;
                    const float m4 = ch.z * dzvx + ch.w * f4at(mzx, q);
                    f4set(mzx, q, m4);
                    dzvx = dzvx + m4;
                }
                const float g = dzvx + dxvz;
                f4set(gS, q, g);
                f4set(xzn, q, f4at(xz0, q) + f4at(c55, q) * a.dt * g);
            }
            if (any_h) {
                st4n(mem + M_DXVZ * a.fs, mxz, n);
                st4n(mem + M_DZVX * a.fs, mzx, n);
            }
            st4n(sxzp, xzn, n);
            if (mir) st4n(st + EL_SXZ * a.fs + (long long)(2 * a.pr + 1 - z) * pt + x,
                          make_float4(-xzn.x, -xzn.y, -xzn.z, -xzn.w), n);
            if (STORE) st4n(a.S + 2 * a.sterm + slot + s * a.fs + o, gS, n);
        }
    }
}

// (256, 4): 64 registers, four CTAs per SM instead of three
template <int R, bool STORE, bool ZR>
__global__ void __launch_bounds__(256, 4) k_el2d_fwd_v4(El2dDev a) {
    pdl_prologue();  // before the first global read (launched with launch_pdl)
    El2dV4 c;
    if (!el2d_v4(a, a.zvx0, c)) return;
    const int x = c.x, z = c.z, n = c.n;
    const long long o = c.o;
    const int pt = a.pitch;
    const bool dvz = z >= a.zvz0;
    const bool pz_hi = (!a.fsurf && z < a.pr) || z >= a.pr + a.nz;
    const bool pz_ih = (!a.fsurf && z <= a.pr) || z >= a.pr + a.nz;
    // per-cell PML tests; the M-PML coefficients and buoyancies are read where
    // they are used (see k_el2d_fwd_s4)
    bool phi[4], pih[4];
    bool any_hi = false, any_ih = false;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        phi[q] = q < n && (el_pml_half(x + q, a.pr, a.nx) || pz_hi);
        pih[q] = q < n && (el_pml_int(x + q, a.pr, a.nx) || pz_ih);
        any_hi |= phi[q];
        any_ih |= pih[q];
    }
    const int s0 = blockIdx.z * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    for (int s = s0; s < s1; ++s) {
        float* st = a.st + s * a.sst;
        const float* sxx = st + EL_SXX * a.fs + o;
        const float* szz = st + EL_SZZ * a.fs + o;
        const float* sxz = st + EL_SXZ * a.fs + o;
        float* mem = st + EL_M0 * a.fs + o;
        // own velocities and memories ahead of the stores (see k_el2d_fwd_s)
        const float4 vx0 = ld4(st + EL_VX * a.fs + o), vz0 = dvz ? ld4(st + EL_VZ * a.fs + o) : zero;
        float4 m_xxx = any_hi ? ld4(mem + M_DXXX * a.fs) : zero, m_zxz = any_hi ? ld4(mem + M_DZXZ * a.fs) : zero;
        float4 m_xxz = dvz && any_ih ? ld4(mem + M_DXXZ * a.fs) : zero;
        float4 m_zzz = dvz && any_ih ? ld4(mem + M_DZZZ * a.fs) : zero;
        float w[2 * R + 4];
        {
            win4<R>(sxx, w);
            float sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 up = ldg4(sxz + k * pt), dn = ldg4(sxz + (1 - k) * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fde[k - 1] * (f4at(up, q) - f4at(dn, q));
            }
            float4 vn, hS;
            const float4 bx = ldg4(a.bx + o);
            const float zsi = ZR ? a.idz * __ldg(a.zfi + z) : a.idz;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float sx = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (w[R + q + k - 1] - w[R + q - k]);
                float hx = a.idx * sx, hz = zsi * sz[q];
                if (phi[q]) {
                    const float4 ch = __ldg(a.phi + o + q);
                    const float m1 = ch.x * hx + ch.y * f4at(m_xxx, q);
                    f4set(m_xxx, q, m1);
                    hx = hx + m1;
                    const float m2 = ch.z * hz + ch.w * f4at(m_zxz, q);
                    f4set(m_zxz, q, m2);
                    hz = hz + m2;
                }
                const float h = hx + hz;
                f4set(vn, q, f4at(vx0, q) + f4at(bx, q) * h);
                f4set(hS, q, h);
            }
            if (any_hi) {
                st4n(mem + M_DXXX * a.fs, m_xxx, n);
                st4n(mem + M_DZXZ * a.fs, m_zxz, n);
            }
            st4n(st + EL_VX * a.fs + o, vn, n);
            if (STORE) st4n(a.S + 3 * a.sterm + slot + s * a.fs + o, hS, n);
        }
        if (dvz) {
            win4<R>(sxz, w);
            float sz[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 1; k <= R; ++k) {
                const float4 up = ldg4(szz + (k - 1) * pt), dn = ldg4(szz - k * pt);
#pragma unroll
                for (int q = 0; q < 4; ++q) sz[q] = sz[q] + c_fde[k - 1] * (f4at(up, q) - f4at(dn, q));
            }
            float4 vn, hS;
            const float4 bz = ldg4(a.bz + o);
            const float zsh = ZR ? a.idz * __ldg(a.zfh + z) : a.idz;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float sx = 0.f;
#pragma unroll
                for (int k = 1; k <= R; ++k) sx = sx + c_fde[k - 1] * (w[R + q + k] - w[R + q + 1 - k]);
                float hx = a.idx * sx, hz = zsh * sz[q];
                if (pih[q]) {
                    const float4 ch = __ldg(a.pih + o + q);
                    const float m1 = ch.x * hx + ch.y * f4at(m_xxz, q);
                    f4set(m_xxz, q, m1);
                    hx = hx + m1;
                    const float m2 = ch.z * hz + ch.w * f4at(m_zzz, q);
                    f4set(m_zzz, q, m2);
                    hz = hz + m2;
                }
                const float h = hx + hz;
                f4set(vn, q, f4at(vz0, q) + f4at(bz, q) * h);
                f4set(hS, q, h);
            }
            if (any_ih) {
                st4n(mem + M_DXXZ * a.fs, m_xxz, n);
                st4n(mem + M_DZZZ * a.fs, m_zzz, n);
            }
            st4n(st + EL_VZ * a.fs + o, vn, n);
            if (STORE) st4n(a.S + 4 * a.sterm + slot + s * a.fs + o, hS, n);
        }
    }
}
