// el3d.cu -- 3D elastic (isotropic / orthorhombic) SSG solver for B200 (sm_100a).
//
// Forward (replaces update_wavefield, add_source and the sampling of
// compute_forward, src/solver/elastic_vhtiort_3d/module_wavefield.f90:52-537,
// :1095-1333 and submodule_forward_modeling.f90:82-145) without a free surface,
// with or without a flat free surface on the uniform grid
// (update_wavefield_free_surface, module_wavefield.f90:549-1090: zero velocities
// above the surface, the traction condition pdzvz = -c13/c33 pdxvx - c23/c33
// pdyvy at row 1, sigma_zz(1) = 0 and odd images of sigma_zz, sigma_yz,
// sigma_xz; the images of sigma_xx, sigma_yy, sigma_xy are never read and are
// not stored), and the exact discrete adjoint with every-k-step checkpoints, Kahan FP32
// correlations for the nine Cij and the three buoyancies, and the FP64 chain
// rule to the model parameters (replaces compute_adjoint / compute_gradient,
// submodule_fwi_gradient.f90).
//
// Nodes (storage index = reference index + pml + R - 1 on each axis):
// normal stresses at (i, j, k); syz at (i, j-1/2, k-1/2); sxz at (i-1/2, j,
// k-1/2); sxy at (i-1/2, j-1/2, k); vx at (i-1/2, j, k); vy at (i, j-1/2, k);
// vz at (i, j, k-1/2). State per shot: 9 fields + 18 CFS-MPML memory volumes.
// With a free surface, the integer-depth nodes are updated from row 1 and the
// half-depth ones (syz, sxz, vz) from row 2; velocity taps of the receivers on
// the surface images (vx, vy (1-k) = (1+k), vz (2-k) = (1+k), k <= 4) are
// mapped onto the rows they copy.
//
// Damping. The reference damps a derivative along axis a of a node in the PML
// shell with d = d_a(pos_a) + sum of ratio_b * d_b(pos_b) over the other axes b
// (module_wavefield.f90:104-145), ratio_b the M-PML ratio of the face of axis b
// the node lies beyond (0 between them) and alpha_a the axis-a profile inside
// its PML, alphamax elsewhere in the shell. With the ratios at zero -- the
// reference's value for the iso parameterisation -- (a, b) of a derivative
// depend only on the node's position along that axis: 1D tables per axis
// (integer and half positions), and a memory whose a is 0 stays exactly 0 and is
// not touched. Anisotropic parameterisations have nonzero ratios (searched on
// the host, mpml.cu): the MP instances of the per-cell kernels compute each
// shell node's (a, b) from the per-axis profiles and the six face-ratio arrays.
//
// One step = two stencil launches (stresses, velocities) + the point kernel;
// the adjoint of a step = velocity-node kernel, source adjoint (optional),
// stress-node kernel, residual injection (the e-array scheme of the 2D solvers:
// each node stores the adjoint PML terms of its own derivatives).
#include <algorithm>
#include <cmath>

#include "mpml.cuh"
#include "ring.cuh"
#include "ssg_base.cuh"
#include "vmesh.hpp"

namespace owl {

__constant__ float c_fd3e[8];

enum { E3_XX = 0, E3_YY, E3_ZZ, E3_YZ, E3_XZ, E3_XY, E3_VX, E3_VY, E3_VZ, E3_M0 };
// memories (and adjoint PML terms) in the order of the forward derivatives
enum { N_XVX = 0, N_YVY, N_ZVZ, N_ZVY, N_YVZ, N_ZVX, N_XVZ, N_YVX, N_XVY, N_XXX, N_YXY, N_ZXZ, N_XXY, N_YYY, N_ZYZ,
       N_XXZ, N_YYZ, N_ZZZ };
constexpr int E3_NST = 9 + 18;
constexpr int E3_NAD = 9 + 18 + 18;

// M-PML tables: per axis the damping profile d and alpha at integer [0] and
// half [1] positions (storage index; d = 0 and alpha = alphamax outside the
// axis' PML), and the face ratios: left / right [z][y] (NYs), front / back
// [z][x], top / bottom [y][x] (pitch), zero outside the padded model
struct E3Mp {
    const float* d[3][2];
    const float* al[3][2];
    const float* face[6];
    float adt;
    // (a, b) of every derivative of every node, computed once per model by
    // k_el3d_mpml_coef: entry q's pair is float2 number q fs + o; q 0..8 the
    // stress nodes' derivatives, q 9..17 the velocity nodes'
    const float* coef;
};

struct El3dDev {
    int nx, ny, nz, P, R, pr, pitch;
    long long plane, fs, sst, sad;
    int x0, x1, y0, y1, z0, z1, nzb, fsurf;
    int NYs, NZs, zchunk;  // storage planes / rows, z chunk of the ring kernels
    float idx, idy, idz, dt;
    int nshots, spt;
    const float *c11, *c12, *c13, *c22, *c23, *c33, *c44e, *c55e, *c66e, *bx, *by, *bz;
    // per axis: a and b at integer and half positions (storage index)
    const float *axi, *bxi, *axh, *bxh, *ayi, *byi, *ayh, *byh, *azi, *bzi, *azh, *bzh;
    // per storage plane: dz / dz_i and dz / dz_h of the depth-refined free-surface
    // mesh, the factors of the z derivatives at integer-z nodes (normal stresses,
    // sxy, vx, vy) and half-z nodes (syz, sxz, vz); 1 on the uniform grid. Read
    // by the per-cell kernels (the ring kernels run without a free surface).
    const float *zfi, *zfh;
    float* st;
    float* S;
    long long sslot, sterm;
    int k;
    int* d_step;
    float* ad;
    float* G;  // [12][group][fs] sums then [12][group][fs] compensations
    long long gg;
    E3Mp mp;
};

__device__ __forceinline__ bool e3_out(int v, int pr, int n, bool half) {
    return half ? (v <= pr || v >= pr + n) : (v < pr || v >= pr + n);
}

template <int R>
__device__ __forceinline__ float stP(const float* f, long long s) {
    float a = 0.f;
#pragma unroll
    for (int q = 1; q <= R; ++q) a = a + c_fd3e[q - 1] * (__ldg(f + q * s) - __ldg(f + (1 - q) * s));
    return a;
}
template <int R>
__device__ __forceinline__ float stM(const float* f, long long s) {
    float a = 0.f;
#pragma unroll
    for (int q = 1; q <= R; ++q) a = a + c_fd3e[q - 1] * (__ldg(f + (q - 1) * s) - __ldg(f - q * s));
    return a;
}
// transposes of P and M, read at the node
template <int R>
__device__ __forceinline__ float tP(const float* e, long long s) {
    float a = 0.f;
#pragma unroll
    for (int q = 1; q <= R; ++q) a = a + c_fd3e[q - 1] * (__ldg(e - q * s) - __ldg(e + (q - 1) * s));
    return a;
}
template <int R>
__device__ __forceinline__ float tM(const float* e, long long s) {
    float a = 0.f;
#pragma unroll
    for (int q = 1; q <= R; ++q) a = a + c_fd3e[q - 1] * (__ldg(e + (1 - q) * s) - __ldg(e + q * s));
    return a;
}

// CPML step with the memory value read ahead: psi' = a D + b psi, D + psi'
__device__ __forceinline__ float pml_up(float D, float a, float b, float psi, float* dst) {
    const float m = a * D + b * psi;
    *dst = m;
    return D + m;
}
// adjoint CPML step with the memory value read ahead: u = q + psih, psih' = b u, q + a u
__device__ __forceinline__ float pml_adr(float q, float a, float b, float psih, float* dst) {
    const float u = q + psih;
    *dst = b * u;
    return q + a * u;
}

// (a, b) of the derivative along axis ax at the node at storage (x, y, z),
// staggered by (hx, hy, hz) (1: half position on that axis): d = own profile +
// ratio * profile of each other axis in the reference's order, alpha of the own
// axis, kappa = 1, damp_coef of module_wavefield.f90:40-43 (the M-PML blocks of
// module_wavefield.f90:101-145 and their counterparts for the other nodes)
__device__ __forceinline__ void e3_mpml(const El3dDev& a, int ax, int x, int y, int z, int hx, int hy, int hz,
                                        float& ca, float& cb) {
    const E3Mp& m = a.mp;
    // beyond a face: reference index <= 0 (integer position) or <= 1 (half
    // position), or >= n + 1 -- the node's own shell test on that axis
    const int lo = a.pr;
    const float rx = x < lo + hx ? __ldg(m.face[0] + z * a.NYs + y)
                   : x >= lo + a.nx ? __ldg(m.face[1] + z * a.NYs + y) : 0.f;
    const float ry = y < lo + hy ? __ldg(m.face[2] + z * a.pitch + x)
                   : y >= lo + a.ny ? __ldg(m.face[3] + z * a.pitch + x) : 0.f;
    const float rz = z < lo + hz ? __ldg(m.face[4] + y * a.pitch + x)
                   : z >= lo + a.nz ? __ldg(m.face[5] + y * a.pitch + x) : 0.f;
    const float dX = __ldg(m.d[0][hx] + x), dY = __ldg(m.d[1][hy] + y), dZ = __ldg(m.d[2][hz] + z);
    float d, al;
    if (ax == 0) { d = dX + ry * dY + rz * dZ; al = __ldg(m.al[0][hx] + x); }
    else if (ax == 1) { d = dY + rx * dX + rz * dZ; al = __ldg(m.al[1][hy] + y); }
    else { d = dZ + rx * dX + ry * dY; al = __ldg(m.al[2][hz] + z); }
    const float b = d + al;
    ca = -2.0f * m.adt * d / (2.0f + m.adt * b);
    cb = (2.0f - m.adt * b) / (2.0f + m.adt * b);
}

// the derivatives of the precomputed table, in the order of k_el3d_mpml_coef:
// (axis, hx, hy, hz) of q = 0..8 (stress nodes) and 9..17 (velocity nodes)
__constant__ int c_e3_coef_node[18][4] = {
    {0, 0, 0, 0}, {1, 0, 0, 0}, {2, 0, 0, 0}, {1, 0, 1, 1}, {2, 0, 1, 1}, {0, 1, 0, 1}, {2, 1, 0, 1}, {0, 1, 1, 0},
    {1, 1, 1, 0}, {0, 1, 0, 0}, {1, 1, 0, 0}, {2, 1, 0, 0}, {0, 0, 1, 0}, {1, 0, 1, 0}, {2, 0, 1, 0}, {0, 0, 0, 1},
    {1, 0, 0, 1}, {2, 0, 0, 1}};
// the order in which a kernel wants entries q0 + 0..8: the forward stress and
// both velocity kernels take them as stored, the adjoint stress kernel swaps
// the two derivatives of each shear node
constexpr int E3_PERM_S = 0, E3_PERM_AS = 1;
template <int PERM>
__device__ __forceinline__ int e3_perm(int q) {
    return PERM == E3_PERM_S ? q : (q < 3 ? q : (q & 1 ? q + 1 : q - 1));
}
// the a of the node's nine derivatives (they decide which memories update);
// each b is loaded where its update needs it (e3_cb), to hold fewer registers
template <int PERM>
__device__ __forceinline__ float2 e3_ab(const El3dDev& a, long long o, int q0, int q) {
    return __ldg(reinterpret_cast<const float2*>(a.mp.coef) + (q0 + e3_perm<PERM>(q)) * a.fs + o);
}
template <int PERM>
__device__ __forceinline__ void e3_coef_load(const El3dDev& a, long long o, int q0, float (&ca)[9]) {
#pragma unroll
    for (int q = 0; q < 9; ++q) ca[q] = e3_ab<PERM>(a, o, q0, q).x;
}
// a and b of one entry: one 8-byte load where both are used together
template <int PERM>
__device__ __forceinline__ float e3_ca(const El3dDev& a, long long o, int q0, int q) {
    return e3_ab<PERM>(a, o, q0, q).x;
}
template <int PERM>
__device__ __forceinline__ float e3_cb(const El3dDev& a, long long o, int q0, int q) {
    return e3_ab<PERM>(a, o, q0, q).y;
}

// one thread per updated cell: the (a, b) of its 18 derivatives (e3_mpml, the
// same arithmetic the kernels used to repeat every step)
__global__ void k_el3d_mpml_coef(El3dDev a, float* __restrict__ out) {
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = a.y0 + blockIdx.y * blockDim.y + threadIdx.y;
    const int z = a.z0 + blockIdx.z;
    if (x >= a.x1 || y >= a.y1 || z >= a.z1) return;
    const long long o = (long long)z * a.plane + (long long)y * a.pitch + x;
    for (int q = 0; q < 18; ++q) {
        float ca, cb;
        e3_mpml(a, c_e3_coef_node[q][0], x, y, z, c_e3_coef_node[q][1], c_e3_coef_node[q][2], c_e3_coef_node[q][3],
                ca, cb);
        reinterpret_cast<float2*>(out)[q * a.fs + o] = make_float2(ca, cb);
    }
}

struct E3Cell {
    int x, y, z, grp;
    long long o;
};
__device__ __forceinline__ bool e3_cell(const El3dDev& a, E3Cell& c) {
    const int zb = blockIdx.z % a.nzb;
    c.grp = blockIdx.z / a.nzb;
    c.x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x;
    c.y = a.y0 + blockIdx.y * blockDim.y + threadIdx.y;
    c.z = a.z0 + zb * blockDim.z + threadIdx.z;
    c.o = (long long)c.z * a.plane + (long long)c.y * a.pitch + c.x;
    return c.x < a.x1 && c.y < a.y1 && c.z < a.z1;
}

#include "el3d_ring.cuh"

// ------------------------------- forward ------------------------------------
template <int R, bool STORE, bool FS, bool MP>
__global__ void __launch_bounds__(256, MP ? 2 : 3) k_el3d_fwd_s(El3dDev a) {
    E3Cell c;
    if (!e3_cell(a, c)) return;
    const long long o = c.o, sy = a.pitch, sz = a.plane;
    const int x = c.x, y = c.y, z = c.z;
    // PML shell of each node type and the 1D coefficients it needs
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
    const bool sh_n = oxi || oyi || ozi, sh_yz = oxi || oyh || ozh, sh_xz = oxh || oyi || ozh, sh_xy = oxh || oyh || ozi;
    const float axi = a.axi[x], bxi = a.bxi[x], axh = a.axh[x], bxh = a.bxh[x];
    const float ayi = a.ayi[y], byi = a.byi[y], ayh = a.ayh[y], byh = a.byh[y];
    const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
    const float c11 = __ldg(a.c11 + o), c12 = __ldg(a.c12 + o), c13 = __ldg(a.c13 + o), c22 = __ldg(a.c22 + o),
                c23 = __ldg(a.c23 + o), c33 = __ldg(a.c33 + o);
    const float g44 = a.dt * __ldg(a.c44e + o), g55 = a.dt * __ldg(a.c55e + o), g66 = a.dt * __ldg(a.c66e + o);
    // 1/dz times the plane's dz scaling (the refined mesh exists only under a
    // free surface: the FS instances read the factors, exactly 1 on the uniform grid)
    const float zsi = FS ? a.idz * __ldg(a.zfi + z) : a.idz, zsh = FS ? a.idz * __ldg(a.zfh + z) : a.idz;
    const int s0 = c.grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    // free surface: row 1, whether the half-depth stresses exist at this row,
    // and the image rows of sigma_zz (2 pr - z) and of syz / sxz (2 pr + 1 - z)
    const bool row1 = FS && z == a.pr, hz_ok = !FS || z > a.pr;
    const bool mir = FS && z > a.pr && z <= a.pr + a.R;
    const long long dzz = (long long)(2 * a.pr - 2 * z) * sz, dsh = dzz + sz;
    // MP: the M-PML (a, b) of each derivative of the node (shell nodes only);
    // otherwise the per-axis 1D tables above
    float ca[9];
    if (MP) {
        if (row1 || sh_n || sh_yz || sh_xz || sh_xy) {
            e3_coef_load<E3_PERM_S>(a, o, 0, ca);
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) ca[q] = 0.f;
        }
    }
    for (int s = s0; s < s1; ++s) {
        float* st = a.st + s * a.sst;
        const float* vx = st + E3_VX * a.fs + o;
        const float* vy = st + E3_VY * a.fs + o;
        const float* vz = st + E3_VZ * a.fs + o;
        float* m = st + E3_M0 * a.fs + o;
        // the cell's old stresses and CPML memories are read ahead of its first
        // store (same buffer: no later plain read could move above a store)
        const float xx0 = st[E3_XX * a.fs + o], yy0 = st[E3_YY * a.fs + o];
        const float zz0 = row1 ? 0.f : st[E3_ZZ * a.fs + o];
        const float yz0 = hz_ok ? st[E3_YZ * a.fs + o] : 0.f, xz0 = hz_ok ? st[E3_XZ * a.fs + o] : 0.f;
        const float xy0 = st[E3_XY * a.fs + o];
        const bool p0 = (row1 || sh_n) && (MP ? ca[0] : axi) != 0.f, p1 = (row1 || sh_n) && (MP ? ca[1] : ayi) != 0.f, p2 = !row1 && sh_n && (MP ? ca[2] : azi) != 0.f;
        const bool p3 = hz_ok && sh_yz && (MP ? ca[3] : ayh) != 0.f, p4 = hz_ok && sh_yz && (MP ? ca[4] : azh) != 0.f;
        const bool p5 = hz_ok && sh_xz && (MP ? ca[5] : axh) != 0.f, p6 = hz_ok && sh_xz && (MP ? ca[6] : azh) != 0.f;
        const bool p7 = sh_xy && (MP ? ca[7] : axh) != 0.f, p8 = sh_xy && (MP ? ca[8] : ayh) != 0.f;
        const float m0 = p0 ? m[N_XVX * a.fs] : 0.f, m1 = p1 ? m[N_YVY * a.fs] : 0.f, m2 = p2 ? m[N_ZVZ * a.fs] : 0.f;
        const float m3 = p3 ? m[N_YVZ * a.fs] : 0.f, m4 = p4 ? m[N_ZVY * a.fs] : 0.f;
        const float m5 = p5 ? m[N_XVZ * a.fs] : 0.f, m6 = p6 ? m[N_ZVX * a.fs] : 0.f;
        const float m7 = p7 ? m[N_XVY * a.fs] : 0.f, m8 = p8 ? m[N_YVX * a.fs] : 0.f;
        float dX = a.idx * stP<R>(vx, 1), dY = a.idy * stP<R>(vy, sy), dZ;
        if (p0) dX = pml_up(dX, MP ? ca[0] : axi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 0) : bxi, m0, m + N_XVX * a.fs);
        if (p1) dY = pml_up(dY, MP ? ca[1] : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 1) : byi, m1, m + N_YVY * a.fs);
        if (row1) {
            dZ = -(c13 / c33) * dX - (c23 / c33) * dY;
        } else {
            dZ = zsi * stP<R>(vz, sz);
            if (p2) dZ = pml_up(dZ, MP ? ca[2] : azi, MP ? e3_cb<E3_PERM_S>(a, o, 0, 2) : bzi, m2, m + N_ZVZ * a.fs);
        }
        st[E3_XX * a.fs + o] = xx0 + a.dt * (c11 * dX + c12 * dY + c13 * dZ);
        st[E3_YY * a.fs + o] = yy0 + a.dt * (c12 * dX + c22 * dY + c23 * dZ);
        if (row1) {
            st[E3_ZZ * a.fs + o] = 0.f;
        } else {
            const float zn = zz0 + a.dt * (c13 * dX + c23 * dY + c33 * dZ);
            st[E3_ZZ * a.fs + o] = zn;
            if (mir) st[E3_ZZ * a.fs + o + dzz] = -zn;
        }
        float dzvy = 0.f, dyvz = 0.f, dzvx = 0.f, dxvz = 0.f;
        if (hz_ok) {
            // syz: dz vy + dy vz
            dzvy = zsh * stM<R>(vy, sz);
            dyvz = a.idy * stM<R>(vz, sy);
            if (p3) dyvz = pml_up(dyvz, MP ? ca[3] : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 3) : byh, m3, m + N_YVZ * a.fs);
            if (p4) dzvy = pml_up(dzvy, MP ? ca[4] : azh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 4) : bzh, m4, m + N_ZVY * a.fs);
            const float yzn = yz0 + g44 * (dzvy + dyvz);
            st[E3_YZ * a.fs + o] = yzn;
            if (mir) st[E3_YZ * a.fs + o + dsh] = -yzn;
            // sxz: dz vx + dx vz
            dzvx = zsh * stM<R>(vx, sz);
            dxvz = a.idx * stM<R>(vz, 1);
            if (p5) dxvz = pml_up(dxvz, MP ? ca[5] : axh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 5) : bxh, m5, m + N_XVZ * a.fs);
            if (p6) dzvx = pml_up(dzvx, MP ? ca[6] : azh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 6) : bzh, m6, m + N_ZVX * a.fs);
            const float xzn = xz0 + g55 * (dzvx + dxvz);
            st[E3_XZ * a.fs + o] = xzn;
            if (mir) st[E3_XZ * a.fs + o + dsh] = -xzn;
        }
        // sxy: dy vx + dx vy
        float dyvx = a.idy * stM<R>(vx, sy), dxvy = a.idx * stM<R>(vy, 1);
        if (p7) dxvy = pml_up(dxvy, MP ? ca[7] : axh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 7) : bxh, m7, m + N_XVY * a.fs);
        if (p8) dyvx = pml_up(dyvx, MP ? ca[8] : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 0, 8) : byh, m8, m + N_YVX * a.fs);
        st[E3_XY * a.fs + o] = xy0 + g66 * (dyvx + dxvy);
        if (STORE) {
            float* S = a.S + slot + s * a.fs + o;
            S[0] = dX; S[a.sterm] = dY; S[2 * a.sterm] = dZ;
            if (hz_ok) { S[3 * a.sterm] = dzvy + dyvz; S[4 * a.sterm] = dzvx + dxvz; }
            S[5 * a.sterm] = dyvx + dxvy;
        }
    }
}

template <int R, bool STORE, bool FS, bool MP>
__global__ void __launch_bounds__(256, MP ? 2 : 3) k_el3d_fwd_v(El3dDev a) {
    E3Cell c;
    if (!e3_cell(a, c)) return;
    const long long o = c.o, sy = a.pitch, sz = a.plane;
    const int x = c.x, y = c.y, z = c.z;
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
    const bool sh_vx = oxh || oyi || ozi, sh_vy = oxi || oyh || ozi, sh_vz = oxi || oyi || ozh;
    // MP: the M-PML (a, b) of each derivative of the node (shell nodes only);
    // otherwise the per-axis 1D tables above
    float ca[9];
    if (MP) {
        if (sh_vx || sh_vy || sh_vz) {
            e3_coef_load<E3_PERM_S>(a, o, 9, ca);
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) ca[q] = 0.f;
        }
    }
    const float axi = a.axi[x], bxi = a.bxi[x], axh = a.axh[x], bxh = a.bxh[x];
    const float ayi = a.ayi[y], byi = a.byi[y], ayh = a.ayh[y], byh = a.byh[y];
    const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
    const float bx = __ldg(a.bx + o), by = __ldg(a.by + o), bz = __ldg(a.bz + o);
    const float zsi = FS ? a.idz * __ldg(a.zfi + z) : a.idz, zsh = FS ? a.idz * __ldg(a.zfh + z) : a.idz;  // see k_el3d_fwd_s
    const int s0 = c.grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    const long long slot = STORE ? (long long)(*a.d_step % a.k) * a.sslot : 0;
    for (int s = s0; s < s1; ++s) {
        float* st = a.st + s * a.sst;
        const float* sxx = st + E3_XX * a.fs + o;
        const float* syy = st + E3_YY * a.fs + o;
        const float* szz = st + E3_ZZ * a.fs + o;
        const float* syz = st + E3_YZ * a.fs + o;
        const float* sxz = st + E3_XZ * a.fs + o;
        const float* sxy = st + E3_XY * a.fs + o;
        float* m = st + E3_M0 * a.fs + o;
        // the cell's old velocities and CPML memories are read ahead of its
        // first store (same buffer: no later plain read could move above a store)
        const bool vz_ok = !FS || z > a.pr;
        const float vx0 = st[E3_VX * a.fs + o], vy0 = st[E3_VY * a.fs + o];
        const float vz0 = vz_ok ? st[E3_VZ * a.fs + o] : 0.f;
        const bool p0 = sh_vx && (MP ? ca[0] : axh) != 0.f, p1 = sh_vx && (MP ? ca[1] : ayi) != 0.f, p2 = sh_vx && (MP ? ca[2] : azi) != 0.f;
        const bool p3 = sh_vy && (MP ? ca[3] : axi) != 0.f, p4 = sh_vy && (MP ? ca[4] : ayh) != 0.f, p5 = sh_vy && (MP ? ca[5] : azi) != 0.f;
        const bool p6 = vz_ok && sh_vz && (MP ? ca[6] : axi) != 0.f, p7 = vz_ok && sh_vz && (MP ? ca[7] : ayi) != 0.f,
                   p8 = vz_ok && sh_vz && (MP ? ca[8] : azh) != 0.f;
        const float m0 = p0 ? m[N_XXX * a.fs] : 0.f, m1 = p1 ? m[N_YXY * a.fs] : 0.f, m2 = p2 ? m[N_ZXZ * a.fs] : 0.f;
        const float m3 = p3 ? m[N_XXY * a.fs] : 0.f, m4 = p4 ? m[N_YYY * a.fs] : 0.f, m5 = p5 ? m[N_ZYZ * a.fs] : 0.f;
        const float m6 = p6 ? m[N_XXZ * a.fs] : 0.f, m7 = p7 ? m[N_YYZ * a.fs] : 0.f, m8 = p8 ? m[N_ZZZ * a.fs] : 0.f;
        // vx: dx sxx (M) + dy sxy (P) + dz sxz (P)
        float h1 = a.idx * stM<R>(sxx, 1), h2 = a.idy * stP<R>(sxy, sy), h3 = zsi * stP<R>(sxz, sz);
        if (p0) h1 = pml_up(h1, MP ? ca[0] : axh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 0) : bxh, m0, m + N_XXX * a.fs);
        if (p1) h2 = pml_up(h2, MP ? ca[1] : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 1) : byi, m1, m + N_YXY * a.fs);
        if (p2) h3 = pml_up(h3, MP ? ca[2] : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 2) : bzi, m2, m + N_ZXZ * a.fs);
        const float hx = h1 + h2 + h3;
        st[E3_VX * a.fs + o] = vx0 + bx * hx;
        // vy: dx sxy (P) + dy syy (M) + dz syz (P)
        h1 = a.idx * stP<R>(sxy, 1); h2 = a.idy * stM<R>(syy, sy); h3 = zsi * stP<R>(syz, sz);
        if (p3) h1 = pml_up(h1, MP ? ca[3] : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 3) : bxi, m3, m + N_XXY * a.fs);
        if (p4) h2 = pml_up(h2, MP ? ca[4] : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 4) : byh, m4, m + N_YYY * a.fs);
        if (p5) h3 = pml_up(h3, MP ? ca[5] : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 5) : bzi, m5, m + N_ZYZ * a.fs);
        const float hy = h1 + h2 + h3;
        st[E3_VY * a.fs + o] = vy0 + by * hy;
        // vz: dx sxz (P) + dy syz (P) + dz szz (M); with a free surface from row 2
        float hz = 0.f;
        if (vz_ok) {
            h1 = a.idx * stP<R>(sxz, 1); h2 = a.idy * stP<R>(syz, sy); h3 = zsh * stM<R>(szz, sz);
            if (p6) h1 = pml_up(h1, MP ? ca[6] : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 6) : bxi, m6, m + N_XXZ * a.fs);
            if (p7) h2 = pml_up(h2, MP ? ca[7] : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 7) : byi, m7, m + N_YYZ * a.fs);
            if (p8) h3 = pml_up(h3, MP ? ca[8] : azh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 8) : bzh, m8, m + N_ZZZ * a.fs);
            hz = h1 + h2 + h3;
            st[E3_VZ * a.fs + o] = vz0 + bz * hz;
        }
        if (STORE) {
            float* S = a.S + slot + s * a.fs + o;
            S[6 * a.sterm] = hx; S[7 * a.sterm] = hy; S[8 * a.sterm] = hz;
        }
    }
}

// ------------------------------- adjoint ------------------------------------
// adjoint planes per shot: 0..8 fields, 9..26 memory adjoints, 27..44 e terms
__device__ __forceinline__ void e3_kahan(float* G, long long gg, long long go, int q, float v) {
    float sm = G[q * gg + go], c = G[(12 + q) * gg + go];
    kahan_add(sm, c, v);
    G[q * gg + go] = sm;
    G[(12 + q) * gg + go] = c;
}

template <int R, bool FS, bool MP>
__global__ void __launch_bounds__(256, MP ? 2 : 3) k_el3d_adj_v(El3dDev a) {
    E3Cell c;
    if (!e3_cell(a, c)) return;
    const long long o = c.o, sy = a.pitch, sz = a.plane;
    const int x = c.x, y = c.y, z = c.z;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
    const bool sh_vx = oxh || oyi || ozi, sh_vy = oxi || oyh || ozi, sh_vz = oxi || oyi || ozh;
    // MP: the M-PML (a, b) of each derivative of the node (shell nodes only);
    // otherwise the per-axis 1D tables above
    float ca[9];
    if (MP) {
        if (sh_vx || sh_vy || sh_vz) {
            e3_coef_load<E3_PERM_S>(a, o, 9, ca);
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) ca[q] = 0.f;
        }
    }
    const float axi = a.axi[x], bxi = a.bxi[x], axh = a.axh[x], bxh = a.bxh[x];
    const float ayi = a.ayi[y], byi = a.byi[y], ayh = a.ayh[y], byh = a.byh[y];
    const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
    const float bx = __ldg(a.bx + o), by = __ldg(a.by + o), bz = __ldg(a.bz + o);
    // the z-derivative e terms carry the node's dz scaling, so that the
    // neighbours' transposed stencils stay plain
    const float fzi = FS ? __ldg(a.zfi + z) : 1.f, fzh = FS ? __ldg(a.zfh + z) : 1.f;
    const int s0 = c.grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    float gx = 0.f, gy = 0.f, gz = 0.f;
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        const float* e = ad + 27 * a.fs + o;
        float* mh = ad + 9 * a.fs + o;
        float* ew = ad + 27 * a.fs + o;
        const long long so = slot + s * a.fs + o;
        // the cell's old values and CPML memories are read ahead of its first
        // store: the stores go to the same buffer, so no later plain read could
        // be moved above them and every read would cost its own round trip
        const bool vz_ok = !FS || z > a.pr;
        const float vx0 = ad[E3_VX * a.fs + o], vy0 = ad[E3_VY * a.fs + o];
        const float vz0 = vz_ok ? ad[E3_VZ * a.fs + o] : 0.f;
        const bool p0 = sh_vx && (MP ? ca[0] : axh) != 0.f, p1 = sh_vx && (MP ? ca[1] : ayi) != 0.f, p2 = sh_vx && (MP ? ca[2] : azi) != 0.f;
        const bool p3 = sh_vy && (MP ? ca[3] : axi) != 0.f, p4 = sh_vy && (MP ? ca[4] : ayh) != 0.f, p5 = sh_vy && (MP ? ca[5] : azi) != 0.f;
        const bool p6 = vz_ok && sh_vz && (MP ? ca[6] : axi) != 0.f, p7 = vz_ok && sh_vz && (MP ? ca[7] : ayi) != 0.f,
                   p8 = vz_ok && sh_vz && (MP ? ca[8] : azh) != 0.f;
        const float m0 = p0 ? mh[N_XXX * a.fs] : 0.f, m1 = p1 ? mh[N_YXY * a.fs] : 0.f, m2 = p2 ? mh[N_ZXZ * a.fs] : 0.f;
        const float m3 = p3 ? mh[N_XXY * a.fs] : 0.f, m4 = p4 ? mh[N_YYY * a.fs] : 0.f, m5 = p5 ? mh[N_ZYZ * a.fs] : 0.f;
        const float m6 = p6 ? mh[N_XXZ * a.fs] : 0.f, m7 = p7 ? mh[N_YYZ * a.fs] : 0.f, m8 = p8 ? mh[N_ZZZ * a.fs] : 0.f;
        // vx^ += Dx^T e_xvx (P) + Dz^T e_zvx (M) + Dy^T e_yvx (M)
        float v = vx0 + a.idx * tP<R>(e + N_XVX * a.fs, 1) + a.idz * tM<R>(e + N_ZVX * a.fs, sz) +
                  a.idy * tM<R>(e + N_YVX * a.fs, sy);
        ad[E3_VX * a.fs + o] = v;
        gx += v * __ldg(a.S + 6 * a.sterm + so);
        float q = bx * v, e1 = q, e2 = q, e3 = q;
        if (p0) e1 = pml_adr(q, MP ? ca[0] : axh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 0) : bxh, m0, mh + N_XXX * a.fs);
        if (p1) e2 = pml_adr(q, MP ? ca[1] : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 1) : byi, m1, mh + N_YXY * a.fs);
        if (p2) e3 = pml_adr(q, MP ? ca[2] : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 2) : bzi, m2, mh + N_ZXZ * a.fs);
        ew[N_XXX * a.fs] = e1; ew[N_YXY * a.fs] = e2; ew[N_ZXZ * a.fs] = e3 * fzi;
        // vy^ += Dy^T e_yvy (P) + Dz^T e_zvy (M) + Dx^T e_xvy (M)
        v = vy0 + a.idy * tP<R>(e + N_YVY * a.fs, sy) + a.idz * tM<R>(e + N_ZVY * a.fs, sz) +
            a.idx * tM<R>(e + N_XVY * a.fs, 1);
        ad[E3_VY * a.fs + o] = v;
        gy += v * __ldg(a.S + 7 * a.sterm + so);
        q = by * v; e1 = q; e2 = q; e3 = q;
        if (p3) e1 = pml_adr(q, MP ? ca[3] : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 3) : bxi, m3, mh + N_XXY * a.fs);
        if (p4) e2 = pml_adr(q, MP ? ca[4] : ayh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 4) : byh, m4, mh + N_YYY * a.fs);
        if (p5) e3 = pml_adr(q, MP ? ca[5] : azi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 5) : bzi, m5, mh + N_ZYZ * a.fs);
        ew[N_XXY * a.fs] = e1; ew[N_YYY * a.fs] = e2; ew[N_ZYZ * a.fs] = e3 * fzi;
        // vz^ += Dz^T e_zvz (P) + Dy^T e_yvz (M) + Dx^T e_xvz (M); with a free surface from row 2
        if (vz_ok) {
            v = vz0 + a.idz * tP<R>(e + N_ZVZ * a.fs, sz) + a.idy * tM<R>(e + N_YVZ * a.fs, sy) +
                a.idx * tM<R>(e + N_XVZ * a.fs, 1);
            ad[E3_VZ * a.fs + o] = v;
            gz += v * __ldg(a.S + 8 * a.sterm + so);
            q = bz * v; e1 = q; e2 = q; e3 = q;
            if (p6) e1 = pml_adr(q, MP ? ca[6] : axi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 6) : bxi, m6, mh + N_XXZ * a.fs);
            if (p7) e2 = pml_adr(q, MP ? ca[7] : ayi, MP ? e3_cb<E3_PERM_S>(a, o, 9, 7) : byi, m7, mh + N_YYZ * a.fs);
            if (p8) e3 = pml_adr(q, MP ? ca[8] : azh, MP ? e3_cb<E3_PERM_S>(a, o, 9, 8) : bzh, m8, mh + N_ZZZ * a.fs);
            ew[N_XXZ * a.fs] = e1; ew[N_YYZ * a.fs] = e2; ew[N_ZZZ * a.fs] = e3 * fzh;
        }
    }
    const long long go = (long long)c.grp * a.fs + o;
    e3_kahan(a.G, a.gg, go, 9, gx);
    e3_kahan(a.G, a.gg, go, 10, gy);
    e3_kahan(a.G, a.gg, go, 11, gz);
}

template <int R, bool FS, bool MP>
__global__ void __launch_bounds__(256, MP ? 2 : 3) k_el3d_adj_s(El3dDev a) {
    E3Cell c;
    if (!e3_cell(a, c)) return;
    const long long o = c.o, sy = a.pitch, sz = a.plane;
    const int x = c.x, y = c.y, z = c.z;
    const int t = *a.d_step;
    const long long slot = (long long)((t - 1) % a.k) * a.sslot;
    const bool oxi = e3_out(x, a.pr, a.nx, false), oxh = e3_out(x, a.pr, a.nx, true);
    const bool oyi = e3_out(y, a.pr, a.ny, false), oyh = e3_out(y, a.pr, a.ny, true);
    const bool ozi = e3_out(z, a.pr, a.nz, false), ozh = e3_out(z, a.pr, a.nz, true);
    const bool sh_n = oxi || oyi || ozi, sh_yz = oxi || oyh || ozh, sh_xz = oxh || oyi || ozh, sh_xy = oxh || oyh || ozi;
    // MP: the M-PML (a, b) of each derivative of the node (shell nodes only);
    // otherwise the per-axis 1D tables above
    float ca[9];
    if (MP) {
        if (sh_n || sh_yz || sh_xz || sh_xy) {
            e3_coef_load<E3_PERM_AS>(a, o, 0, ca);
        } else {
#pragma unroll
            for (int q = 0; q < 9; ++q) ca[q] = 0.f;
        }
    }
    const float axi = a.axi[x], bxi = a.bxi[x], axh = a.axh[x], bxh = a.bxh[x];
    const float ayi = a.ayi[y], byi = a.byi[y], ayh = a.ayh[y], byh = a.byh[y];
    const float azi = a.azi[z], bzi = a.bzi[z], azh = a.azh[z], bzh = a.bzh[z];
    const float c11 = __ldg(a.c11 + o), c12 = __ldg(a.c12 + o), c13 = __ldg(a.c13 + o), c22 = __ldg(a.c22 + o),
                c23 = __ldg(a.c23 + o), c33 = __ldg(a.c33 + o);
    const float g44 = a.dt * __ldg(a.c44e + o), g55 = a.dt * __ldg(a.c55e + o), g66 = a.dt * __ldg(a.c66e + o);
    const int s0 = c.grp * a.spt, s1 = min(a.nshots, s0 + a.spt);
    // free surface: row 1 (traction condition, sigma_zz overwritten by 0), the
    // half-depth stresses from row 2, and the image rows whose adjoint folds back
    // onto this node with the image's minus (sigma_zz: 2 pr - z, syz / sxz: 2 pr + 1 - z)
    const bool row1 = FS && z == a.pr, hz_ok = !FS || z > a.pr;
    const bool mir = FS && z > a.pr && z <= a.pr + a.R;
    const long long dzz = (long long)(2 * a.pr - 2 * z) * sz, dsh = dzz + sz;
    const float r13 = c13 / c33, r23 = c23 / c33;
    const float fzi = FS ? __ldg(a.zfi + z) : 1.f, fzh = FS ? __ldg(a.zfh + z) : 1.f;  // see k_el3d_adj_v
    float G[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int s = s0; s < s1; ++s) {
        float* ad = a.ad + s * a.sad;
        const float* e = ad + 27 * a.fs + o;
        float* ew = ad + 27 * a.fs + o;
        float* mh = ad + 9 * a.fs + o;
        const float* S = a.S + slot + s * a.fs + o;
        // the cell's old values and CPML memories are read ahead of its first
        // store (same buffer: no later plain read could move above a store)
        const float xx0 = ad[E3_XX * a.fs + o], yy0 = ad[E3_YY * a.fs + o];
        const float zz0 = row1 ? 0.f : ad[E3_ZZ * a.fs + o];
        const float yz0 = hz_ok ? ad[E3_YZ * a.fs + o] : 0.f, xz0 = hz_ok ? ad[E3_XZ * a.fs + o] : 0.f;
        const float xy0 = ad[E3_XY * a.fs + o];
        const bool p0 = (row1 || sh_n) && (MP ? ca[0] : axi) != 0.f, p1 = (row1 || sh_n) && (MP ? ca[1] : ayi) != 0.f, p2 = !row1 && sh_n && (MP ? ca[2] : azi) != 0.f;
        const bool p3 = hz_ok && sh_yz && (MP ? ca[3] : azh) != 0.f, p4 = hz_ok && sh_yz && (MP ? ca[4] : ayh) != 0.f;
        const bool p5 = hz_ok && sh_xz && (MP ? ca[5] : azh) != 0.f, p6 = hz_ok && sh_xz && (MP ? ca[6] : axh) != 0.f;
        const bool p7 = sh_xy && (MP ? ca[7] : ayh) != 0.f, p8 = sh_xy && (MP ? ca[8] : axh) != 0.f;
        const float m0 = p0 ? mh[N_XVX * a.fs] : 0.f, m1 = p1 ? mh[N_YVY * a.fs] : 0.f, m2 = p2 ? mh[N_ZVZ * a.fs] : 0.f;
        const float m3 = p3 ? mh[N_ZVY * a.fs] : 0.f, m4 = p4 ? mh[N_YVZ * a.fs] : 0.f;
        const float m5 = p5 ? mh[N_ZVX * a.fs] : 0.f, m6 = p6 ? mh[N_XVZ * a.fs] : 0.f;
        const float m7 = p7 ? mh[N_YVX * a.fs] : 0.f, m8 = p8 ? mh[N_XVY * a.fs] : 0.f;
        const float xh = xx0 + a.idx * tM<R>(e + N_XXX * a.fs, 1);
        const float yh = yy0 + a.idy * tM<R>(e + N_YYY * a.fs, sy);
        float zh = 0.f, yzh = 0.f, xzh = 0.f;
        if (!row1) {
            float dzz_s = a.idz * tM<R>(e + N_ZZZ * a.fs, sz);
            if (mir) {
                const float* em = e + N_ZZZ * a.fs + dzz;
                float f = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) f = f + c_fd3e[q - 1] * __ldg(em + q * sz);
                dzz_s = dzz_s + a.idz * f;
            }
            zh = zz0 + dzz_s;
        }
        if (hz_ok) {
            float dyz = a.idz * tP<R>(e + N_ZYZ * a.fs, sz) + a.idy * tP<R>(e + N_YYZ * a.fs, sy);
            float dxz = a.idz * tP<R>(e + N_ZXZ * a.fs, sz) + a.idx * tP<R>(e + N_XXZ * a.fs, 1);
            if (mir) {
                const float* ey = e + N_ZYZ * a.fs + dsh;
                const float* ex = e + N_ZXZ * a.fs + dsh;
                float fy = 0.f, fx = 0.f;
#pragma unroll
                for (int q = 1; q <= R; ++q) {
                    fy = fy + c_fd3e[q - 1] * __ldg(ey + (q - 1) * sz);
                    fx = fx + c_fd3e[q - 1] * __ldg(ex + (q - 1) * sz);
                }
                dyz = dyz + a.idz * fy;
                dxz = dxz + a.idz * fx;
            }
            yzh = yz0 + dyz;
            xzh = xz0 + dxz;
            ad[E3_YZ * a.fs + o] = yzh;
            ad[E3_XZ * a.fs + o] = xzh;
        }
        const float xyh = xy0 + a.idy * tP<R>(e + N_YXY * a.fs, sy) + a.idx * tP<R>(e + N_XXY * a.fs, 1);
        ad[E3_XX * a.fs + o] = xh; ad[E3_YY * a.fs + o] = yh; ad[E3_ZZ * a.fs + o] = zh;
        ad[E3_XY * a.fs + o] = xyh;
        const float dX = __ldg(S), dY = __ldg(S + a.sterm), dZ = __ldg(S + 2 * a.sterm);
        float qx, qy, qz = 0.f;
        if (row1) {
            // dZ = -(c13 dX + c23 dY) / c33 and sigma_zz(1) = 0
            G[0] += xh * dX;
            G[1] += xh * dY + yh * dX;
            G[2] += xh * (dZ - r13 * dX) - yh * r23 * dX;
            G[3] += yh * dY;
            G[4] += yh * (dZ - r23 * dY) - xh * r13 * dY;
            G[5] += -(xh * r13 + yh * r23) * dZ;
            const float w = a.dt * (c13 * xh + c23 * yh);
            qx = a.dt * (c11 * xh + c12 * yh) - r13 * w;
            qy = a.dt * (c12 * xh + c22 * yh) - r23 * w;
            if (p0) qx = pml_adr(qx, MP ? ca[0] : axi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 0) : bxi, m0, mh + N_XVX * a.fs);
            if (p1) qy = pml_adr(qy, MP ? ca[1] : ayi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 1) : byi, m1, mh + N_YVY * a.fs);
        } else {
            G[0] += xh * dX;
            G[1] += xh * dY + yh * dX;
            G[2] += xh * dZ + zh * dX;
            G[3] += yh * dY;
            G[4] += yh * dZ + zh * dY;
            G[5] += zh * dZ;
            qx = a.dt * (c11 * xh + c12 * yh + c13 * zh);
            qy = a.dt * (c12 * xh + c22 * yh + c23 * zh);
            qz = a.dt * (c13 * xh + c23 * yh + c33 * zh);
            if (p0) qx = pml_adr(qx, MP ? ca[0] : axi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 0) : bxi, m0, mh + N_XVX * a.fs);
            if (p1) qy = pml_adr(qy, MP ? ca[1] : ayi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 1) : byi, m1, mh + N_YVY * a.fs);
            if (p2) qz = pml_adr(qz, MP ? ca[2] : azi, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 2) : bzi, m2, mh + N_ZVZ * a.fs);
        }
        ew[N_XVX * a.fs] = qx; ew[N_YVY * a.fs] = qy; ew[N_ZVZ * a.fs] = qz * fzi;
        float q, e1, e2;
        if (hz_ok) {
            G[6] += yzh * __ldg(S + 3 * a.sterm);
            G[7] += xzh * __ldg(S + 4 * a.sterm);
            q = g44 * yzh; e1 = q; e2 = q;
            if (p3) e1 = pml_adr(q, MP ? ca[3] : azh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 3) : bzh, m3, mh + N_ZVY * a.fs);
            if (p4) e2 = pml_adr(q, MP ? ca[4] : ayh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 4) : byh, m4, mh + N_YVZ * a.fs);
            ew[N_ZVY * a.fs] = e1 * fzh; ew[N_YVZ * a.fs] = e2;
            q = g55 * xzh; e1 = q; e2 = q;
            if (p5) e1 = pml_adr(q, MP ? ca[5] : azh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 5) : bzh, m5, mh + N_ZVX * a.fs);
            if (p6) e2 = pml_adr(q, MP ? ca[6] : axh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 6) : bxh, m6, mh + N_XVZ * a.fs);
            ew[N_ZVX * a.fs] = e1 * fzh; ew[N_XVZ * a.fs] = e2;
        }
        G[8] += xyh * __ldg(S + 5 * a.sterm);
        q = g66 * xyh; e1 = q; e2 = q;
        if (p7) e1 = pml_adr(q, MP ? ca[7] : ayh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 7) : byh, m7, mh + N_YVX * a.fs);
        if (p8) e2 = pml_adr(q, MP ? ca[8] : axh, MP ? e3_cb<E3_PERM_AS>(a, o, 0, 8) : bxh, m8, mh + N_XVY * a.fs);
        ew[N_YVX * a.fs] = e1; ew[N_XVY * a.fs] = e2;
    }
    const long long go = (long long)c.grp * a.fs + o;
#pragma unroll
    for (int q = 0; q < 9; ++q) e3_kahan(a.G, a.gg, go, q, G[q]);
}

#include "el3d_ring_adj.cuh"

// ---- Thomsen parameterisation (thomsen_to_cij3d, src/lib/module_anisotropy.f90:336-381) ----
// Dual numbers (value, derivative) for the forward-mode derivatives of the Cij
// set-up in the chain rule; float / double evaluate the same code.
struct Dual {
    double v, d;
};
__host__ __device__ inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ inline double tval(Dual a) { return a.v; }
__host__ __device__ inline double tval(double a) { return a; }
__host__ __device__ inline double tval(float a) { return a; }
__host__ __device__ inline Dual tsqrt(Dual a) {
    const double r = sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}
__host__ __device__ inline Dual tabs(Dual a) { return a.v < 0 ? -a : a; }
__host__ __device__ inline Dual tcos(Dual a) { return {cos(a.v), -a.d * sin(a.v)}; }
__host__ __device__ inline Dual tsin(Dual a) { return {sin(a.v), a.d * cos(a.v)}; }
__host__ __device__ inline double tsqrt(double a) { return sqrt(a); }
__host__ __device__ inline double tabs(double a) { return fabs(a); }
__host__ __device__ inline double tcos(double a) { return cos(a); }
__host__ __device__ inline double tsin(double a) { return sin(a); }
__host__ __device__ inline float tsqrt(float a) { return sqrtf(a); }
__host__ __device__ inline float tabs(float a) { return fabsf(a); }
__host__ __device__ inline float tcos(float a) { return cosf(a); }
__host__ __device__ inline float tsin(float a) { return sinf(a); }
template <typename T>
__host__ __device__ inline T tc(double v) { return T(v); }
template <>
__host__ __device__ inline Dual tc<Dual>(double v) { return Dual{v, 0.0}; }

// p: vp, vs, epsilon, delta, gamma, theta, phi, rho -> c: the nine ORT moduli
// (c11 c12 c13 c22 c23 c33 c44 c55 c66) and rho. A tilt rotates the tensor by
// rotation_matrix([0, -theta, -phi], 'xyz') and bond_matrix (:127-170,
// :233-291): restated as r = Rz(-phi) Ry(-theta), C' = M C M^T with the Bond
// matrix M of r; the solver keeps the nine ORT entries of C'.
template <typename T>
__host__ __device__ void thomsen3d_cij(const T* p, T* c) {
    const T vp = p[0], vs = p[1], eps = p[2], del = p[3], gam = p[4], the = p[5], phi = p[6], rho = p[7];
    const T c33 = vp * vp * rho, c44 = vs * vs * rho;
    const T c11 = c33 * (tc<T>(1) + tc<T>(2) * eps), c66 = c44 * (tc<T>(1) + tc<T>(2) * gam);
    const T c12 = c11 - tc<T>(2) * c66;
    const T tmp = tc<T>(2) * c33 * (c33 - c44) * del + (c33 - c44) * (c33 - c44);
    const T c13 = tsqrt(tabs(tmp)) - c44;
    c[0] = c11; c[1] = c12; c[2] = c13; c[3] = c11; c[4] = c13; c[5] = c33; c[6] = c44; c[7] = c44; c[8] = c66;
    c[9] = rho;
    if ((tval(the) != 0.0 || tval(phi) != 0.0) && !(tval(eps) == 0.0 && tval(del) == 0.0 && tval(gam) == 0.0)) {
        const T cb = tcos(-the), sb = tsin(-the), cg = tcos(-phi), sg = tsin(-phi);
        const T z0 = tc<T>(0);
        const T r[3][3] = {{cg * cb, -sg, cg * sb}, {sg * cb, cg, sg * sb}, {-sb, z0, cb}};
        T M[6][6];
        const int pi[6] = {0, 1, 2, 1, 0, 0}, pj[6] = {0, 1, 2, 2, 2, 1};  // Voigt index pairs
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                const int i = pi[a], j = pj[a], k = pi[b], l = pj[b];
                if (a < 3) M[a][b] = b < 3 ? r[i][k] * r[i][k] : tc<T>(2) * r[i][k] * r[i][l];
                else M[a][b] = b < 3 ? r[i][k] * r[j][k] : r[i][k] * r[j][l] + r[i][l] * r[j][k];
            }
        const T C6[6][6] = {{c11, c12, c13, z0, z0, z0}, {c12, c11, c13, z0, z0, z0}, {c13, c13, c33, z0, z0, z0},
                            {z0, z0, z0, c44, z0, z0},   {z0, z0, z0, z0, c44, z0},   {z0, z0, z0, z0, z0, c66}};
        T MC[6][6];
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                T acc = tc<T>(0);
                for (int q = 0; q < 6; ++q) acc = acc + M[a][q] * C6[q][b];
                MC[a][b] = acc;
            }
        auto rot = [&](int a, int b) {
            T acc = tc<T>(0);
            for (int q = 0; q < 6; ++q) acc = acc + MC[a][q] * M[b][q];
            return acc;
        };
        c[0] = rot(0, 0); c[1] = rot(0, 1); c[2] = rot(0, 2); c[3] = rot(1, 1); c[4] = rot(1, 2); c[5] = rot(2, 2);
        c[6] = rot(3, 3); c[7] = rot(4, 4); c[8] = rot(5, 5);
    }
}

// FP64 chain rule on the padded model grid: d J / d (c11 c12 c13 c22 c23 c33 c44 c55 c66 rho),
// then the parameters (iso: vp, vs, rho; cij: the nine moduli and rho; thomsen:
// the eight parameters through dual-number derivatives of thomsen3d_cij)
__global__ void k_el3d_chain(El3dDev a, int ngroups, int iso, const float* __restrict__ p0, const float* __restrict__ p1,
                             const float* __restrict__ tpar,
                             const float* __restrict__ c44p, const float* __restrict__ c55p,
                             const float* __restrict__ c66p, const float* __restrict__ rhop, double* __restrict__ gpad,
                             int nxq, int nyq, int nzq) {
    const long long n = (long long)nxq * nyq * nzq;
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < n;
         cell += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(cell % nxq), iy = (int)((cell / nxq) % nyq), iz = (int)(cell / ((long long)nxq * nyq));
        const int x = a.R - 1 + ix, y = a.R - 1 + iy, z = a.R - 1 + iz;
        const long long o = (long long)z * a.plane + (long long)y * a.pitch + x;
        auto sumG = [&](int q, long long oo) {
            double v = 0;
            for (int g = 0; g < ngroups; ++g)
                v += (double)a.G[q * a.gg + g * a.fs + oo] - (double)a.G[(12 + q) * a.gg + g * a.fs + oo];
            return v;
        };
        auto inside = [&](int xx, int yy, int zz) {
            return xx >= a.x0 && xx < a.x1 && yy >= a.y0 && yy < a.y1 && zz >= a.z0 && zz < a.z1;
        };
        const double dt = a.dt;
        double dc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (inside(x, y, z))
            for (int q = 0; q < 6; ++q) dc[q] = dt * sumG(q, o);
        const double cc[3] = {c44p[o], c55p[o], c66p[o]};
        const float* ce[3] = {a.c44e, a.c55e, a.c66e};
        for (int d1 = 0; d1 <= 1; ++d1)
            for (int d2 = 0; d2 <= 1; ++d2) {
                // syz nodes (x, y+d1, z+d2), sxz nodes (x+d1, y, z+d2), sxy nodes (x+d1, y+d2, z)
                const int nx3[3] = {x, x + d1, x + d1}, ny3[3] = {y + d1, y, y + d2}, nz3[3] = {z + d2, z + d2, z};
                for (int q = 0; q < 3; ++q) {
                    if (!inside(nx3[q], ny3[q], nz3[q])) continue;
                    const long long on = (long long)nz3[q] * a.plane + (long long)ny3[q] * a.pitch + nx3[q];
                    const double e = ce[q][on];
                    if (e != 0.0) dc[6 + q] += dt * sumG(6 + q, on) * e * e / (4.0 * cc[q] * cc[q]);
                }
            }
        for (int d = 0; d <= 1; ++d) {
            const long long sx = 1, sy = a.pitch, sz = a.plane;
            const int px[3] = {x + d, x, x}, py[3] = {y, y + d, y}, pz[3] = {z, z, z + d};
            const long long st[3] = {sx, sy, sz};
            for (int q = 0; q < 3; ++q) {
                if (!inside(px[q], py[q], pz[q])) continue;
                const long long on = (long long)pz[q] * a.plane + (long long)py[q] * a.pitch + px[q];
                const double re = 0.5 * ((double)rhop[on - st[q]] + (double)rhop[on]);
                dc[9] -= 0.5 * dt * sumG(9 + q, on) / (re * re);
            }
        }
        const long long npad = n;
        if (tpar) {
            double pv[8];
            for (int q = 0; q < 8; ++q) pv[q] = tpar[q * a.fs + o];
            for (int q = 0; q < 8; ++q) {
                Dual pd[8], cd[10];
                for (int r = 0; r < 8; ++r) pd[r] = Dual{pv[r], r == q ? 1.0 : 0.0};
                thomsen3d_cij(pd, cd);
                double g = 0.0;
                for (int r = 0; r < 10; ++r) g += dc[r] * cd[r].d;
                gpad[q * npad + cell] += g;
            }
        } else if (iso) {
            const double vp = p0[o], vs = p1[o], rho = rhop[o];
            const double sn = dc[0] + dc[3] + dc[5], so = dc[1] + dc[2] + dc[4], ss = dc[6] + dc[7] + dc[8];
            gpad[cell] += 2.0 * rho * vp * (sn + so);
            gpad[npad + cell] += 2.0 * rho * vs * ss - 4.0 * rho * vs * so;
            gpad[2 * npad + cell] += vp * vp * sn + (vp * vp - 2.0 * vs * vs) * so + vs * vs * ss + dc[9];
        } else {
            for (int q = 0; q < 10; ++q) gpad[q * npad + cell] += dc[q];
        }
    }
}

// Refined free-surface mesh: the mesh cells' d J / d (c11 .. c66, rho) (gpad
// planes 0..9, written by the cij branch of k_el3d_chain) to the regular padded
// planes -- the transpose of the depth interpolation that maps the regular Cij
// to the mesh (regular plane r gets the sum over mesh planes f of w(f, r) g(f),
// the pairs zptr / zrow / zw) -- then the Jacobian of the parameterisation at
// the regular cell: iso from (vp, vs, rho) in jpar, thomsen from its eight
// parameters, cij the identity. FP64, one thread per regular padded cell.
__global__ void k_el3d_zmap(const double* __restrict__ gmesh, long long npad_m, const int* __restrict__ zptr,
                            const int* __restrict__ zrow, const double* __restrict__ zw, int aniso,
                            const float* __restrict__ jpar, long long npad_r, double* __restrict__ gout, int nxq,
                            int nyq) {
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < npad_r;
         cell += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(cell % nxq), iy = (int)((cell / nxq) % nyq), iz = (int)(cell / ((long long)nxq * nyq));
        double dc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int e = zptr[iz]; e < zptr[iz + 1]; ++e) {
            const long long cm = ((long long)zrow[e] * nyq + iy) * nxq + ix;
            const double w = zw[e];
            for (int q = 0; q < 10; ++q) dc[q] += w * gmesh[q * npad_m + cm];
        }
        if (aniso == OWL_ANISO_THOMSEN) {
            double pv[8];
            for (int q = 0; q < 8; ++q) pv[q] = jpar[q * npad_r + cell];
            for (int q = 0; q < 8; ++q) {
                Dual pd[8], cd[10];
                for (int r = 0; r < 8; ++r) pd[r] = Dual{pv[r], r == q ? 1.0 : 0.0};
                thomsen3d_cij(pd, cd);
                double g = 0.0;
                for (int r = 0; r < 10; ++r) g += dc[r] * cd[r].d;
                gout[q * npad_r + cell] = g;
            }
        } else if (aniso == OWL_ANISO_ISO) {
            const double vp = jpar[cell], vs = jpar[npad_r + cell], rho = jpar[2 * npad_r + cell];
            const double sn = dc[0] + dc[3] + dc[5], so = dc[1] + dc[2] + dc[4], ss = dc[6] + dc[7] + dc[8];
            gout[cell] = 2.0 * rho * vp * (sn + so);
            gout[npad_r + cell] = 2.0 * rho * vs * ss - 4.0 * rho * vs * so;
            gout[2 * npad_r + cell] = vp * vp * sn + (vp * vp - 2.0 * vs * vs) * so + vs * vs * ss + dc[9];
        } else {
            for (int q = 0; q < 10; ++q) gout[q * npad_r + cell] = dc[q];
        }
    }
}

// ============================================================================
// host engine
// ============================================================================
namespace {
// per-axis damping tables (module_cfspml.f90:517-600 profiles, damp_coef macro of
// module_wavefield.f90:40-43, kappa = 1, zero M-PML ratio)
// (low = false: no damping at the low end, the free-surface top, module_cfspml.f90:573-585)
// (rows: the per-row spacing of the refined free-surface mesh, the reference's
// dz_i(k) of module_cfspml.f90:581-582, else the uniform d)
void e3_axis(int n, int pml, int R, int len, float d, float dt, float pmlvp, float alphamax, std::vector<float>& out,
             bool low = true, const VMesh* rows = nullptr) {
    out.assign(4 * (size_t)len, 0.f);  // ai, bi, ah, bh
    const float R0 = 1.0e-5f, adt = std::fabs(dt);
    auto ab = [&](float dd, float al, float& a, float& b) {
        const float bb = dd + al;
        a = -2.0f * adt * dd / (2.0f + adt * bb);
        b = (2.0f - adt * bb) / (2.0f + adt * bb);
    };
    for (int i = -pml + 1; i <= n + pml; ++i) {
        float nd, ndh;
        if (i <= 1) {
            if (!low) continue;
            nd = (float)std::abs(i - 1) * 1.0f / (float)pml;
            ndh = std::fabs((float)(i - 1) - 0.5f) * 1.0f / (float)pml;
        } else if (i >= n) {
            nd = (float)std::abs(i - n) * 1.0f / (float)pml;
            ndh = std::fabs((float)(i - n) - 0.5f) * 1.0f / (float)pml;
        } else {
            continue;
        }
        const float di = rows && rows->refined ? rows->get(rows->dzi, i) : d;
        const float c0 = std::log(1.0f / R0) * 3.0f * pmlvp / (2.0f * (float)pml * di);
        const int x = i + pml + R - 1;
        ab(c0 * (nd * nd), std::max(alphamax * (1.0f - nd), 0.25f * alphamax), out[x], out[len + x]);
        ab(c0 * (ndh * ndh), std::max(alphamax * (1.0f - ndh), 0.25f * alphamax), out[2 * len + x], out[3 * len + x]);
    }
}
VMesh checked_vmesh3(const owl_ssg_desc& d) {
    try {
        return build_vmesh(d);
    } catch (const std::invalid_argument& e) {
        throw OwlError(OWL_ERR_INVALID, e.what());
    }
}

owl_ssg_desc with_rows3(owl_ssg_desc d, int nz) {
    d.nz = nz;
    return d;
}

int el3d_nparam(int aniso) { return aniso == OWL_ANISO_ISO ? 3 : aniso == OWL_ANISO_THOMSEN ? 8 : 10; }

// Cij (c11, c12, c13, c22, c23, c33, c44, c55, c66, rho) of one model cell from
// its parameters (module_vars.f90:278-296, 362-375); pp gets the parameters
void e3_cell_cij(int aniso, const float* const* f, size_t src, float* v, float* pp) {
    if (aniso == OWL_ANISO_ISO) {
        const float vp = f[0][src], vs = f[1][src], rho = f[2][src];
        const float a11 = rho * (vp * vp), a44 = rho * (vs * vs), a12 = a11 - 2 * a44;
        const float w[10] = {a11, a12, a12, a11, a12, a11, a44, a44, a44, rho};
        std::copy(w, w + 10, v);
        pp[0] = vp; pp[1] = vs; pp[2] = rho;
    } else if (aniso == OWL_ANISO_THOMSEN) {
        for (int q = 0; q < 8; ++q) pp[q] = f[q][src];
        thomsen3d_cij(pp, v);
    } else {
        for (int q = 0; q < 10; ++q) v[q] = pp[q] = f[q][src];
    }
}
}  // namespace

// refine_nz of the refined free-surface mesh (module_vars.f90:424-428 of the 3D
// solver): ceiling(0.5 lambda / dz), lambda = sqrt(max of the means of c44 / rho,
// c55 / rho, c66 / rho over the padded surface plane) / f0_min
int el3d_refine_rows(const owl_ssg_desc& d, int np, const float* const* f, float f0_min) {
    OWL_CHECK(np == el3d_nparam(d.aniso) && f, OWL_ERR_INVALID,
              "elastic 3D model needs " + std::to_string(el3d_nparam(d.aniso)) + " parameters for this parameterisation");
    for (int q = 0; q < np; ++q) OWL_CHECK(f[q], OWL_ERR_INVALID, "null model parameter");
    OWL_CHECK(d.nx >= 1 && d.ny >= 1 && d.nz >= 1 && d.pml >= 0 && d.dz > 0, OWL_ERR_INVALID, "bad grid");
    float sum[3] = {0.f, 0.f, 0.f};
    long long cnt = 0;
    for (int j = -d.pml; j <= d.ny + d.pml + 1; ++j)
        for (int i = -d.pml; i <= d.nx + d.pml + 1; ++i) {
            const int ii = std::min(std::max(i, 1), d.nx), jj = std::min(std::max(j, 1), d.ny);
            const size_t src = ((size_t)(ii - 1) * d.ny + (jj - 1)) * d.nz;
            float v[10], pp[10];
            e3_cell_cij(d.aniso, f, src, v, pp);
            OWL_CHECK(v[9] > 0, OWL_ERR_INVALID, "rho must be positive");
            for (int q = 0; q < 3; ++q) sum[q] += v[6 + q] / v[9];
            ++cnt;
        }
    const float m = std::max({sum[0] / (float)cnt, sum[1] / (float)cnt, sum[2] / (float)cnt});
    const float lambda = std::sqrt(m) / f0_min;
    return (int)std::ceil(0.5f * lambda / d.dz);
}

struct El3dEngine : SsgBase {
    int aniso;
    float idx, idy, idz;
    // depth-refined free-surface mesh: the engine runs on the mesh's planes (nz
    // of the base), the model and the gradient stay on the regular nz_model planes
    VMesh vm;
    int nz_model;
    DevBuf<float> zfi, zfh, jparp;
    DevBuf<double> zw, gzmap;
    DevBuf<int> zptr, zrow;
    ZInterp zt;
    DevBuf<float> c11, c12, c13, c22, c23, c33, c44e, c55e, c66e, bxp, byp, bzp;
    DevBuf<float> c44p, c55p, c66p, rhop, p0p, p1p, tabx, taby, tabz, tparp;
    // M-PML: nonzero face ratios, the faces in the layout of owl_ssg_mpml_ratios,
    // per-axis profiles (d and alpha at integer and half positions) and the
    // faces in storage layout
    bool mpml = false;
    std::vector<float> h_faces;
    DevBuf<float> mp_prof, mp_face, mp_coef;
    const std::vector<float>* mpml_faces() const override { return &h_faces; }

    // the M-PML tables of the model (module_cfspml.f90:421-625): damping and
    // alpha profiles per axis, and the six faces' ratios (zero for iso)
    void build_mpml(const std::vector<float>* hc, float pmlvp, float alphamax) {
        const bool fsf = desc.free_surface != 0;
        const int len[3] = {pitch, NYs, NZs}, nn[3] = {nx, ny, nz};
        const float dd[3] = {desc.dx, desc.dy, desc.dz};
        const float R0 = 1.0e-5f;
        std::vector<float> prof;
        for (int ax = 0; ax < 3; ++ax) {
            const int L = len[ax], n = nn[ax];
            std::vector<float> t(4 * (size_t)L, 0.f);
            std::fill(t.begin() + 2 * L, t.end(), alphamax);
            const bool low = !(ax == 2 && fsf);  // no top PML under a free surface
            for (int i = -P + 1; i <= n + P; ++i) {
                float nd, ndh;
                if (i <= 1) {
                    if (!low) continue;
                    nd = (float)std::abs(i - 1) * 1.0f / (float)P;
                    ndh = std::fabs((float)(i - 1) - 0.5f) * 1.0f / (float)P;
                } else if (i >= n) {
                    nd = (float)std::abs(i - n) * 1.0f / (float)P;
                    ndh = std::fabs((float)(i - n) - 0.5f) * 1.0f / (float)P;
                } else {
                    continue;
                }
                const float di = ax == 2 && vm.refined ? vm.get(vm.dzi, i) : dd[ax];
                const float c0 = std::log(1.0f / R0) * 3.0f * pmlvp / (2.0f * (float)P * di);
                const int x = i + pr - 1;
                t[x] = c0 * (nd * nd);
                t[L + x] = c0 * (ndh * ndh);
                t[2 * (size_t)L + x] = std::max(alphamax * (1.0f - nd), 0.25f * alphamax);
                t[3 * (size_t)L + x] = std::max(alphamax * (1.0f - ndh), 0.25f * alphamax);
            }
            prof.insert(prof.end(), t.begin(), t.end());
        }
        const size_t fx = (size_t)NYp * NZp, fy = (size_t)NXp * NZp, fz = (size_t)NXp * NYp;
        h_faces.assign(2 * (fx + fy + fz), 0.f);
        float* fL = h_faces.data();
        float* fR = fL + fx;
        float* fF = fR + fx;
        float* fB = fF + fy;
        float* fT = fB + fy;
        float* fO = fT + fz;
        if (aniso != OWL_ANISO_ISO) {
            // the x / y faces span the rows the solver updates: from row 1 under a free surface
            const int z1 = fsf ? 1 : -P + 1, n2 = nz + P - z1 + 1, zoff = z1 + P - 1;
            auto cell = [&](int i, int j, int k, float* c) {
                const long long o = soff(i, j, k);
                for (int q = 0; q < 9; ++q) c[q] = hc[q][o];
            };
            mpml_face(NYp, n2, 0, [&](int a, int b, float* c) { cell(1, -P + 1 + a, z1 + b, c); },
                      fL + (size_t)zoff * NYp, NYp);
            mpml_face(NYp, n2, 0, [&](int a, int b, float* c) { cell(nx, -P + 1 + a, z1 + b, c); },
                      fR + (size_t)zoff * NYp, NYp);
            mpml_face(NXp, n2, 1, [&](int a, int b, float* c) { cell(-P + 1 + a, 1, z1 + b, c); },
                      fF + (size_t)zoff * NXp, NXp);
            mpml_face(NXp, n2, 1, [&](int a, int b, float* c) { cell(-P + 1 + a, ny, z1 + b, c); },
                      fB + (size_t)zoff * NXp, NXp);
            mpml_face(NXp, NYp, 2, [&](int a, int b, float* c) { cell(-P + 1 + a, -P + 1 + b, 1, c); }, fT, NXp);
            mpml_face(NXp, NYp, 2, [&](int a, int b, float* c) { cell(-P + 1 + a, -P + 1 + b, nz, c); }, fO, NXp);
        }
        mpml = std::any_of(h_faces.begin(), h_faces.end(), [](float v) { return v != 0.f; });
        // storage layout: x faces [z][y] (NYs), y faces [z][x], z faces [y][x] (pitch)
        const size_t sx = (size_t)NZs * NYs, sy = (size_t)NZs * pitch, sz = (size_t)NYs * pitch;
        std::vector<float> hf(2 * (sx + sy + sz), 0.f);
        for (int k = 0; k < NZp; ++k)
            for (int j = 0; j < NYp; ++j) {
                hf[(size_t)(k + R) * NYs + (j + R)] = fL[(size_t)k * NYp + j];
                hf[sx + (size_t)(k + R) * NYs + (j + R)] = fR[(size_t)k * NYp + j];
            }
        for (int k = 0; k < NZp; ++k)
            for (int i = 0; i < NXp; ++i) {
                hf[2 * sx + (size_t)(k + R) * pitch + (i + R)] = fF[(size_t)k * NXp + i];
                hf[2 * sx + sy + (size_t)(k + R) * pitch + (i + R)] = fB[(size_t)k * NXp + i];
            }
        for (int j = 0; j < NYp; ++j)
            for (int i = 0; i < NXp; ++i) {
                hf[2 * sx + 2 * sy + (size_t)(j + R) * pitch + (i + R)] = fT[(size_t)j * NXp + i];
                hf[2 * sx + 2 * sy + sz + (size_t)(j + R) * pitch + (i + R)] = fO[(size_t)j * NXp + i];
            }
        mp_prof.upload(prof.data(), prof.size(), stream);
        mp_face.upload(hf.data(), hf.size(), stream);
        // the per-node (a, b) of every shell derivative, once per model: the
        // per-cell kernels load them instead of recomputing 18 damping
        // coefficients (two divisions each) every step
        if (!mpml) {
            mp_coef.release();
            return;
        }
        mp_coef.reserve(36 * (size_t)fs);
        const El3dDev a = dev(1);
        const dim3 b(32, 8), g((a.x1 - a.x0 + 31) / 32, (a.y1 - a.y0 + 7) / 8, a.z1 - a.z0);
        k_el3d_mpml_coef<<<g, b, 0, stream>>>(a, mp_coef.p);
        OWL_LAUNCH_CHECK();
    }
    E3Mp mp_view() const {
        E3Mp m{};
        const int len[3] = {pitch, NYs, NZs};
        size_t off = 0;
        for (int ax = 0; ax < 3; ++ax) {
            m.d[ax][0] = mp_prof.p + off;
            m.d[ax][1] = mp_prof.p + off + len[ax];
            m.al[ax][0] = mp_prof.p + off + 2 * (size_t)len[ax];
            m.al[ax][1] = mp_prof.p + off + 3 * (size_t)len[ax];
            off += 4 * (size_t)len[ax];
        }
        const size_t sx = (size_t)NZs * NYs, sy = (size_t)NZs * pitch, sz = (size_t)NYs * pitch;
        m.face[0] = mp_face.p;
        m.face[1] = mp_face.p + sx;
        m.face[2] = mp_face.p + 2 * sx;
        m.face[3] = mp_face.p + 2 * sx + sy;
        m.face[4] = mp_face.p + 2 * sx + 2 * sy;
        m.face[5] = mp_face.p + 2 * sx + 2 * sy + sz;
        m.adt = std::fabs(dt);
        m.coef = mp_coef.p;
        return m;
    }

    explicit El3dEngine(const owl_ssg_desc& d) : El3dEngine(d, checked_vmesh3(d)) {}
    El3dEngine(const owl_ssg_desc& d, VMesh m) : SsgBase(with_rows3(d, m.nz), 3), vm(std::move(m)), nz_model(d.nz) {
        aniso = d.aniso;
        OWL_CHECK(aniso == OWL_ANISO_ISO || aniso == OWL_ANISO_CIJ || aniso == OWL_ANISO_THOMSEN, OWL_ERR_UNSUPPORTED,
                  "elastic 3D takes the iso (vp, vs, rho), thomsen (vp, vs, epsilon, delta, gamma, theta, phi, rho) "
                  "or cij (nine moduli, rho) parameterisation");
        idx = (float)(1.0 / (double)d.dx);
        idy = (float)(1.0 / (double)d.dy);
        idz = (float)(1.0 / (double)d.dz);
        OWL_CUDA(cudaMemcpyToSymbol(c_fd3e, fd_coefs(R), sizeof(float) * R));
        sst = E3_NST * fs;  // fs is a multiple of 32 floats (pitch rounded to 32)
        sad = E3_NAD * fs;
        nS = 9;
        ngrad = 12;
        nparam = el3d_nparam(aniso);
        ncomp = 3;
        for (int f = 0; f < E3_NST; ++f) st_segments.push_back({f * fs, fs});
        // dz scalings of the storage planes (1 outside the mesh arrays and on the uniform grid)
        std::vector<float> hi(NZs, 1.f), hh(NZs, 1.f);
        if (vm.refined) {
            for (int z = 0; z < NZs; ++z) {
                const int k = z - pr + 1;
                if (k < -P || k > nz + P + 1) continue;
                hi[z] = vm.get(vm.si, k);
                hh[z] = vm.get(vm.sh, k);
            }
            zt = build_zinterp(vm, nz_model, d.dz);
            // transpose of the depth interpolation, per regular padded plane
            std::vector<std::vector<std::pair<int, double>>> by((size_t)nz_model + 2 * P + 2);
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

    // refined mesh: gpad holds the mesh cells' d J / d (c11 .. c66, rho)
    int grad_planes() const override { return vm.refined ? 10 : nparam; }

    float* st_field(int f) const override { return f < 9 ? st.p + f * fs : nullptr; }
    float* ad_field(int f) const override { return f < 9 ? ad.p + f * fs : nullptr; }
    int rho_param() const override { return vm.refined ? 9 : nparam - 1; }
    std::vector<int> tune_spt(int) const override { return {1, 2, 4}; }
    // forward pass: 2 = thread per cell (2 planes per block), 1 = the z-marching
    // ring kernels (half-width 4, no free surface)
    // (the adjoint pass likewise, with the ring adjoint kernels)
    std::vector<int> tune_tz(int) const override {
        if (ring_ok()) return {2, 1};
        return {2};
    }
    // the ring kernels: half-width 4, no free surface (M-PML ratios: the per-node
    // coefficient table on the shell nodes)
    bool ring_ok() const { return R == 4 && !desc.free_surface; }
    // tile_z = 1 asks for the ring kernels of both passes (where they apply), anything else the per-cell ones
    void launch_params(const owl_run_opts& o) override {
        tile_x = 32;
        tz_f = (o.tile_z == 1 && ring_ok()) ? 1 : 2;
        tz_a = tz_f;
    }

    void set_model(int np, const float* const* f) override {
        OWL_CHECK(np == nparam && f, OWL_ERR_INVALID,
                  "elastic 3D model needs " + std::to_string(nparam) + " parameters for this parameterisation");
        for (int q = 0; q < np; ++q) OWL_CHECK(f[q], OWL_ERR_INVALID, "null model parameter");
        std::vector<float> hc[10];
        for (auto& v : hc) v.assign(fs, 0.f);
        std::vector<float> hp0, hp1, htp;
        if (aniso == OWL_ANISO_ISO) { hp0.assign(fs, 0.f); hp1.assign(fs, 0.f); }
        if (aniso == OWL_ANISO_THOMSEN) htp.assign((size_t)8 * fs, 0.f);
        const int nzr = nz_model;
        auto regular = [&](int i, int j, int k, float* v, float* pp) {
            const int ii = std::min(std::max(i, 1), nx), jj = std::min(std::max(j, 1), ny),
                      kk = std::min(std::max(k, 1), nzr);
            const size_t src = ((size_t)(ii - 1) * ny + (jj - 1)) * nzr + (kk - 1);
            e3_cell_cij(aniso, f, src, v, pp);
            for (int q = 0; q < 10; ++q) OWL_CHECK(std::isfinite(v[q]), OWL_ERR_INVALID, "non-finite model value");
            OWL_CHECK(v[9] > 0 && v[0] > 0 && v[3] > 0 && v[5] > 0 && v[6] > 0 && v[7] > 0 && v[8] > 0,
                      OWL_ERR_INVALID, "rho, c11, c22, c33, c44, c55, c66 must be positive");
        };
        // pmlvp over the six faces of the regular model (module_vars.f90:384-406)
        float pv = -1e30f;
        auto face = [&](int i, int j, int k, const float* v) {
            if (i == 1 || i == nx || j == 1 || j == ny || k == 1 || k == nzr)
                for (int q : {0, 3, 5}) pv = std::max(pv, v[q] / v[9]);
        };
        if (!vm.refined) {
            // Cij of the padded model (module_vars.f90:278-296, 362-375; padding by pml+1, :409-418)
            for (int k = -P; k <= nz + P + 1; ++k)
                for (int j = -P; j <= ny + P + 1; ++j)
                    for (int i = -P; i <= nx + P + 1; ++i) {
                        const long long o = soff(i, j, k);
                        float v[10], pp[10];
                        regular(i, j, k, v, pp);
                        if (aniso == OWL_ANISO_ISO) { hp0[o] = pp[0]; hp1[o] = pp[1]; }
                        if (aniso == OWL_ANISO_THOMSEN)
                            for (int q = 0; q < 8; ++q) htp[(size_t)q * fs + o] = pp[q];
                        for (int q = 0; q < 10; ++q) hc[q][o] = v[q];
                        if (i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nzr) face(i, j, k, v);
                    }
        } else {
            // per (x, y) column: the regular padded column's Cij, interpolated
            // linearly to the mesh planes (map_regular_to_irregular,
            // module_vars.f90:164-180 of the 3D solver); the parameters of the
            // regular cells for the chain rule
            const int nq = nzr + 2 * P + 2, npj = aniso == OWL_ANISO_ISO ? 3 : aniso == OWL_ANISO_THOMSEN ? 8 : 0;
            const size_t npr = (size_t)nxq() * nyq() * nq;
            std::vector<float> hj((size_t)npj * npr, 0.f), col((size_t)10 * nq);
            for (int j = -P; j <= ny + P + 1; ++j)
                for (int i = -P; i <= nx + P + 1; ++i) {
                    for (int k = -P; k <= nzr + P + 1; ++k) {
                        float v[10], pp[10];
                        regular(i, j, k, v, pp);
                        for (int q = 0; q < 10; ++q) col[(size_t)q * nq + (k + P)] = v[q];
                        const size_t cell = ((size_t)(k + P) * nyq() + (j + P)) * nxq() + (i + P);
                        for (int q = 0; q < npj; ++q) hj[(size_t)q * npr + cell] = pp[q];
                        if (i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nzr) face(i, j, k, v);
                    }
                    for (int k = -P; k <= nz + P + 1; ++k) {
                        const int r0 = zt.r0[(size_t)(k + P)];
                        const long long o = soff(i, j, k);
                        for (int q = 0; q < 10; ++q)
                            hc[q][o] = zinterp_apply(zt, k, P, col[(size_t)q * nq + (r0 + P)],
                                                     col[(size_t)q * nq + (r0 + 1 + P)]);
                    }
                }
            if (npj) jparp.upload(hj.data(), hj.size(), stream);
        }
        // harmonic shear moduli and buoyancies (module_wavefield.f90:30-38)
        std::vector<float> h44(fs, 0.f), h55(fs, 0.f), h66(fs, 0.f), hbx(fs, 0.f), hby(fs, 0.f), hbz(fs, 0.f);
        const std::vector<float>& r = hc[9];
        for (int k = -P + 1; k <= nz + P; ++k)
            for (int j = -P + 1; j <= ny + P; ++j)
                for (int i = -P + 1; i <= nx + P; ++i) {
                    const long long o = soff(i, j, k);
                    h44[o] = 4.0f / (1.0f / hc[6][soff(i, j - 1, k - 1)] + 1.0f / hc[6][soff(i, j, k - 1)] +
                                     1.0f / hc[6][soff(i, j - 1, k)] + 1.0f / hc[6][o]);
                    h55[o] = 4.0f / (1.0f / hc[7][soff(i - 1, j, k - 1)] + 1.0f / hc[7][soff(i, j, k - 1)] +
                                     1.0f / hc[7][soff(i - 1, j, k)] + 1.0f / hc[7][o]);
                    h66[o] = 4.0f / (1.0f / hc[8][soff(i - 1, j - 1, k)] + 1.0f / hc[8][soff(i, j - 1, k)] +
                                     1.0f / hc[8][soff(i - 1, j, k)] + 1.0f / hc[8][o]);
                    hbx[o] = dt / (0.5f * (r[soff(i - 1, j, k)] + r[o]));
                    hby[o] = dt / (0.5f * (r[soff(i, j - 1, k)] + r[o]));
                    hbz[o] = dt / (0.5f * (r[soff(i, j, k - 1)] + r[o]));
                }
        // dt_stable (module_vars.f90:500-537; on the refined mesh the least over
        // the cells, each with its plane's smaller spacing)
        const float pmlvp = std::sqrt(pv);
        const float* cf = fd_coefs(R);
        float temp = 0.f;
        for (int q = 0; q < R; ++q) temp += std::fabs(cf[q]);
        if (!vm.refined) {
            float maxv = 0.f;
            for (int k = 1; k <= nz; ++k)
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const long long o = soff(i, j, k);
                        for (int q : {0, 3, 5}) maxv = std::max(maxv, std::sqrt(hc[q][o] / r[o]));
                    }
            dt_stable_ = 1.0f / (temp * maxv * std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (desc.dy * desc.dy) +
                                                         1.0f / (desc.dz * desc.dz)));
        } else {
            float best = 3.0e38f;
            for (int k = 1; k <= nz; ++k) {
                const float hz = std::min(vm.get(vm.dzi, k), vm.get(vm.dzh, k));
                const float g = std::sqrt(1.0f / (desc.dx * desc.dx) + 1.0f / (desc.dy * desc.dy) + 1.0f / (hz * hz));
                for (int j = 1; j <= ny; ++j)
                    for (int i = 1; i <= nx; ++i) {
                        const long long o = soff(i, j, k);
                        const float mv = std::max({std::sqrt(hc[0][o] / r[o]), std::sqrt(hc[3][o] / r[o]),
                                                   std::sqrt(hc[5][o] / r[o])});
                        best = std::min(best, 1.0f / (temp * mv * g));
                    }
            }
            dt_stable_ = best;
        }
        if (dt > dt_stable_ && !desc.allow_dt_adjust)
            throw OwlError(OWL_ERR_UNSTABLE, "dt = " + std::to_string(dt) + " exceeds the stable dt " +
                                                 std::to_string(dt_stable_));
        const float alphamax = (float)(1.0 * (double)desc.f0_max * 3.14159265358979323846);
        std::vector<float> tx, ty, tz;
        e3_axis(nx, P, R, pitch, desc.dx, dt, pmlvp, alphamax, tx);
        e3_axis(ny, P, R, NYs, desc.dy, dt, pmlvp, alphamax, ty);
        e3_axis(nz, P, R, NZs, desc.dz, dt, pmlvp, alphamax, tz, desc.free_surface == 0, &vm);
        build_mpml(hc, pmlvp, alphamax);
        c11.upload(hc[0].data(), fs, stream); c12.upload(hc[1].data(), fs, stream); c13.upload(hc[2].data(), fs, stream);
        c22.upload(hc[3].data(), fs, stream); c23.upload(hc[4].data(), fs, stream); c33.upload(hc[5].data(), fs, stream);
        c44e.upload(h44.data(), fs, stream); c55e.upload(h55.data(), fs, stream); c66e.upload(h66.data(), fs, stream);
        bxp.upload(hbx.data(), fs, stream); byp.upload(hby.data(), fs, stream); bzp.upload(hbz.data(), fs, stream);
        c44p.upload(hc[6].data(), fs, stream); c55p.upload(hc[7].data(), fs, stream); c66p.upload(hc[8].data(), fs, stream);
        rhop.upload(r.data(), fs, stream);
        if (aniso == OWL_ANISO_ISO) { p0p.upload(hp0.data(), fs, stream); p1p.upload(hp1.data(), fs, stream); }
        if (aniso == OWL_ANISO_THOMSEN) tparp.upload(htp.data(), htp.size(), stream);
        tabx.upload(tx.data(), tx.size(), stream);
        taby.upload(ty.data(), ty.size(), stream);
        tabz.upload(tz.data(), tz.size(), stream);
        OWL_CUDA(cudaStreamSynchronize(stream));
        h_rhop = hc[9];
        model_set = true;
        invalidate_graphs();
    }

    // ---- sources / receivers (module_wavefield.f90:1095-1333, submodule_forward_modeling.f90:82-145)
    int src_ncomp(const owl_source& q) const override {
        OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION || q.mechanism == OWL_SRC_FORCE || q.mechanism == OWL_SRC_MT,
                  OWL_ERR_UNSUPPORTED, "unknown source mechanism");
        return q.mechanism == OWL_SRC_FORCE ? 3 : 1;
    }
    // with a free surface, no tap above row 2 (module_wavefield.f90:1147-1315)
    void src_taps(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rc, float& rv) const override {
        const size_t n0 = taps.size();
        src_taps_all(q, comp, taps, rc, rv);
        if (desc.free_surface)
            taps.erase(std::remove_if(taps.begin() + n0, taps.end(), [](const TapPt& t) { return t.k < 2; }), taps.end());
    }
    void src_taps_all(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rc, float& rv) const {
        const float* ix = q.interp_ix; const float* iy = q.interp_iy; const float* iz = q.interp_iz;
        const float* hx = q.interp_hx; const float* hy = q.interp_hy; const float* hz = q.interp_hz;
        if (q.mechanism == OWL_SRC_FORCE) {
            OWL_CHECK(in_wavefield(q.gx, q.gy, q.gz), OWL_ERR_INVALID, "force source outside the grid");
            rv = h_rhop[soff(q.gx, q.gy, q.gz)];
            rc = pad_index(q.gx, q.gy, q.gz);
            const float w0 = comp == 0 ? std::sin(q.polar) * std::cos(q.azimuth)
                           : comp == 1 ? std::sin(q.polar) * std::sin(q.azimuth) : std::cos(q.polar);
            for (int irz = -4; irz <= 4; ++irz)
                for (int iry = -4; iry <= 4; ++iry)
                    for (int irx = -4; irx <= 4; ++irx) {
                        const int a = irx + 4, b = iry + 4, c = irz + 4;
                        if (comp == 0) taps.push_back(TapPt{E3_VX, q.hx + irx, q.gy + iry, q.gz + irz, w0 / rv * hx[a] * iy[b] * iz[c]});
                        else if (comp == 1) taps.push_back(TapPt{E3_VY, q.gx + irx, q.hy + iry, q.gz + irz, w0 / rv * ix[a] * hy[b] * iz[c]});
                        else taps.push_back(TapPt{E3_VZ, q.gx + irx, q.gy + iry, q.hz + irz, w0 / rv * ix[a] * iy[b] * hz[c]});
                    }
            return;
        }
        const bool mt = q.mechanism == OWL_SRC_MT;
        // dz_s: the local spacing dz_i(gz) on the refined mesh (module_wavefield.f90:1107-1111)
        OWL_CHECK(!vm.refined || (q.gz >= -P && q.gz <= nz + P + 1), OWL_ERR_INVALID, "source outside the grid");
        const float dzs = vm.refined ? vm.get(vm.dzi, q.gz) : desc.dz;
        const float inv = 1.0f / (desc.dx * desc.dy * dzs);
        for (int irz = -4; irz <= 4; ++irz)
            for (int iry = -4; iry <= 4; ++iry)
                for (int irx = -4; irx <= 4; ++irx) {
                    const int a = irx + 4, b = iry + 4, c = irz + 4;
                    const float w = ix[a] * iy[b] * iz[c];
                    taps.push_back(TapPt{E3_XX, q.gx + irx, q.gy + iry, q.gz + irz, -inv * (mt ? q.mt[0] : 1.f) * w});
                    taps.push_back(TapPt{E3_YY, q.gx + irx, q.gy + iry, q.gz + irz, -inv * (mt ? q.mt[1] : 1.f) * w});
                    taps.push_back(TapPt{E3_ZZ, q.gx + irx, q.gy + iry, q.gz + irz, -inv * (mt ? q.mt[2] : 1.f) * w});
                    if (mt) {
                        taps.push_back(TapPt{E3_XY, q.hx + irx, q.hy + iry, q.gz + irz, -inv * q.mt[3] * hx[a] * hy[b] * iz[c]});
                        taps.push_back(TapPt{E3_XZ, q.hx + irx, q.gy + iry, q.hz + irz, -inv * q.mt[4] * hx[a] * iy[b] * hz[c]});
                        taps.push_back(TapPt{E3_YZ, q.gx + irx, q.hy + iry, q.hz + irz, -inv * q.mt[5] * ix[a] * hy[b] * hz[c]});
                    }
                }
    }
    // with a free surface the sampling reads the velocity images vx, vy (1-k) =
    // (1+k) and vz (2-k) = (1+k), k = 1..4 (submodule_forward_modeling.f90:66-82):
    // those taps go to the rows they copy; rows above the images hold zero
    void rec_taps(const owl_receiver& q, int comp, std::vector<TapPt>& taps) const override {
        const bool fsf = desc.free_surface != 0;
        // the staggered axis of the component uses the half-node weights; taps
        // with a zero factor are dropped here (the table keeps none of them),
        // which keeps a node-centred receiver at 8 taps instead of 9^3
        const float* fx = comp == 0 ? q.interp_hx : q.interp_ix;
        const float* fy = comp == 1 ? q.interp_hy : q.interp_iy;
        const float* fz = comp == 2 ? q.interp_hz : q.interp_iz;
        const int i0 = comp == 0 ? q.hx : q.gx, j0 = comp == 1 ? q.hy : q.gy, k0 = comp == 2 ? q.hz : q.gz;
        const int field = comp == 0 ? E3_VX : comp == 1 ? E3_VY : E3_VZ;
        for (int irz = -4; irz <= 4; ++irz) {
            if (fz[irz + 4] == 0.f) continue;
            for (int iry = -4; iry <= 4; ++iry) {
                if (fy[iry + 4] == 0.f) continue;
                for (int irx = -4; irx <= 4; ++irx) {
                    if (fx[irx + 4] == 0.f) continue;
                    TapPt t{field, i0 + irx, j0 + iry, k0 + irz, fx[irx + 4] * fy[iry + 4] * fz[irz + 4] * q.weight};
                    if (fsf) {
                        const int top = comp == 2 ? 1 : 0;  // last image row: vz images rows <= 1
                        if (t.k <= top) {
                            if (t.k < top - 3) continue;
                            t.k = top + 2 - t.k;  // vx, vy: 2 - k; vz: 3 - k
                        }
                    }
                    taps.push_back(t);
                }
            }
        }
    }

    El3dDev dev(int S) const {
        El3dDev a{};
        a.nx = nx; a.ny = ny; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch;
        a.plane = plane; a.fs = fs; a.sst = sst; a.sad = sad;
        a.x0 = R; a.x1 = R + NXp; a.y0 = R; a.y1 = R + NYp; a.z1 = R + NZp;
        a.fsurf = desc.free_surface != 0;
        a.z0 = a.fsurf ? pr : R;  // with a free surface nothing above row 1 is updated
        a.nzb = (a.z1 - a.z0 + 1) / 2;
        a.NYs = NYs;
        a.NZs = NZs;
        a.idx = idx; a.idy = idy; a.idz = idz; a.dt = dt;
        a.nshots = S;
        a.c11 = c11.p; a.c12 = c12.p; a.c13 = c13.p; a.c22 = c22.p; a.c23 = c23.p; a.c33 = c33.p;
        a.c44e = c44e.p; a.c55e = c55e.p; a.c66e = c66e.p; a.bx = bxp.p; a.by = byp.p; a.bz = bzp.p;
        a.axi = tabx.p; a.bxi = tabx.p + pitch; a.axh = tabx.p + 2 * pitch; a.bxh = tabx.p + 3 * pitch;
        a.ayi = taby.p; a.byi = taby.p + NYs; a.ayh = taby.p + 2 * NYs; a.byh = taby.p + 3 * NYs;
        a.azi = tabz.p; a.bzi = tabz.p + NZs; a.azh = tabz.p + 2 * NZs; a.bzh = tabz.p + 3 * NZs;
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
        a.mp = mp_view();
        return a;
    }

    template <int RR>
    void launch_r(int id, int S, bool store) {
        El3dDev a = dev(S);
        const bool FF = a.fsurf != 0;  // free-surface variants of the kernels
        const bool fwd = id == OWL_K_FWD_P || id == OWL_K_FWD_V;
        a.spt = fwd ? spt_f : spt_a;
        const int groups = (S + a.spt - 1) / a.spt;
        OWL_CHECK((long long)a.nzb * groups < 65536, OWL_ERR_UNSUPPORTED, "too many z blocks x shot groups");
        const dim3 b(32, 4, 2), g((NXp + 31) / 32, (NYp + 3) / 4, a.nzb * groups);
        const bool ring = (fwd ? tz_f : tz_a) == 1 && RR == 4 && !FF;
        if (ring) {
            OWL_CHECK(fwd ? (!store || a.S) : (a.ad && a.S && a.G), OWL_ERR_INVALID, "buffers not allocated");
            const int rows = a.z1 - a.z0;
            const long long xy = (long long)((NXp + 31) / 32) * ((NYp + 7) / 8);
            const long long want = std::max<long long>(1, (148LL * 64 + xy - 1) / xy);
            a.zchunk = (int)std::max<long long>(16, (rows + want - 1) / want);
            const int nzc = (rows + a.zchunk - 1) / a.zchunk;
            OWL_CHECK((long long)nzc * groups < 65536, OWL_ERR_UNSUPPORTED, "too many z chunks x shot groups");
            const dim3 br(32, 8), gr((NXp + 31) / 32, (NYp + 7) / 8, nzc * groups);
            if (mpml) launch_ring<true>(id, store, a, gr, br);
            else launch_ring<false>(id, store, a, gr, br);
            return;
        }
        if (fwd) OWL_CHECK(!store || a.S, OWL_ERR_INVALID, "stencil-term buffer not allocated");
        else OWL_CHECK(a.ad && a.S && a.G, OWL_ERR_INVALID, "adjoint buffers not allocated");
        if (mpml) launch_cell<RR, true>(id, store, FF, a, g, b);
        else launch_cell<RR, false>(id, store, FF, a, g, b);
    }
    int step_launches(int kind) const override {
        if (kind != 2) return SsgBase::step_launches(kind);
        return 2 + (want_src_now ? 1 : 0) + (nb_sct <= 4 ? 1 : 2);
    }
    // the z-marching ring kernels (half-width 4); MP: M-PML coefficients per shell node
    template <bool MP>
    void launch_ring(int id, bool store, const El3dDev& a, dim3 gr, dim3 br) {
        if (id == OWL_K_ADJ_P) {
            constexpr int sm = e3ra_bytes_v<4>();
            OWL_CUDA(cudaFuncSetAttribute(k_el3d_adj_v_ring<4, MP>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k_el3d_adj_v_ring<4, MP><<<gr, br, sm, stream>>>(a);
        } else if (id == OWL_K_ADJ_V) {
            constexpr int sm = e3ra_bytes_s<4>();
            OWL_CUDA(cudaFuncSetAttribute(k_el3d_adj_s_ring<4, MP>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k_el3d_adj_s_ring<4, MP><<<gr, br, sm, stream>>>(a);
        } else if (id == OWL_K_FWD_P) {
            constexpr int sm = e3r_bytes_s<4>();
            auto k = store ? k_el3d_fwd_s_ring<4, true, MP> : k_el3d_fwd_s_ring<4, false, MP>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<gr, br, sm, stream>>>(a);
        } else {
            constexpr int sm = e3r_bytes_v<4>();
            auto k = store ? k_el3d_fwd_v_ring<4, true, MP> : k_el3d_fwd_v_ring<4, false, MP>;
            OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            k<<<gr, br, sm, stream>>>(a);
        }
    }
    // the per-cell kernels; MP: M-PML coefficients per shell node
    template <int RR, bool MP>
    void launch_cell(int id, bool store, bool FF, const El3dDev& a, dim3 g, dim3 b) {
        if (id == OWL_K_FWD_P) {
            auto k = store ? (FF ? k_el3d_fwd_s<RR, true, true, MP> : k_el3d_fwd_s<RR, true, false, MP>)
                           : (FF ? k_el3d_fwd_s<RR, false, true, MP> : k_el3d_fwd_s<RR, false, false, MP>);
            k<<<g, b, 0, stream>>>(a);
        } else if (id == OWL_K_FWD_V) {
            auto k = store ? (FF ? k_el3d_fwd_v<RR, true, true, MP> : k_el3d_fwd_v<RR, true, false, MP>)
                           : (FF ? k_el3d_fwd_v<RR, false, true, MP> : k_el3d_fwd_v<RR, false, false, MP>);
            k<<<g, b, 0, stream>>>(a);
        } else if (id == OWL_K_ADJ_P) {
            (FF ? k_el3d_adj_v<RR, true, MP> : k_el3d_adj_v<RR, false, MP>)<<<g, b, 0, stream>>>(a);
        } else {
            (FF ? k_el3d_adj_s<RR, true, MP> : k_el3d_adj_s<RR, false, MP>)<<<g, b, 0, stream>>>(a);
        }
    }
    void launch_kernel(int id, int S, bool store) override {
        if (R == 4) launch_r<4>(id, S, store);
        else launch_r<8>(id, S, store);
    }

    // the adjoint of a step: velocity nodes, source adjoint (optional), stress
    // nodes, then the residual of the sampling of step t
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

    // compulsory bytes per launch (fields once per shot, materials once per
    // launch, memories and e terms once, Kahan sums once per shot group);
    // PML memory traffic is not counted (it is a fraction of the shell)
    int n_store_p() const override { return 6; }

    // CPML memories read and written per shot by the stress-node (q0 = 0) or
    // velocity-node (q0 = 9) kernels: a derivative along axis a carries one
    // where the node lies in the a-PML (per-axis CFS-PML) or anywhere in the
    // node's PML shell (M-PML: every derivative is damped there)
    double memory_cells(int q0) const {
        static const int node[18][4] = {
            {0, 0, 0, 0}, {1, 0, 0, 0}, {2, 0, 0, 0}, {1, 0, 1, 1}, {2, 0, 1, 1}, {0, 1, 0, 1}, {2, 1, 0, 1}, {0, 1, 1, 0},
            {1, 1, 1, 0}, {0, 1, 0, 0}, {1, 1, 0, 0}, {2, 1, 0, 0}, {0, 0, 1, 0}, {1, 0, 1, 0}, {2, 0, 1, 0}, {0, 0, 0, 1},
            {1, 0, 0, 1}, {2, 0, 0, 1}};
        const double full[3] = {(double)NXp, (double)NYp, (double)NZp};
        const bool fsf = desc.free_surface != 0;
        // shell cells along an axis: P on each side, one more on the low side at half positions
        auto out = [&](int ax, int h) { return (ax == 2 && fsf) ? (double)P : 2.0 * P + h; };
        double n = 0;
        for (int q = q0; q < q0 + 9; ++q) {
            const int ax = node[q][0];
            if (mpml) {
                double in = 1;
                for (int b = 0; b < 3; ++b) in *= full[b] - out(b, node[q][1 + b]);
                n += full[0] * full[1] * full[2] - in;
            } else {
                double f = out(ax, node[q][1 + ax]);
                for (int b = 0; b < 3; ++b)
                    if (b != ax) f *= full[b];
                n += f;
            }
        }
        return n;
    }
    double alg_bytes(int id, int S, int groups) const override {
        const double cells = (double)NXp * NYp * NZp;
        switch (id) {
            case OWL_K_FWD_P:
                return S * (cells * (3 * 4.0 + 6 * 8.0) + memory_cells(0) * 8.0) + cells * 9 * 4.0;
            case OWL_K_FWD_V:
                return S * (cells * (6 * 4.0 + 3 * 8.0) + memory_cells(9) * 8.0) + cells * 3 * 4.0;
            case OWL_K_ADJ_P:
                return S * (cells * (9 * 4.0 + 3 * 8.0 + 9 * 4.0 + 3 * 4.0) + memory_cells(9) * 8.0) + cells * 3 * 4.0 +
                       groups * cells * 3 * 16.0;
            case OWL_K_ADJ_V:
                return S * (cells * (9 * 4.0 + 6 * 8.0 + 9 * 4.0 + 6 * 4.0) + memory_cells(0) * 8.0) + cells * 9 * 4.0 +
                       groups * cells * 9 * 16.0;
        }
        return 0;
    }

    void chain_rule(int S, int groups) override {
        El3dDev a = dev(S);
        const long long n = (long long)nxq() * nyq() * nzq();
        const int nb = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
        // refined mesh: d J / d Cij of the mesh cells (the cij branch), mapped in fold_out
        const bool iso = aniso == OWL_ANISO_ISO && !vm.refined;
        k_el3d_chain<<<nb, 256, 0, stream>>>(a, groups, iso ? 1 : 0, iso ? p0p.p : nullptr, iso ? p1p.p : nullptr,
                                             aniso == OWL_ANISO_THOMSEN && !vm.refined ? tparp.p : nullptr, c44p.p,
                                             c55p.p, c66p.p, rhop.p, gpad.p, nxq(), nyq(), nzq());
        OWL_LAUNCH_CHECK();
        launches++;
    }

    // refined mesh: the mesh cells' d J / d Cij to the regular planes and the
    // model parameters (k_el3d_zmap), then the fold of the padding
    void fold_out(float* grad, int mem) override {
        if (!vm.refined) {
            SsgBase::fold_out(grad, mem);
            return;
        }
        const int nzq_r = nz_model + 2 * P + 2;
        const long long npr = (long long)nxq() * nyq() * nzq_r;
        gzmap.reserve((size_t)nparam * npr);
        const int nb = (int)std::min<long long>((npr + 255) / 256, 148LL * 16);
        k_el3d_zmap<<<nb, 256, 0, stream>>>(gpad.p, (long long)npad(), zptr.p, zrow.p, zw.p, aniso, jparp.p, npr,
                                            gzmap.p, nxq(), nyq());
        OWL_LAUNCH_CHECK();
        launches++;
        const size_t nm = (size_t)nx * ny * nz_model;
        seis_tmp.reserve((size_t)nparam * nm);
        for (int q = 0; q < nparam; ++q) {
            launch_fold(gzmap.p + (size_t)q * npr, nxq(), nyq(), P, nx, ny, nz_model, 3, seis_tmp.p + (size_t)q * nm,
                        stream);
            launches++;
        }
        copy_out(grad, seis_tmp.p, (size_t)nparam * nm * sizeof(float), mem);
    }
};

Engine* make_el3d_engine(const owl_ssg_desc& d) { return new El3dEngine(d); }

}  // namespace owl
