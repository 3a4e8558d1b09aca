// noalloc.cu -- 2D acoustic forward modelling of one shot that allocates no
// device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// model a shot -- host applications whose device memory is owned by another
// allocator or reserved up front as a fixed budget (for instance a framework's
// caching allocator holding all of HBM, or a service with a fixed per-process
// device-memory quota), where one more cudaMalloc either fails or breaks the
// budget. The regular entry points (owl_ssg_create / owl_ssg_forward) allocate
// their buffers on the handle.
//
// How: every buffer of the run (padded materials, CFS-PML coefficients,
// wavefields, PML memory, trace buffer, source and receiver descriptions)
// lives in one file-scope static device array, g_noalloc_scratch, of
// OWL_NOALLOC_MAX_FLOATS floats. Every GPU that loads the library holds that
// array until the process exits. In host code the array's name is a host-side
// stand-in, not a device address, so its device address is looked up with
// cudaGetSymbolAddress once per device (with that device current) on the
// first call made on that device, and kept for the life of the process. Make
// that first call before any stream capture starts. A call made after
// cudaDeviceReset on that device is not supported: the kept address dates from
// before the reset. All calls share the array and it keeps the last call's
// contents: each call clears what must start at zero. Calls whose GPU work
// overlapped would race on the array; this entry point therefore holds a
// process-wide lock for the whole call and returns only after its GPU work has
// finished, so calls from several host threads run one after another.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace owl {

static __device__ __align__(256) float g_noalloc_scratch[OWL_NOALLOC_MAX_FLOATS];

namespace {

constexpr int NA_MAX_DEVICES = 64;
constexpr int NA_MAX_SOURCES = 16;
constexpr int NA_MAX_AXIS = 16384;

float* g_scratch_addr[NA_MAX_DEVICES] = {nullptr};
std::mutex g_call_mu;  // held for a whole call: the array and the host staging buffer below are shared
float g_pml_host[8 * NA_MAX_AXIS];

// device address of g_noalloc_scratch on the current device (looked up once per device)
float* scratch_on_current_device() {
    int dev = 0;
    OWL_CUDA(cudaGetDevice(&dev));
    OWL_CHECK(dev >= 0 && dev < NA_MAX_DEVICES, OWL_ERR_UNSUPPORTED, "device index beyond the no-alloc table");
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw OwlError(OWL_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    return g_scratch_addr[dev];
}

struct NaSrc {  // one explosion source as prepared by prepare_geometry / prepare_stf
    int gx, gz, nbeg, nt_stf;
    float amp;
    float ix[9], iz[9];
    long long stf_off;  // offset of its STF samples in the scratch array
};

struct NaRec {
    int gx, gz;
    float ix[9], iz[9];
    float weight;
};

struct NaDev {
    int nx, nz, P, R, pr, pitch, NZs, x0, x1, z0, z1, nt, nsrc, nrec;
    float dt, idx, idz;
    float *vp_in, *rho_in;  // (nz, nx) z fastest, copied from the caller
    float *dtbk, *dtbx, *dtbz, *pml;  // pml: axi, bxi, axh, bxh (pitch each), azi, bzi, azh, bzh (NZs each)
    float *p, *vx, *vz, *m1, *m2, *m3, *m4;
    float* rec;  // [t][r]
    float* seis; // [r][t]
    const NaSrc* src;
    const NaRec* recs;
    float* base;
};

__constant__ float c_fdna[8];

__device__ __forceinline__ long long na_off(const NaDev& a, int i, int j) {
    return (long long)(j + a.pr - 1) * a.pitch + (i + a.pr - 1);
}

// padded materials (edge replication by pml + 1) and cleared wavefields, in the
// operation order of the regular path's set_model
__global__ void k_na_setup(NaDev a, long long fs) {
    const long long n = fs;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        a.p[q] = 0.f; a.vx[q] = 0.f; a.vz[q] = 0.f;
        a.m1[q] = 0.f; a.m2[q] = 0.f; a.m3[q] = 0.f; a.m4[q] = 0.f;
        a.dtbk[q] = 0.f; a.dtbx[q] = 0.f; a.dtbz[q] = 0.f;
        const int x = (int)(q % a.pitch), z = (int)(q / a.pitch);
        const int i = x - a.pr + 1, j = z - a.pr + 1;
        auto rho_at = [&](int ii, int jj) {
            ii = min(max(ii, 1), a.nx);
            jj = min(max(jj, 1), a.nz);
            return a.rho_in[(long long)(ii - 1) * a.nz + (jj - 1)];
        };
        if (i >= -a.P && i <= a.nx + a.P + 1 && j >= -a.P && j <= a.nz + a.P + 1) {
            const int ii = min(max(i, 1), a.nx), jj = min(max(j, 1), a.nz);
            const float v = a.vp_in[(long long)(ii - 1) * a.nz + (jj - 1)];
            const float r = rho_at(i, j);
            a.dtbk[q] = a.dt * (r * v * v);
        }
        if (i >= -a.P + 1 && i <= a.nx + a.P && j >= -a.P + 1 && j <= a.nz + a.P) {
            const float re = 0.5f * (rho_at(i, j) + rho_at(i - 1, j));
            a.dtbx[q] = a.dt / re;
            const float rz = 0.5f * (rho_at(i, j) + rho_at(i, j - 1));
            a.dtbz[q] = a.dt / rz;
        }
    }
    const long long nr = (long long)a.nt * a.nrec;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nr; q += (long long)gridDim.x * blockDim.x)
        a.rec[q] = 0.f;
}

template <int R>
__global__ void k_na_fwd_p(NaDev a) {
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x, z = a.z0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const bool px = x < a.pr || x >= a.pr + a.nx, pz = z < a.pr || z >= a.pr + a.nz;
    float sx = 0.f, sz = 0.f;
#pragma unroll
    for (int k = 1; k <= R; ++k) sx = sx + c_fdna[k - 1] * (a.vx[o + k] - a.vx[o + 1 - k]);
#pragma unroll
    for (int k = 1; k <= R; ++k) sz = sz + c_fdna[k - 1] * (a.vz[o + (long long)k * a.pitch] - a.vz[o + (long long)(1 - k) * a.pitch]);
    float gx = a.idx * sx, gz = a.idz * sz;
    if (px) {
        float m = a.pml[x] * gx + a.pml[a.pitch + x] * a.m1[o];
        a.m1[o] = m;
        gx = gx + m;
    }
    if (pz) {
        const float* zc = a.pml + 4 * a.pitch;
        float m = zc[z] * gz + zc[a.NZs + z] * a.m2[o];
        a.m2[o] = m;
        gz = gz + m;
    }
    a.p[o] = a.p[o] - a.dtbk[o] * (gx + gz);
}

template <int R>
__global__ void k_na_fwd_v(NaDev a) {
    const int x = a.x0 + blockIdx.x * blockDim.x + threadIdx.x, z = a.z0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.x1 || z >= a.z1) return;
    const long long o = (long long)z * a.pitch + x;
    const bool px = x <= a.pr || x >= a.pr + a.nx, pz = z <= a.pr || z >= a.pr + a.nz;
    float sx = 0.f, sz = 0.f;
#pragma unroll
    for (int k = 1; k <= R; ++k) sx = sx + c_fdna[k - 1] * (a.p[o + k - 1] - a.p[o - k]);
#pragma unroll
    for (int k = 1; k <= R; ++k) sz = sz + c_fdna[k - 1] * (a.p[o + (long long)(k - 1) * a.pitch] - a.p[o - (long long)k * a.pitch]);
    float hx = a.idx * sx, hz = a.idz * sz;
    if (px) {
        float m = a.pml[2 * a.pitch + x] * hx + a.pml[3 * a.pitch + x] * a.m3[o];
        a.m3[o] = m;
        hx = hx + m;
    }
    if (pz) {
        const float* zc = a.pml + 4 * a.pitch;
        float m = zc[2 * a.NZs + z] * hz + zc[3 * a.NZs + z] * a.m4[o];
        a.m4[o] = m;
        hz = hz + m;
    }
    a.vx[o] = a.vx[o] - a.dtbx[o] * hx;
    a.vz[o] = a.vz[o] - a.dtbz[o] * hz;
}

// add_source(t) (sources in order, taps of one source in parallel), then the
// receivers of step tr (sequential sum over nonzero taps, z outer, x inner)
__global__ void k_na_point(NaDev a, int t, int tr) {
    if (t >= 1) {
        for (int k = 0; k < a.nsrc; ++k) {
            const NaSrc& q = a.src[k];
            if (t >= q.nbeg && t <= q.nbeg + q.nt_stf - 1) {
                const float A = a.base[q.stf_off + (t - q.nbeg)] * q.amp * a.dt;
                for (int e = threadIdx.x; e < 81; e += blockDim.x) {
                    const int irz = e / 9 - 4, irx = e % 9 - 4;
                    const float w = q.ix[irx + 4] * q.iz[irz + 4];
                    if (w != 0.f && A != 0.f) {
                        float* f = a.p + na_off(a, q.gx + irx, q.gz + irz);
                        *f = *f + A * w;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (tr >= 1 && tr <= a.nt) {
        for (int r = threadIdx.x; r < a.nrec; r += blockDim.x) {
            const NaRec& q = a.recs[r];
            float acc = 0.f;
            if (q.weight != 0.f) {
                for (int irz = -4; irz <= 4; ++irz)
                    for (int irx = -4; irx <= 4; ++irx) {
                        const float w = q.ix[irx + 4] * q.iz[irz + 4] * q.weight;
                        if (w != 0.f) acc = acc + a.p[na_off(a, q.gx + irx, q.gz + irz)] * w;
                    }
            }
            a.rec[(long long)(tr - 1) * a.nrec + r] = acc;
        }
    }
}

__global__ void k_na_transpose(NaDev a) {
    const long long n = (long long)a.nt * a.nrec;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q / a.nt), t = (int)(q % a.nt);
        a.seis[q] = a.rec[(long long)t * a.nrec + r];
    }
}

long long up64(long long v) { return (v + 63) / 64 * 64; }

}  // namespace

void forward_noalloc(const owl_ssg_desc* d, const float* vp, const float* rho, const owl_shot* shot, float* seis) {
    OWL_CHECK(d && vp && rho && shot && seis, OWL_ERR_INVALID, "null argument");
    OWL_CHECK(d->medium == OWL_ACOUSTIC_ISO_2D, OWL_ERR_UNSUPPORTED, "the no-alloc forward is 2D acoustic only");
    OWL_CHECK(!d->free_surface, OWL_ERR_UNSUPPORTED, "the no-alloc forward has no free surface");
    OWL_CHECK(d->fdhalf == 4 || d->fdhalf == 8, OWL_ERR_INVALID, "fdhalf must be 4 or 8");
    OWL_CHECK(d->nx >= 8 && d->nz >= 8 && d->pml >= 1 && d->nt >= 1 && d->dt > 0 && d->dx > 0 && d->dz > 0,
              OWL_ERR_INVALID, "bad grid or time axis");
    OWL_CHECK(shot->nsrc >= 0 && shot->nsrc <= NA_MAX_SOURCES && shot->nrec >= 0 && (shot->nsrc == 0 || shot->src) &&
                  (shot->nrec == 0 || shot->rec),
              OWL_ERR_INVALID, "the no-alloc forward takes at most 16 sources and a receiver array");
    const int nx = d->nx, nz = d->nz, P = d->pml, R = d->fdhalf, pr = P + R;
    const int NXs = nx + 2 * P + 2 * R, NZs = nz + 2 * P + 2 * R;
    const int pitch = (NXs + 31) / 32 * 32;
    OWL_CHECK(pitch <= NA_MAX_AXIS && NZs <= NA_MAX_AXIS, OWL_ERR_INVALID, "grid axis beyond the no-alloc limit");
    const long long fs = (long long)pitch * NZs, nm = (long long)nx * nz;
    long long stf_total = 0;
    for (int k = 0; k < shot->nsrc; ++k) {
        const owl_source& q = shot->src[k];
        OWL_CHECK(q.mechanism == OWL_SRC_EXPLOSION, OWL_ERR_UNSUPPORTED, "the no-alloc forward takes explosion sources");
        OWL_CHECK(q.nt_stf >= 0 && (q.nt_stf == 0 || q.stf), OWL_ERR_INVALID, "bad source STF");
        OWL_CHECK(q.gx - 4 >= -P - R + 1 && q.gx + 4 <= nx + P + R && q.gz - 4 >= -P - R + 1 && q.gz + 4 <= nz + P + R,
                  OWL_ERR_INVALID, "source taps outside the padded grid");
        stf_total += up64(q.nt_stf);
    }
    for (int r = 0; r < shot->nrec; ++r) {
        const owl_receiver& q = shot->rec[r];
        OWL_CHECK(q.weight == 0.f || (q.gx - 4 >= -P - R + 1 && q.gx + 4 <= nx + P + R && q.gz - 4 >= -P - R + 1 &&
                                      q.gz + 4 <= nz + P + R),
                  OWL_ERR_INVALID, "receiver taps outside the padded grid");
    }
    // scratch layout (floats, 64-aligned pieces)
    const long long n_src_f = up64(NA_MAX_SOURCES * (long long)sizeof(NaSrc) / 4 + 1);
    const long long n_rec_f = up64((long long)shot->nrec * sizeof(NaRec) / 4 + 1);
    const long long n_trace = up64((long long)d->nt * shot->nrec);
    long long off = 0;
    const long long o_vp = off; off += up64(nm);
    const long long o_rho = off; off += up64(nm);
    const long long o_mat = off; off += 3 * fs;
    const long long o_pml = off; off += up64(4LL * pitch + 4LL * NZs);
    const long long o_st = off; off += 7 * fs;
    const long long o_rec = off; off += n_trace;
    const long long o_seis = off; off += n_trace;
    const long long o_src = off; off += n_src_f;
    const long long o_recs = off; off += n_rec_f;
    const long long o_stf = off; off += stf_total;
    if (off > (long long)OWL_NOALLOC_MAX_FLOATS)
        throw OwlError(OWL_ERR_INVALID, "the run needs " + std::to_string(off) + " floats of scratch, more than the " +
                                            std::to_string((long long)OWL_NOALLOC_MAX_FLOATS) +
                                            " of the no-alloc array (OWL_NOALLOC_MAX_FLOATS)");
    std::lock_guard<std::mutex> lk(g_call_mu);
    float* base = scratch_on_current_device();

    // models and stability as in set_model (module_vars.f90:121-125)
    float maxv = -1e30f;
    for (long long q = 0; q < nm; ++q) {
        OWL_CHECK(std::isfinite(vp[q]) && std::isfinite(rho[q]) && vp[q] > 0 && rho[q] > 0, OWL_ERR_INVALID,
                  "vp and rho must be finite and positive");
        maxv = std::max(maxv, vp[q]);
    }
    {
        const float* c = fd_coefs(R);
        float temp = 0.f;
        for (int k = 0; k < R; ++k) temp += std::fabs(c[k]);
        const float dts = 1.0f / (temp * maxv * std::sqrt(1.0f / (d->dx * d->dx) + 1.0f / (d->dz * d->dz)));
        OWL_CHECK(d->dt <= dts, OWL_ERR_UNSTABLE, "dt exceeds the stable dt " + std::to_string(dts));
    }
    // CFS-PML coefficients on the host (module_cfspml.f90:68-131), in the staging buffer
    float maxv_edge = -1e30f;
    for (int j = 1; j <= nz; ++j)
        maxv_edge = std::max({maxv_edge, vp[(long long)0 * nz + (j - 1)], vp[(long long)(nx - 1) * nz + (j - 1)]});
    for (int i = 1; i <= nx; ++i)
        maxv_edge = std::max({maxv_edge, vp[(long long)(i - 1) * nz + 0], vp[(long long)(i - 1) * nz + (nz - 1)]});
    const float alphamax = (float)(1.0 * (double)d->f0_max * 3.14159265358979323846);
    float* hp = g_pml_host;
    std::memset(hp, 0, sizeof(float) * (4 * pitch + 4 * NZs));
    auto fill = [&](int n, int len, float dd, float* outp) {
        for (int i = -P + 1; i <= n + P; ++i) {
            float disti = 0.f, disth = 0.f;
            if (i <= 1) {
                disti = std::fabs((float)(i - 1) * dd);
                disth = std::fabs(((float)(i - 1) - 0.5f) * dd);
            } else if (i >= n + 1) {
                disti = std::fabs((float)(i - n) * dd);
                disth = std::fabs(((float)(i - n) - 0.5f) * dd);
            }
            if (i <= 1 || i >= n + 1) {
                const int x = i + P + R - 1;
                damp_coef(maxv_edge, dd, disti, P, d->dt, alphamax, outp[x], outp[len + x]);
                damp_coef(maxv_edge, dd, disth, P, d->dt, alphamax, outp[2 * len + x], outp[3 * len + x]);
            }
        }
    };
    fill(nx, pitch, d->dx, hp);
    fill(nz, NZs, d->dz, hp + 4 * pitch);

    NaSrc hs[NA_MAX_SOURCES];
    std::memset(hs, 0, sizeof(hs));
    long long so = o_stf;
    for (int k = 0; k < shot->nsrc; ++k) {
        const owl_source& q = shot->src[k];
        hs[k].gx = q.gx; hs[k].gz = q.gz; hs[k].nbeg = q.nbeg; hs[k].nt_stf = q.nt_stf; hs[k].amp = q.amp;
        std::memcpy(hs[k].ix, q.interp_ix, sizeof(hs[k].ix));
        std::memcpy(hs[k].iz, q.interp_iz, sizeof(hs[k].iz));
        hs[k].stf_off = so;
        if (q.nt_stf) OWL_CUDA(cudaMemcpy(base + so, q.stf, sizeof(float) * q.nt_stf, cudaMemcpyHostToDevice));
        so += up64(q.nt_stf);
    }
    OWL_CUDA(cudaMemcpy(base + o_src, hs, sizeof(hs), cudaMemcpyHostToDevice));
    // receivers in chunks through a fixed stack buffer
    {
        NaRec chunk[256];
        for (int r0 = 0; r0 < shot->nrec; r0 += 256) {
            const int n = std::min(256, shot->nrec - r0);
            for (int r = 0; r < n; ++r) {
                const owl_receiver& q = shot->rec[r0 + r];
                chunk[r].gx = q.gx; chunk[r].gz = q.gz; chunk[r].weight = q.weight;
                std::memcpy(chunk[r].ix, q.interp_ix, sizeof(chunk[r].ix));
                std::memcpy(chunk[r].iz, q.interp_iz, sizeof(chunk[r].iz));
            }
            OWL_CUDA(cudaMemcpy(reinterpret_cast<char*>(base + o_recs) + (size_t)r0 * sizeof(NaRec), chunk,
                                sizeof(NaRec) * n, cudaMemcpyHostToDevice));
        }
    }
    OWL_CUDA(cudaMemcpy(base + o_vp, vp, sizeof(float) * nm, cudaMemcpyHostToDevice));
    OWL_CUDA(cudaMemcpy(base + o_rho, rho, sizeof(float) * nm, cudaMemcpyHostToDevice));
    OWL_CUDA(cudaMemcpy(base + o_pml, hp, sizeof(float) * (4 * pitch + 4 * NZs), cudaMemcpyHostToDevice));
    OWL_CUDA(cudaMemcpyToSymbol(c_fdna, fd_coefs(R), sizeof(float) * R));

    NaDev a{};
    a.nx = nx; a.nz = nz; a.P = P; a.R = R; a.pr = pr; a.pitch = pitch; a.NZs = NZs;
    a.x0 = R; a.x1 = R + nx + 2 * P; a.z0 = R; a.z1 = R + nz + 2 * P;
    a.nt = d->nt; a.nsrc = shot->nsrc; a.nrec = shot->nrec;
    a.dt = d->dt;
    a.idx = (float)(1.0 / (double)d->dx);
    a.idz = (float)(1.0 / (double)d->dz);
    a.vp_in = base + o_vp; a.rho_in = base + o_rho;
    a.dtbk = base + o_mat; a.dtbx = base + o_mat + fs; a.dtbz = base + o_mat + 2 * fs;
    a.pml = base + o_pml;
    a.p = base + o_st; a.vx = a.p + fs; a.vz = a.p + 2 * fs;
    a.m1 = a.p + 3 * fs; a.m2 = a.p + 4 * fs; a.m3 = a.p + 5 * fs; a.m4 = a.p + 6 * fs;
    a.rec = base + o_rec; a.seis = base + o_seis;
    a.src = reinterpret_cast<const NaSrc*>(base + o_src);
    a.recs = reinterpret_cast<const NaRec*>(base + o_recs);
    a.base = base;

    k_na_setup<<<148 * 4, 256>>>(a, fs);
    OWL_LAUNCH_CHECK();
    const dim3 b(32, 8), g((nx + 2 * P + 31) / 32, (nz + 2 * P + 7) / 8);
    k_na_point<<<1, 256>>>(a, 0, 1);
    for (int t = 1; t <= d->nt; ++t) {
        if (R == 4) {
            k_na_fwd_p<4><<<g, b>>>(a);
            k_na_fwd_v<4><<<g, b>>>(a);
        } else {
            k_na_fwd_p<8><<<g, b>>>(a);
            k_na_fwd_v<8><<<g, b>>>(a);
        }
        k_na_point<<<1, 256>>>(a, t, t + 1);
    }
    OWL_LAUNCH_CHECK();
    if (n_trace) {
        k_na_transpose<<<148 * 2, 256>>>(a);
        OWL_LAUNCH_CHECK();
        OWL_CUDA(cudaMemcpy(seis, base + o_seis, sizeof(float) * (size_t)d->nt * shot->nrec, cudaMemcpyDeviceToHost));
    }
    OWL_CUDA(cudaDeviceSynchronize());
}

}  // namespace owl

extern "C" int owl_ssg_forward_noalloc(const owl_ssg_desc* desc, int nparam, const float* const* fields,
                                       const owl_shot* shot, float* seis) {
    try {
        OWL_CHECK(nparam == 2 && fields && fields[0] && fields[1], OWL_ERR_INVALID, "acoustic model needs vp and rho");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            throw owl::OwlError(OWL_ERR_NO_DEVICE, "no CUDA device available");
        }
        owl::forward_noalloc(desc, fields[0], fields[1], shot, seis);
        return OWL_OK;
    } catch (const owl::OwlError& e) {
        owl::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        owl::set_last_error(e.what());
        return OWL_ERR_INVALID;
    }
}
