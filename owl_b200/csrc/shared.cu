// shared.cu -- kernels and host helpers used by every medium.
#include <algorithm>
#include <cmath>

#include "engine.cuh"

#include <cstdlib>

#include <cudaTypedefs.h>

#include "tma.cuh"

namespace owl {

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("OWL_NO_PDL");
        return !(e && e[0] == '1');
    }();
    return on;
}


int nint_f(float v) { return (int)std::lround(v); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda)
CUtensorMap make_tensor_map_f32(const float* base, int rank, const uint64_t* dims, const uint64_t* stride_bytes,
                                const uint32_t* box) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess) fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    OWL_CHECK(encode != nullptr, OWL_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    OWL_CHECK(rank >= 1 && rank <= 5 && ((uintptr_t)base % 16) == 0, OWL_ERR_INVALID, "tensor map base or rank");
    cuuint64_t gd[5], gs[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; ++i) {
        gd[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
        OWL_CHECK(box[i] >= 1 && box[i] <= 256, OWL_ERR_INVALID, "tensor map box extent");
    }
    OWL_CHECK((box[0] * 4) % 16 == 0, OWL_ERR_INVALID, "tensor map box row must be a multiple of 16 bytes");
    for (int i = 0; i + 1 < rank; ++i) {
        gs[i] = stride_bytes[i];
        OWL_CHECK(stride_bytes[i] % 16 == 0, OWL_ERR_INVALID, "tensor map strides must be multiples of 16 bytes");
    }
    CUtensorMap m;
    const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, const_cast<float*>(base), gd, gs,
                              bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    OWL_CHECK(r == CUDA_SUCCESS, OWL_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

void damp_coef(float bdvp, float d, float dist, int pml, float dt, float alphamax, float& a, float& b) {
    // npower_d = 2, npower_a = 1, kmax = 1, R0 = 1e-5 (module_cfspml.f90:27-30,68-70)
    const float R0 = 1.0e-5f, kmax = 1.0f;
    float nd = dist / ((float)pml * d);
    float alpha = std::max(alphamax * (1.0f - nd), 0.25f * alphamax);
    float damp = bdvp * (2.0f + 1.0f) * std::log(1.0f / R0) / (2.0f * (float)pml * d) * (nd * nd);
    float k = 1.0f + (kmax - 1.0f) * (nd * nd);
    float adt = std::fabs(dt);
    a = -2.0f * adt * damp / k / (2.0f + adt * (alpha + damp / k));
    b = (2.0f - adt * (alpha + damp / k)) / (2.0f + adt * (alpha + damp / k));
}

Pml1DHost build_pml_1d(int n, int pml, int R, int len, float d, float dt, float pmlvp, float alphamax) {
    Pml1DHost h;
    h.ai.assign(len, 0.f);
    h.bi.assign(len, 0.f);
    h.ah.assign(len, 0.f);
    h.bh.assign(len, 0.f);
    for (int i = -pml + 1; i <= n + pml; ++i) {
        float disti = 0.f, disth = 0.f;
        if (i <= 1) {
            disti = std::fabs((float)(i - 1) * d);
            disth = std::fabs(((float)(i - 1) - 0.5f) * d);
        } else if (i >= n + 1) {
            disti = std::fabs((float)(i - n) * d);
            disth = std::fabs(((float)(i - n) - 0.5f) * d);
        }
        if (i <= 1 || i >= n + 1) {
            int x = i + pml + R - 1;
            damp_coef(pmlvp, d, disti, pml, dt, alphamax, h.ai[x], h.bi[x]);
            damp_coef(pmlvp, d, disth, pml, dt, alphamax, h.ah[x], h.bh[x]);
        }
    }
    return h;
}

// ---------------------------------------------------------------------------
// record buffer [t][rtot]  <->  seismogram [rtot][t]
// ---------------------------------------------------------------------------
__global__ void k_transpose(const float* __restrict__ in, float* __restrict__ out, int rows, int cols) {
    // in: rows x cols, out: cols x rows
    __shared__ float tile[32][33];
    int c = blockIdx.x * 32 + threadIdx.x;
    for (int r = blockIdx.y * 32 + threadIdx.y; r < min(rows, (int)(blockIdx.y * 32 + 32)); r += 8)
        if (c < cols) tile[r - blockIdx.y * 32][threadIdx.x] = in[(size_t)r * cols + c];
    __syncthreads();
    int r2 = blockIdx.y * 32 + threadIdx.x;
    for (int c2 = blockIdx.x * 32 + threadIdx.y; c2 < min(cols, (int)(blockIdx.x * 32 + 32)); c2 += 8)
        if (r2 < rows) out[(size_t)c2 * rows + r2] = tile[threadIdx.x][c2 - blockIdx.x * 32];
}

static void launch_transpose(const float* in, float* out, int rows, int cols, cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return;
    dim3 b(32, 8), g((cols + 31) / 32, (rows + 31) / 32);
    k_transpose<<<g, b, 0, s>>>(in, out, rows, cols);
    OWL_LAUNCH_CHECK();
}

// Cubic-convolution resampling of trace rows (Keys' kernel, a = -1/2): output
// sample i of a row sits at t = oout + i dout, read from the input samples
// j0-1 .. j0+2 around x = (t - oin) / din (indices clamped to the row; x within
// 1e-4 of a node snaps to it), zero outside [0, nin - 1]. Linear in the data;
// exact on input nodes.
__global__ void k_resample_rows(const float* __restrict__ in, int nin, double din, double oin, float* __restrict__ out,
                                int nout, double dout, double oout, int ntr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nout) return;
    double x = (oout + (double)i * dout - oin) / din;
    // sampling intervals arrive in single precision: a position within 1e-4 of
    // an input node is that node (equal samplings copy, the last sample stays inside)
    if (fabs(x - rint(x)) <= 1.0e-4) x = rint(x);
    const bool inside = x >= 0.0 && x <= (double)(nin - 1);
    const int j0 = inside ? (int)floor(x) : 0;
    const float u = inside ? (float)(x - (double)j0) : 0.f;
    const float u2 = u * u, u3 = u2 * u;
    const float w0 = 0.5f * (-u3 + 2.f * u2 - u), w1 = 0.5f * (3.f * u3 - 5.f * u2 + 2.f);
    const float w2 = 0.5f * (-3.f * u3 + 4.f * u2 + u), w3 = 0.5f * (u3 - u2);
    const int ja = max(j0 - 1, 0), jb = j0, jc = min(j0 + 1, nin - 1), jd = min(j0 + 2, nin - 1);
    for (int r = blockIdx.y; r < ntr; r += gridDim.y) {
        const float* f = in + (size_t)r * nin;
        out[(size_t)r * nout + i] = inside ? w0 * f[ja] + w1 * f[jb] + w2 * f[jc] + w3 * f[jd] : 0.f;
    }
}

void launch_resample_rows(const float* in, int nin, double din, double oin, float* out, int nout, double dout,
                          double oout, int ntr, cudaStream_t s) {
    if (ntr <= 0 || nout <= 0) return;
    dim3 g((nout + 255) / 256, std::min(ntr, 65535));
    k_resample_rows<<<g, 256, 0, s>>>(in, nin, din, oin, out, nout, dout, oout, ntr);
    OWL_LAUNCH_CHECK();
}

void launch_transpose_rec_to_seis(const float* rec, float* seis, int nt, int rtot, cudaStream_t s) {
    launch_transpose(rec, seis, nt, rtot, s);
}
void launch_transpose_seis_to_rec(const float* seis, float* rec, int nt, int rtot, cudaStream_t s) {
    launch_transpose(seis, rec, rtot, nt, s);
}

// residual and misfit: one CTA per shot, fixed assignment -> deterministic
__global__ void k_residual_l2(const float* __restrict__ syn, const float* __restrict__ obs, float* __restrict__ res,
                              const unsigned char* __restrict__ live, const int* __restrict__ shot_rec_ptr, int nt,
                              int rtot, double* __restrict__ misfit) {
    int s = blockIdx.x;
    int r0 = shot_rec_ptr[s], r1 = shot_rec_ptr[s + 1];
    int nr = r1 - r0;
    double acc = 0.0;
    long long n = (long long)nr * nt;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) {
        int t = (int)(q / nr), r = r0 + (int)(q % nr);
        size_t o = (size_t)t * rtot + r;
        float rv = 0.f;
        if (live[r]) {
            rv = syn[o] - obs[o];
            double dd = (double)obs[o] - (double)syn[o];
            acc += dd * dd;
        }
        res[o] = rv;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && misfit) misfit[s] = red[0];
}

void launch_residual_l2(const float* syn, const float* obs, float* res, const unsigned char* live,
                        const int* shot_rec_ptr, int nshots, int nt, int rtot, double* misfit, cudaStream_t s) {
    if (nshots <= 0) return;
    k_residual_l2<<<nshots, 256, 0, s>>>(syn, obs, res, live, shot_rec_ptr, nt, rtot, misfit);
    OWL_LAUNCH_CHECK();
}

// per-trace L2 misfit sum_t (obs - syn)^2 in FP64: one warp per trace, a fixed
// lane / shuffle order (deterministic); traces of weight 0 give 0
__global__ void k_trace_misfit(const float* __restrict__ syn, const float* __restrict__ obs,
                               const unsigned char* __restrict__ live, int nt, int rtot, double* __restrict__ tm) {
    const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (r >= rtot) return;
    double acc = 0.0;
    if (live[r])
        for (int t = lane; t < nt; t += 32) {
            const double d = (double)obs[(size_t)t * rtot + r] - (double)syn[(size_t)t * rtot + r];
            acc += d * d;
        }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) tm[r] = acc;
}

// per-shot sums of the trace misfits, in trace order
__global__ void k_shot_misfit(const double* __restrict__ tm, const int* __restrict__ shot_rec_ptr, int nshots,
                              double* __restrict__ misfit) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nshots) return;
    double acc = 0.0;
    for (int r = shot_rec_ptr[s]; r < shot_rec_ptr[s + 1]; ++r) acc += tm[r];
    misfit[s] = acc;
}

void launch_shot_misfit(const double* trace_misfit, const int* shot_rec_ptr, int nshots, double* misfit,
                        cudaStream_t s) {
    if (nshots <= 0) return;
    k_shot_misfit<<<(nshots + 127) / 128, 128, 0, s>>>(trace_misfit, shot_rec_ptr, nshots, misfit);
    OWL_LAUNCH_CHECK();
}

void launch_trace_misfit(const float* syn, const float* obs, const unsigned char* live, const int* shot_rec_ptr,
                         int nshots, int nt, int rtot, double* trace_misfit, double* misfit, cudaStream_t s) {
    if (rtot > 0) {
        k_trace_misfit<<<(rtot + 7) / 8, 256, 0, s>>>(syn, obs, live, nt, rtot, trace_misfit);
        OWL_LAUNCH_CHECK();
    }
    if (nshots > 0) {
        k_shot_misfit<<<(nshots + 127) / 128, 128, 0, s>>>(trace_misfit, shot_rec_ptr, nshots, misfit);
        OWL_LAUNCH_CHECK();
    }
}

__global__ void k_check_finite(const float* __restrict__ f, size_t n, int* flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        bad |= !isfinite(f[i]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

void launch_check_finite(const float* f, size_t n, int* flag, cudaStream_t s) {
    if (!n) return;
    k_check_finite<<<148 * 4, 256, 0, s>>>(f, n, flag);
    OWL_LAUNCH_CHECK();
}

__global__ void k_fill_f64(double* p, size_t n, double v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
void launch_fill_f64(double* p, size_t n, double v, cudaStream_t s) {
    if (!n) return;
    k_fill_f64<<<148 * 2, 256, 0, s>>>(p, n, v);
    OWL_LAUNCH_CHECK();
}

}  // namespace owl
