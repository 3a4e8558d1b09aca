// adjsrc.cu -- data-domain misfits and adjoint sources on the GPU.
//
// Replaces compute_adjsrc_waveform / _corr / _envelope / _phase / _adaptive
// (src/inverse/module_inversion_adjoint_source.f90:371-537, penalty
// xcorr_penalty :321-363) and the trace selection of compute_adjoint_source
// (:1038-1070). Traces are rows of nt samples; a gather (one shot's one
// component) is a contiguous run of rows.
//
//   k_trace_norms  one warp per trace: FP64 norms of obs and syn
//   k_gather_live  one thread per gather: the discard rule (weight 0, norm
//                  below threshold x the gather's largest, or a zero norm)
//   k_adjsrc       a persistent grid, one CTA per trace at a time: misfit (FP64
//                  block sums in a fixed order) and adjoint source
//   k_gather_sum   per-gather sums of the trace misfits, in trace order
//
// The transforms are length-N DFTs by Bluestein's algorithm (the trace times a
// chirp, an M-point radix-2 FFT in shared memory, the product with the
// precomputed spectrum of the conjugate chirp, an inverse M-point FFT, the
// chirp again), so any N -- the trace length for the Hilbert transform, a
// 2-3-5-smooth length for the adaptive misfit -- takes the same path. FLIT's
// helpers (hilbert, envelope, instant_phase, fft / ifft, taper, rescale,
// next_power_235) are restated from their usual definitions: the analytic
// signal from a length-n DFT, an unnormalised forward / 1/n inverse DFT, Hann
// ramps for taper.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "adjsrc.cuh"
#include "engine.cuh"  // launch_resample_rows

namespace owl {

int next_power_235(int n) {
    for (int m = std::max(1, n);; ++m) {
        int k = m;
        for (int p : {2, 3, 5})
            while (k % p == 0) k /= p;
        if (k == 1) return m;
    }
}

namespace {

constexpr int MAX_DFT_M = 16384;  // 128 KB of float2 work in shared memory

void host_fft(std::vector<std::complex<double>>& a) {
    const size_t M = a.size();
    for (size_t i = 1, j = 0; i < M; ++i) {
        size_t bit = M >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= M; len <<= 1) {
        const double ang = -2.0 * M_PI / (double)len;
        for (size_t i = 0; i < M; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const std::complex<double> w = std::polar(1.0, ang * (double)k);
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

struct DftDev {
    int N, M, logM;
    const float2* chirp;
    const float2* bf;
    const float2* tw;
};

DftDev dev(const DftTables& t) { return DftDev{t.N, t.M, t.logM, t.chirp.p, t.bf.p, t.tw.p}; }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// in-place radix-2 FFT (exp(-i ...)) of a[0..M) in shared memory, M = 2^logM >= 2
__device__ void fft_pow2(float2* a, int M, int logM, const float2* __restrict__ tw) {
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int i = tid; i < M; i += nth) {
        const int j = (int)(__brev((unsigned)i) >> (32 - logM));
        if (i < j) {
            const float2 t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    __syncthreads();
    for (int s = 1; s <= logM; ++s) {
        const int half = 1 << (s - 1), tstride = M >> s;
        for (int b = tid; b < M / 2; b += nth) {
            const int pos = b & (half - 1);
            const int i = ((b >> (s - 1)) << s) + pos, j = i + half;
            const float2 w = tw[pos * tstride];
            const float2 u = a[i], v = cmul(w, a[j]);
            a[i] = make_float2(u.x + v.x, u.y + v.y);
            a[j] = make_float2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

// length-N DFT of a[0..N) in place (a[0..M) is work); inverse: the 1/N-normalised
// inverse DFT, conj(DFT(conj x)) / N
__device__ void dft(float2* a, const DftDev& d, bool inverse) {
    const int tid = threadIdx.x, nth = blockDim.x;
    __syncthreads();
    for (int n = tid; n < d.M; n += nth) {
        float2 v = make_float2(0.f, 0.f);
        if (n < d.N) {
            v = a[n];
            if (inverse) v.y = -v.y;
            v = cmul(v, d.chirp[n]);
        }
        a[n] = v;
    }
    __syncthreads();
    fft_pow2(a, d.M, d.logM, d.tw);
    for (int k = tid; k < d.M; k += nth) {
        float2 v = cmul(a[k], d.bf[k]);
        v.y = -v.y;  // the inverse M-point FFT as conj(FFT(conj))
        a[k] = v;
    }
    __syncthreads();
    fft_pow2(a, d.M, d.logM, d.tw);
    const float sM = 1.f / (float)d.M, sN = 1.f / (float)d.N;
    for (int k = tid; k < d.N; k += nth) {
        float2 y = a[k];
        y = make_float2(y.x * sM, -y.y * sM);
        float2 X = cmul(d.chirp[k], y);
        if (inverse) X = make_float2(X.x * sN, -X.y * sN);
        a[k] = X;
    }
    __syncthreads();
}

// analytic signal of the real part of a[0..N): X[0] (and X[N/2], N even) kept,
// the positive frequencies doubled, the negative ones zeroed
__device__ void analytic(float2* a, const DftDev& d) {
    dft(a, d, false);
    const int N = d.N;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const float h = (k == 0 || (N % 2 == 0 && k == N / 2)) ? 1.f : (k < (N + 1) / 2 ? 2.f : 0.f);
        a[k] = make_float2(a[k].x * h, a[k].y * h);
    }
    dft(a, d, true);
}

// block reductions with a fixed summation order (every thread gets the result)
__device__ double block_sum(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    return t;
}

__device__ float block_max(float v, float* red) {
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = red[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) t = fmaxf(t, red[i]);
    return t;
}

__global__ void k_trace_norms(const float* __restrict__ syn, const float* __restrict__ obs, int nt, int ntr,
                              double* __restrict__ nrm) {
    const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (r >= ntr) return;
    double so = 0.0, ss = 0.0;
    for (int t = lane; t < nt; t += 32) {
        const double o = obs[(size_t)r * nt + t], s = syn[(size_t)r * nt + t];
        so += o * o;
        ss += s * s;
    }
    for (int o = 16; o; o >>= 1) {
        so += __shfl_xor_sync(0xffffffffu, so, o);
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if (lane == 0) {
        nrm[2 * r] = sqrt(so);
        nrm[2 * r + 1] = sqrt(ss);
    }
}

__global__ void k_gather_live(const int* __restrict__ gptr, int ngather, const double* __restrict__ nrm,
                              const unsigned char* __restrict__ wlive, double thr, unsigned char* __restrict__ live) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngather) return;
    double mo = 0.0, ms = 0.0;
    for (int r = gptr[g]; r < gptr[g + 1]; ++r) {
        mo = fmax(mo, nrm[2 * r]);
        ms = fmax(ms, nrm[2 * r + 1]);
    }
    for (int r = gptr[g]; r < gptr[g + 1]; ++r) {
        const double no = nrm[2 * r], ns = nrm[2 * r + 1];
        const bool w = wlive ? wlive[r] != 0 : true;
        live[r] = (w && !(no < thr * mo) && !(ns < thr * ms) && no * ns != 0.0) ? 1 : 0;
    }
}

__global__ void k_gather_sum(const double* __restrict__ tm, const int* __restrict__ gptr, int ngather,
                             double* __restrict__ gm) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngather) return;
    double acc = 0.0;
    for (int r = gptr[g]; r < gptr[g + 1]; ++r) acc += tm[r];
    gm[g] = acc;
}

__global__ void k_nonzero(const float* __restrict__ w, int n, unsigned char* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = w[i] != 0.f ? 1 : 0;
}

struct AdjArgs {
    int kind, nt, ntr;
    const float* syn;
    const float* obs;
    const unsigned char* live;
    float* adj;
    double* tm;
    DftDev hil, awi;
    const float* pen;   // adaptive: penalty per circular lag bin (awi.N)
    const float* ramp;  // Hann ramp of tl samples
    int tl;
    float deconv_eps;
    float* scratch;    // per CTA: 4 nt floats
    float2* cscratch;  // per CTA: awi.N complex
};

__device__ __forceinline__ float ramp_at(const AdjArgs& g, int i) { return i < g.tl ? g.ramp[i] : 1.f; }

__global__ void __launch_bounds__(256) k_adjsrc(AdjArgs g) {
    extern __shared__ float2 work[];
    __shared__ double redd[32];
    __shared__ float redf[32];
    const int tid = threadIdx.x, nth = blockDim.x, nt = g.nt;
    float* s1 = g.scratch + (size_t)blockIdx.x * 4 * nt;
    float* s2 = s1 + nt;
    float* s3 = s2 + nt;
    float* s4 = s3 + nt;
    float2* cd = g.cscratch + (size_t)blockIdx.x * g.awi.N;
    for (int r = blockIdx.x; r < g.ntr; r += gridDim.x) {
        const float* sy = g.syn + (size_t)r * nt;
        const float* ob = g.obs + (size_t)r * nt;
        float* ad = g.adj ? g.adj + (size_t)r * nt : nullptr;
        if (!g.live[r]) {
            if (ad)
                for (int t = tid; t < nt; t += nth) ad[t] = 0.f;
            if (tid == 0 && g.tm) g.tm[r] = 0.0;
            continue;
        }
        double m = 0.0;
        if (g.kind == OWL_MISFIT_WAVEFORM) {
            double acc = 0.0;
            for (int t = tid; t < nt; t += nth) {
                const double dd = (double)ob[t] - (double)sy[t];
                acc += dd * dd;
                if (ad) ad[t] = sy[t] - ob[t];
            }
            m = block_sum(acc, redd);
        } else if (g.kind == OWL_MISFIT_CORR) {
            double ss = 0.0, oo = 0.0, so = 0.0;
            float ms = 0.f, mo = 0.f;
            for (int t = tid; t < nt; t += nth) {
                const double s = sy[t], o = ob[t];
                ss += s * s;
                oo += o * o;
                so += s * o;
                ms = fmaxf(ms, fabsf(sy[t]));
                mo = fmaxf(mo, fabsf(ob[t]));
            }
            ss = block_sum(ss, redd);
            oo = block_sum(oo, redd);
            so = block_sum(so, redd);
            ms = block_max(ms, redf);
            mo = block_max(mo, redf);
            const double ns = sqrt(ss), no = sqrt(oo);
            double acc = 0.0;
            if (ms == 0.f && mo != 0.f) {
                for (int t = tid; t < nt; t += nth) {
                    const double v = (double)ob[t] / no;
                    acc += v * v;
                    if (ad) ad[t] = (float)(-v);
                }
            } else {
                for (int t = tid; t < nt; t += nth) {
                    const double v = (double)sy[t] / ns - (double)ob[t] / no;
                    acc += v * v;
                    if (ad) ad[t] = (float)((so / ss * (double)sy[t] - (double)ob[t]) / (no * ns));
                }
            }
            m = block_sum(acc, redd);
        } else if (g.kind == OWL_MISFIT_ENVELOPE || g.kind == OWL_MISFIT_PHASE) {
            const bool env = g.kind == OWL_MISFIT_ENVELOPE;
            for (int t = tid; t < nt; t += nth) work[t] = make_float2(ob[t], 0.f);
            analytic(work, g.hil);
            for (int t = tid; t < nt; t += nth) {
                const float2 z = work[t];
                s1[t] = env ? sqrtf(z.x * z.x + z.y * z.y) : atan2f(z.y, z.x);
            }
            __syncthreads();
            for (int t = tid; t < nt; t += nth) work[t] = make_float2(sy[t], 0.f);
            analytic(work, g.hil);
            double acc = 0.0;
            float mx = 0.f;
            for (int t = tid; t < nt; t += nth) {
                const float2 z = work[t];
                const float e2 = z.x * z.x + z.y * z.y;
                const float u = env ? sqrtf(e2) : atan2f(z.y, z.x);
                s2[t] = u;
                s3[t] = z.y;
                s4[t] = e2;
                const double dd = (double)s1[t] - (double)u;
                acc += dd * dd;
                mx = fmaxf(mx, env ? u : e2);
            }
            m = block_sum(acc, redd);
            mx = block_max(mx, redf);
            for (int t = tid; t < nt; t += nth) {
                float v;
                if (env) {
                    const float coef = mx == 0.f ? 0.f : (s2[t] - s1[t]) / (s2[t] + 1.0e-2f * mx);
                    s4[t] = coef;
                    v = s3[t] * coef;
                } else {
                    const float er = s4[t] + 5.0e-2f * mx;
                    s4[t] = er;
                    v = (s2[t] - s1[t]) * sy[t] / er;
                }
                work[t] = make_float2(v, 0.f);
            }
            analytic(work, g.hil);
            if (ad)
                for (int t = tid; t < nt; t += nth)
                    ad[t] = env ? sy[t] * s4[t] - work[t].y : -(s2[t] - s1[t]) * s3[t] / s4[t] + work[t].y;
        } else {  // OWL_MISFIT_ADAPTIVE
            const int N = g.awi.N;
            for (int k = tid; k < N; k += nth)
                work[k] = make_float2(k < nt ? ob[k] * ramp_at(g, k) * ramp_at(g, nt - 1 - k) : 0.f, 0.f);
            dft(work, g.awi, false);
            float mx = 0.f;
            for (int k = tid; k < N; k += nth) {
                const float2 D = work[k];
                cd[k] = D;
                mx = fmaxf(mx, D.x * D.x + D.y * D.y);
            }
            mx = block_max(mx, redf);
            const float eps = g.deconv_eps * mx;
            for (int k = tid; k < N; k += nth)
                work[k] = make_float2(k < nt ? sy[k] * ramp_at(g, k) * ramp_at(g, nt - 1 - k) : 0.f, 0.f);
            dft(work, g.awi, false);
            for (int k = tid; k < N; k += nth) {
                const float2 U = work[k], D = cd[k];
                const float q = 1.f / (D.x * D.x + D.y * D.y + eps);
                work[k] = make_float2((U.x * D.x + U.y * D.y) * q, (U.y * D.x - U.x * D.y) * q);
            }
            dft(work, g.awi, true);
            double sxx = 0.0, swx = 0.0;
            for (int k = tid; k < N; k += nth) {
                const double xc = work[k].x, wx = (double)g.pen[k] * xc;
                sxx += xc * xc;
                swx += wx * wx;
            }
            sxx = block_sum(sxx, redd);
            swx = block_sum(swx, redd);
            m = 0.5 * swx / sxx;
            for (int k = tid; k < N; k += nth) {
                const double w = g.pen[k];
                work[k] = make_float2((float)((w * w - 2.0 * m) * (double)work[k].x / sxx), 0.f);
            }
            dft(work, g.awi, false);
            for (int k = tid; k < N; k += nth) {
                const float2 G = work[k], D = cd[k];
                const float q = 1.f / (D.x * D.x + D.y * D.y + eps);
                work[k] = make_float2((G.x * D.x - G.y * D.y) * q, (G.x * D.y + G.y * D.x) * q);
            }
            dft(work, g.awi, true);
            if (ad)
                for (int t = tid; t < nt; t += nth) ad[t] = work[t].x * ramp_at(g, nt - 1 - t);
        }
        if (tid == 0 && g.tm) g.tm[r] = m;
        __syncthreads();
    }
}

// spectra products of the adaptive misfits: a conj(b) / (|b|^2 + eps) and a b / (|b|^2 + eps)
__device__ __forceinline__ float2 deconv_conj(float2 a, float2 b, float eps) {
    const float q = 1.f / (b.x * b.x + b.y * b.y + eps);
    return make_float2((a.x * b.x + a.y * b.y) * q, (a.y * b.x - a.x * b.y) * q);
}
__device__ __forceinline__ float2 deconv_mul(float2 a, float2 b, float eps) {
    const float q = 1.f / (b.x * b.x + b.y * b.y + eps);
    return make_float2((a.x * b.x - a.y * b.y) * q, (a.x * b.y + a.y * b.x) * q);
}

struct LocArgs {
    int nt, ntr, ngather, hw;
    const int* gptr;
    const float* syn;
    const float* obs;
    const unsigned char* live;
    float* adj;
    double* tm;
    DftDev dft;         // length next_power_235(2 nt) (local) or next_power_235(4 nt) (space-time)
    const float* pen;   // penalty per circular lag bin (dft.N)
    const float* ramp;  // Hann ramp of tl samples
    int tl;
    float deconv_eps, sigma;  // sigma: Gaussian window in samples (local)
    float* scratch;           // per CTA: 4 N floats (local)
    float2* cscratch;         // per CTA: 2 N (local) or 3 N (space-time) complex
};

__device__ __forceinline__ float ramp_l(const LocArgs& g, int i) { return i < g.tl ? g.ramp[i] : 1.f; }

// compute_adjsrc_local_adaptive (:545-625): the adaptive matching filter of the
// trace under a Gaussian window centred on each sample; misfit sum of the
// squared window misfits, adjoint the window adjoints weighted by the window and
// normalised by the sum of the squared windows. One CTA per trace.
__global__ void __launch_bounds__(256) k_adjsrc_local(LocArgs g) {
    extern __shared__ float2 work[];
    __shared__ double redd[32];
    __shared__ float redf[32];
    const int tid = threadIdx.x, nth = blockDim.x, nt = g.nt, N = g.dft.N;
    float* u = g.scratch + (size_t)blockIdx.x * 4 * N;
    float* d = u + N;
    float* acc = d + N;
    float* sac = acc + N;
    float2* cd = g.cscratch + (size_t)blockIdx.x * 2 * N;
    float2* cu = cd + N;
    for (int r = blockIdx.x; r < g.ntr; r += gridDim.x) {
        float* ad = g.adj ? g.adj + (size_t)r * nt : nullptr;
        if (!g.live[r]) {
            if (ad)
                for (int t = tid; t < nt; t += nth) ad[t] = 0.f;
            if (tid == 0 && g.tm) g.tm[r] = 0.0;
            continue;
        }
        const float* sy = g.syn + (size_t)r * nt;
        const float* ob = g.obs + (size_t)r * nt;
        for (int k = tid; k < N; k += nth) {
            const float rp = k < nt ? ramp_l(g, k) * ramp_l(g, nt - 1 - k) : 0.f;
            u[k] = k < nt ? sy[k] * rp : 0.f;
            d[k] = k < nt ? ob[k] * rp : 0.f;
            acc[k] = 0.f;
            sac[k] = 0.f;
        }
        __syncthreads();
        // eps from the whole trace's spectrum, eta from its matching filter
        for (int k = tid; k < N; k += nth) work[k] = make_float2(d[k], 0.f);
        dft(work, g.dft, false);
        float mx = 0.f;
        for (int k = tid; k < N; k += nth) {
            cd[k] = work[k];
            mx = fmaxf(mx, work[k].x * work[k].x + work[k].y * work[k].y);
        }
        mx = block_max(mx, redf);
        float eps = g.deconv_eps * mx;
        if (eps == 0.f) eps = 1.0e-30f;
        for (int k = tid; k < N; k += nth) work[k] = make_float2(u[k], 0.f);
        dft(work, g.dft, false);
        for (int k = tid; k < N; k += nth) work[k] = deconv_conj(work[k], cd[k], eps);
        dft(work, g.dft, true);
        float mxx = 0.f;
        for (int k = tid; k < N; k += nth) mxx = fmaxf(mxx, work[k].x * work[k].x);
        mxx = block_max(mxx, redf);
        float eta = g.deconv_eps * mxx;
        if (eta == 0.f) eta = 1.0e-30f;
        const float inv2s2 = 1.f / (2.f * g.sigma * g.sigma);
        double m = 0.0;
        for (int i = 1; i <= nt; ++i) {
            // window spectra: U = F(u g), D = F(d g), a_k = k + 1
            for (int k = tid; k < N; k += nth) {
                const float x = (float)(k + 1 - i);
                work[k] = make_float2(u[k] * expf(-x * x * inv2s2), 0.f);
            }
            dft(work, g.dft, false);
            for (int k = tid; k < N; k += nth) cu[k] = work[k];
            for (int k = tid; k < N; k += nth) {
                const float x = (float)(k + 1 - i);
                work[k] = make_float2(d[k] * expf(-x * x * inv2s2), 0.f);
            }
            dft(work, g.dft, false);
            for (int k = tid; k < N; k += nth) {
                cd[k] = work[k];
                work[k] = deconv_conj(cu[k], work[k], eps);
            }
            dft(work, g.dft, true);
            double sxx = 0.0, swx = 0.0;
            for (int k = tid; k < N; k += nth) {
                const double xc = work[k].x, wx = (double)g.pen[k] * xc;
                sxx += xc * xc;
                swx += wx * wx;
            }
            sxx = block_sum(sxx, redd) + (double)eta;
            swx = block_sum(swx, redd);
            const double vt = swx / sxx;
            m += vt * vt;
            for (int k = tid; k < N; k += nth) {
                const double w = g.pen[k];
                work[k] = make_float2((float)(vt * (w * w - vt) * (double)work[k].x / sxx), 0.f);
            }
            dft(work, g.dft, false);
            for (int k = tid; k < N; k += nth) work[k] = deconv_mul(work[k], cd[k], eps);
            dft(work, g.dft, true);
            for (int k = tid; k < N; k += nth) {
                const float x = (float)(k + 1 - i), gw = expf(-x * x * inv2s2);
                acc[k] += work[k].x * gw;
                sac[k] += gw * gw;
            }
        }
        __syncthreads();
        if (ad)
            for (int t = tid; t < nt; t += nth) ad[t] = acc[t] / sac[t] * ramp_l(g, nt - 1 - t);
        if (tid == 0 && g.tm) g.tm[r] = m;
        __syncthreads();
    }
}

// gather of trace r (gptr ascending)
__device__ int gather_index(const int* gptr, int ngather, int r) {
    int lo = 0, hi = ngather - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (gptr[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// compute_adjsrc_adaptive_spacetime (:630-700): the matching filter averaged
// over the trace and its hw neighbours on each side within the gather (dropped
// traces count as zero traces and are left out of the average), misfit as the
// adaptive one, adjoint through the centre trace's spectrum. One CTA per trace.
__global__ void __launch_bounds__(256) k_adjsrc_spacetime(LocArgs g) {
    extern __shared__ float2 work[];
    __shared__ double redd[32];
    __shared__ float redf[32];
    const int tid = threadIdx.x, nth = blockDim.x, nt = g.nt, N = g.dft.N;
    float2* cs = g.cscratch + (size_t)blockIdx.x * 3 * N;  // summed filter spectra
    float2* cd = cs + N;                                   // a neighbour's D
    float2* cc = cd + N;                                   // the centre trace's D
    for (int r = blockIdx.x; r < g.ntr; r += gridDim.x) {
        float* ad = g.adj ? g.adj + (size_t)r * nt : nullptr;
        if (!g.live[r]) {
            if (ad)
                for (int t = tid; t < nt; t += nth) ad[t] = 0.f;
            if (tid == 0 && g.tm) g.tm[r] = 0.0;
            continue;
        }
        const int gi = gather_index(g.gptr, g.ngather, r), g0 = g.gptr[gi], g1 = g.gptr[gi + 1];
        for (int k = tid; k < N; k += nth) cs[k] = make_float2(0.f, 0.f);
        int l = 0;
        float eps_c = 0.f;
        for (int q = r - g.hw; q <= r + g.hw; ++q) {
            if (q < g0 || q >= g1 || !g.live[q]) continue;
            const float* sy = g.syn + (size_t)q * nt;
            const float* ob = g.obs + (size_t)q * nt;
            for (int k = tid; k < N; k += nth)
                work[k] = make_float2(k < nt ? ob[k] * ramp_l(g, k) * ramp_l(g, nt - 1 - k) : 0.f, 0.f);
            dft(work, g.dft, false);
            float mx = 0.f;
            for (int k = tid; k < N; k += nth) {
                cd[k] = work[k];
                if (q == r) cc[k] = work[k];
                mx = fmaxf(mx, work[k].x * work[k].x + work[k].y * work[k].y);
            }
            mx = block_max(mx, redf);
            const float eps = g.deconv_eps * mx;
            if (q == r) eps_c = eps;
            if (!(eps > 0.f)) continue;
            for (int k = tid; k < N; k += nth)
                work[k] = make_float2(k < nt ? sy[k] * ramp_l(g, k) * ramp_l(g, nt - 1 - k) : 0.f, 0.f);
            dft(work, g.dft, false);
            for (int k = tid; k < N; k += nth) {
                const float2 v = deconv_conj(work[k], cd[k], eps);
                cs[k] = make_float2(cs[k].x + v.x, cs[k].y + v.y);
            }
            ++l;
        }
        for (int k = tid; k < N; k += nth) work[k] = cs[k];
        dft(work, g.dft, true);
        double sxx = 0.0, swx = 0.0;
        const float il = l > 0 ? 1.f / (float)l : 0.f;
        for (int k = tid; k < N; k += nth) {
            const double xc = (double)(work[k].x * il), wx = (double)g.pen[k] * xc;
            sxx += xc * xc;
            swx += wx * wx;
        }
        sxx = block_sum(sxx, redd);
        swx = block_sum(swx, redd);
        const double m = l > 0 ? 0.5 * swx / sxx : 0.0;
        for (int k = tid; k < N; k += nth) {
            const double w = g.pen[k];
            work[k] = make_float2((float)((w * w - 2.0 * m) * (double)(work[k].x * il) / sxx), 0.f);
        }
        dft(work, g.dft, false);
        for (int k = tid; k < N; k += nth) work[k] = deconv_mul(work[k], cc[k], eps_c);
        dft(work, g.dft, true);
        if (ad)
            for (int t = tid; t < nt; t += nth) ad[t] = work[t].x * ramp_l(g, nt - 1 - t);
        if (tid == 0 && g.tm) g.tm[r] = m;
        __syncthreads();
    }
}

}  // namespace

void DftTables::build(int n, cudaStream_t s) {
    if (n == N) return;
    OWL_CHECK(n >= 1, OWL_ERR_INVALID, "DFT length must be positive");
    int m = 2, lg = 1;
    while (m < 2 * n - 1) {
        m <<= 1;
        ++lg;
    }
    OWL_CHECK(m <= MAX_DFT_M, OWL_ERR_INVALID, "trace too long for the on-chip DFT (length " + std::to_string(n) + ")");
    std::vector<float2> hc(n), hb(m), ht(m / 2);
    std::vector<std::complex<double>> c(n), b(m, 0.0);
    for (int i = 0; i < n; ++i) {
        const long long r = ((long long)i * i) % (2LL * n);
        c[i] = std::polar(1.0, -M_PI * (double)r / (double)n);
        hc[i] = make_float2((float)c[i].real(), (float)c[i].imag());
    }
    for (int i = 0; i < n; ++i) b[i] = std::conj(c[i]);
    for (int i = 1; i < n; ++i) b[m - i] = std::conj(c[i]);
    host_fft(b);
    for (int i = 0; i < m; ++i) hb[i] = make_float2((float)b[i].real(), (float)b[i].imag());
    for (int j = 0; j < m / 2; ++j) {
        const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * (double)j / (double)m);
        ht[j] = make_float2((float)w.real(), (float)w.imag());
    }
    chirp.upload(hc.data(), hc.size(), s);
    bf.upload(hb.data(), hb.size(), s);
    tw.upload(ht.data(), ht.size(), s);
    // the uploads read host vectors that end with this scope
    OWL_CUDA(cudaStreamSynchronize(s));
    N = n;
    M = m;
    logM = lg;
}

// xcorr_penalty (:321-363) laid out on the nnt circular lags of an adaptive
// misfit: maxlag = ceiling(tlag_max / dt) (at most (nnt - 1) / 2), lag i at
// bin i, lag -i at bin nnt - i
static std::vector<float> awi_penalty(const owl_misfit_opts& o, float tlag, int nnt) {
    int maxlag = (int)std::ceil(tlag / o.dt);
    maxlag = std::max(0, std::min(maxlag, (nnt - 1) / 2));
    const double pw = std::fabs(o.penalty_power != 0.f ? (double)o.penalty_power : 1.0);
    std::vector<double> p(2 * maxlag + 1);
    const double sc = 1.0 / std::sqrt(2.0 * std::log(100.0));
    for (int i = -maxlag; i <= maxlag; ++i) {
        const double t = (double)i * (double)o.dt;
        double w;
        switch (o.penalty) {
            case OWL_PENALTY_POWER: w = std::pow(std::fabs(t / tlag), pw); break;
            case OWL_PENALTY_GAUSSIAN: w = std::exp(-t * t / (sc * (double)tlag * (double)tlag)); break;
            case OWL_PENALTY_EXP: w = std::exp(-std::fabs(t) / (sc * (double)tlag)); break;
            default: w = std::fabs(t / tlag); break;
        }
        p[i + maxlag] = w;
    }
    if (o.penalty == OWL_PENALTY_GAUSSIAN || o.penalty == OWL_PENALTY_EXP) {
        // rescale to [0, 1], power, 1 - w
        const double lo = *std::min_element(p.begin(), p.end()), hi = *std::max_element(p.begin(), p.end());
        for (double& w : p) w = 1.0 - std::pow(hi > lo ? (w - lo) / (hi - lo) : 0.0, pw);
    }
    std::vector<float> hp(nnt, 0.f);
    for (int i = 0; i <= maxlag; ++i) hp[i] = (float)p[maxlag + i];
    for (int i = 1; i <= maxlag; ++i) hp[nnt - i] = (float)p[maxlag - i];
    return hp;
}

void AdjointSource::run(const owl_misfit_opts& o, int ngather, const int* h_gather_ptr, int nt, const float* syn,
                        const float* obs, const unsigned char* weight_live, float* adj, double* tm, double* gm,
                        cudaStream_t s, float* tau) {
    OWL_CHECK(o.misfit >= OWL_MISFIT_WAVEFORM && o.misfit <= OWL_MISFIT_DTW_VECTOR, OWL_ERR_INVALID,
              "bad misfit type");
    OWL_CHECK(nt >= 1 && ngather >= 0 && (ngather == 0 || h_gather_ptr), OWL_ERR_INVALID, "bad trace layout");
    OWL_CHECK(ngather == 0 || h_gather_ptr[0] == 0, OWL_ERR_INVALID, "gather_ptr[0] must be 0");
    for (int g = 0; g < ngather; ++g)
        OWL_CHECK(h_gather_ptr[g + 1] >= h_gather_ptr[g], OWL_ERR_INVALID, "gather_ptr must not decrease");
    const int ntr = ngather ? h_gather_ptr[ngather] : 0;
    if (ntr == 0) {
        if (gm && ngather) OWL_CUDA(cudaMemsetAsync(gm, 0, sizeof(double) * ngather, s));
        return;
    }
    OWL_CHECK(syn && obs, OWL_ERR_INVALID, "null trace buffer");
    const double thr = o.discard_threshold == 0.f ? 1.0e-6 : std::max(0.0, (double)o.discard_threshold);
    gptr.upload(h_gather_ptr, (size_t)ngather + 1, s);
    nrm.reserve(2 * (size_t)ntr);
    live.reserve(ntr);
    k_trace_norms<<<(ntr + 7) / 8, 256, 0, s>>>(syn, obs, nt, ntr, nrm.p);
    k_gather_live<<<(ngather + 127) / 128, 128, 0, s>>>(gptr.p, ngather, nrm.p, weight_live, thr, live.p);
    OWL_LAUNCH_CHECK();
    launches += 2;

    const bool dtw = o.misfit == OWL_MISFIT_DTW || o.misfit == OWL_MISFIT_DTW_VECTOR;
    if (o.adj_nt > 0 && o.adj_nt != nt && !dtw) {
        // adj_nt (:1082-1089, :1111-1152): the misfit on the traces resampled to
        // adj_nt samples over the same span (cubic), the adjoint resampled back;
        // the trace selection is that of the traces as given (DTW resamples
        // only its shift computation: run_dtw)
        OWL_CHECK(o.dt > 0.f && o.adj_nt >= 2, OWL_ERR_INVALID, "adj_nt needs dt and at least 2 samples");
        const int nn = o.adj_nt;
        const float dd = ((float)(nt - 1) * o.dt) / (float)(nn - 1);
        DevBuf<float> rs, ro, ra;
        DevBuf<unsigned char> keep;
        rs.reserve((size_t)ntr * nn);
        ro.reserve((size_t)ntr * nn);
        keep.reserve(ntr);
        OWL_CUDA(cudaMemcpyAsync(keep.p, live.p, ntr, cudaMemcpyDeviceToDevice, s));
        launch_resample_rows(syn, nt, o.dt, 0.0, rs.p, nn, dd, 0.0, ntr, s);
        launch_resample_rows(obs, nt, o.dt, 0.0, ro.p, nn, dd, 0.0, ntr, s);
        if (adj) ra.reserve((size_t)ntr * nn);
        owl_misfit_opts o2 = o;
        o2.adj_nt = 0;
        o2.dt = dd;
        o2.discard_threshold = -1.f;  // the selection made above; zero traces stay zero
        run(o2, ngather, h_gather_ptr, nn, rs.p, ro.p, keep.p, adj ? ra.p : nullptr, tm, gm, s);
        if (adj) launch_resample_rows(ra.p, nn, dd, 0.0, adj, nt, o.dt, 0.0, ntr, s);
        OWL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    if (dtw) {
        if (o.misfit == OWL_MISFIT_DTW_VECTOR) {
            const int vc = std::max(1, o.ncomp);
            OWL_CHECK(ngather % vc == 0, OWL_ERR_INVALID, "dtw-vector: the gathers must come in groups of ncomp");
            for (int g = 0; g < ngather; g += vc)
                for (int c = 1; c < vc; ++c)
                    OWL_CHECK(h_gather_ptr[g + c + 1] - h_gather_ptr[g + c] == h_gather_ptr[g + 1] - h_gather_ptr[g],
                              OWL_ERR_INVALID, "dtw-vector: the component gathers of a shot must hold equal trace counts");
        }
        DevBuf<double> tmp;
        if (!tm && gm) {
            tmp.reserve(ntr);
            tm = tmp.p;
        }
        run_dtw(o, ngather, nt, ntr, syn, obs, adj, tm, tau, s);
        if (gm) {
            k_gather_sum<<<(ngather + 127) / 128, 128, 0, s>>>(tm, gptr.p, ngather, gm);
            OWL_LAUNCH_CHECK();
            launches++;
        }
        OWL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    if (o.misfit == OWL_MISFIT_LOCAL_ADAPTIVE || o.misfit == OWL_MISFIT_ADAPTIVE_SPACETIME) {
        OWL_CHECK(o.dt > 0.f, OWL_ERR_INVALID, "the adaptive misfits need the sample interval dt");
        const bool loc = o.misfit == OWL_MISFIT_LOCAL_ADAPTIVE;
        const int nnt = next_power_235(loc ? 2 * nt : 4 * nt);
        awl.build(nnt, s);
        const float tlag = o.tlag_max > 0.f ? o.tlag_max : 0.1f * (float)(nt - 1) * o.dt;
        const std::vector<float> hp = awi_penalty(o, tlag, nnt);
        pen.upload(hp.data(), hp.size(), s);
        const int tl = (int)std::floor(0.025f * (float)nt + 0.5f);
        std::vector<float> hramp(std::max(tl, 1));
        for (int i = 0; i < tl; ++i) hramp[i] = (float)(0.5 * (1.0 - std::cos(M_PI * (double)i / (double)tl)));
        ramp.upload(hramp.data(), hramp.size(), s);
        DevBuf<double> tmp;
        if (!tm && gm) {
            tmp.reserve(ntr);
            tm = tmp.p;
        }
        LocArgs la{};
        la.nt = nt;
        la.ntr = ntr;
        la.ngather = ngather;
        la.hw = o.adaptive_half_window > 0 ? o.adaptive_half_window : 3;
        la.gptr = gptr.p;
        la.syn = syn;
        la.obs = obs;
        la.live = live.p;
        la.adj = adj;
        la.tm = tm;
        la.dft = dev(awl);
        la.pen = pen.p;
        la.ramp = ramp.p;
        la.tl = tl;
        la.deconv_eps = o.deconv_eps > 0.f ? o.deconv_eps : 0.1f;
        la.sigma = (o.lawi_sigma > 0.f ? o.lawi_sigma : 0.25f) / o.dt;
        const size_t smem = (size_t)awl.M * sizeof(float2);
        auto k = loc ? k_adjsrc_local : k_adjsrc_spacetime;
        OWL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0, nsm = 0, dev_id = 0;
        OWL_CUDA(cudaGetDevice(&dev_id));
        OWL_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id));
        OWL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, smem));
        const int grid = std::max(1, std::min(ntr, nsm * std::max(1, per_sm)));
        scratch.reserve(loc ? (size_t)grid * 4 * nnt : 1);
        cscratch.reserve((size_t)grid * (loc ? 2 : 3) * nnt);
        la.scratch = scratch.p;
        la.cscratch = cscratch.p;
        k<<<grid, 256, smem, s>>>(la);
        OWL_LAUNCH_CHECK();
        launches++;
        if (gm) {
            k_gather_sum<<<(ngather + 127) / 128, 128, 0, s>>>(tm, gptr.p, ngather, gm);
            OWL_LAUNCH_CHECK();
            launches++;
        }
        OWL_CUDA(cudaStreamSynchronize(s));
        return;
    }
    AdjArgs a{};
    a.kind = o.misfit;
    a.nt = nt;
    a.ntr = ntr;
    a.syn = syn;
    a.obs = obs;
    a.live = live.p;
    a.adj = adj;
    DevBuf<double> tmp_tm;
    if (!tm && gm) {
        tmp_tm.reserve(ntr);
        tm = tmp_tm.p;
    }
    a.tm = tm;
    int M = 0;
    std::vector<float> hramp, hp;
    if (o.misfit == OWL_MISFIT_ENVELOPE || o.misfit == OWL_MISFIT_PHASE) {
        hil.build(nt, s);
        a.hil = dev(hil);
        M = hil.M;
    }
    if (o.misfit == OWL_MISFIT_ADAPTIVE) {
        OWL_CHECK(o.dt > 0.f, OWL_ERR_INVALID, "the adaptive misfit needs the sample interval dt");
        const int nnt = next_power_235(2 * nt);
        awi.build(nnt, s);
        a.awi = dev(awi);
        M = awi.M;
        const float tlag = o.tlag_max > 0.f ? o.tlag_max : 0.1f * (float)(nt - 1) * o.dt;
        hp = awi_penalty(o, tlag, nnt);
        const int tl = (int)std::floor(0.025f * (float)nt + 0.5f);
        pen.upload(hp.data(), hp.size(), s);
        a.pen = pen.p;
        hramp.resize(std::max(tl, 1));
        for (int i = 0; i < tl; ++i) hramp[i] = (float)(0.5 * (1.0 - std::cos(M_PI * (double)i / (double)tl)));
        ramp.upload(hramp.data(), hramp.size(), s);
        a.ramp = ramp.p;
        a.tl = tl;
        a.deconv_eps = o.deconv_eps > 0.f ? o.deconv_eps : 0.1f;
    }
    const size_t smem = (size_t)M * sizeof(float2);
    OWL_CUDA(cudaFuncSetAttribute(k_adjsrc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 1)));
    int per_sm = 0, nsm = 0, dev_id = 0;
    OWL_CUDA(cudaGetDevice(&dev_id));
    OWL_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id));
    OWL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjsrc, 256, smem));
    const int grid = std::max(1, std::min(ntr, nsm * std::max(1, per_sm)));
    const bool fft = M > 0;
    scratch.reserve(fft ? (size_t)grid * 4 * nt : 1);
    cscratch.reserve(o.misfit == OWL_MISFIT_ADAPTIVE ? (size_t)grid * awi.N : 1);
    a.scratch = scratch.p;
    a.cscratch = cscratch.p;
    k_adjsrc<<<grid, 256, smem, s>>>(a);
    OWL_LAUNCH_CHECK();
    launches++;
    if (gm) {
        k_gather_sum<<<(ngather + 127) / 128, 128, 0, s>>>(tm, gptr.p, ngather, gm);
        OWL_LAUNCH_CHECK();
        launches++;
    }
    // tmp_tm and the host tables end with this scope
    OWL_CUDA(cudaStreamSynchronize(s));
}

void launch_nonzero(const float* w, int n, unsigned char* out, cudaStream_t s) {
    if (n <= 0) return;
    k_nonzero<<<(n + 255) / 256, 256, 0, s>>>(w, n, out);
    OWL_LAUNCH_CHECK();
}

}  // namespace owl
