// optim.cu -- search directions and gradient processing on the GPU.
//
// compute_search_direction (src/inverse/module_inversion_search_direction.f90:
// steepest descent, Polak-Ribiere conjugate gradient :38-86, two-loop L-BFGS
// :91-246) over fields that stay in device memory: every dot product is an FP64
// reduction in a fixed order (per-block partials, then one block), the vector
// updates are elementwise kernels, and s_i = x_{i+1} - x_i, y_i = g_{i+1} - g_i
// are formed on the fly from the models and gradients the caller keeps, as the
// reference reads them from its iteration directories.
//
// The gradient processing of process_model_single_parameter
// (src/inverse/2d/module_gradient.f90:733-892): Gaussian smoothing (separable,
// one pass per axis, edge samples replicated), Blackman taper ramps at the
// ends of each axis, mask, scale and max balance. FLIT's gauss_filt and taper
// are restated (a Gaussian of the given standard deviation in cells truncated
// at 3 sigma and normalised; Blackman ramps 0.42 - 0.5 cos(pi i / l) +
// 0.08 cos(2 pi i / l), i = 0..l-1, from each end).
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace owl {

namespace {

constexpr int RED_BLOCKS = 148 * 8;

// partial sums of up to three products per block: (s.q, y.s, y.y) with
// s = x1 - x0 (or x1 alone), y = g1 - g0 (or g1 alone), q
__global__ void __launch_bounds__(256) k_dots(long long n, const float* __restrict__ x1, const float* __restrict__ x0,
                                              const float* __restrict__ g1, const float* __restrict__ g0,
                                              const float* __restrict__ q, double* __restrict__ part) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double s = x1 ? (double)x1[i] - (x0 ? (double)x0[i] : 0.0) : 0.0;
        const double y = (double)g1[i] - (g0 ? (double)g0[i] : 0.0);
        const double qq = q ? (double)q[i] : 0.0;
        a += s * qq;
        b += y * s;
        c += y * (q ? qq : y);
    }
    __shared__ double red[3][8];
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = a;
        red[1][w] = b;
        red[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int i = 0; i < 8; ++i) t += red[threadIdx.x][i];
        part[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
    }
}

__global__ void k_sum_parts(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int i = 0; i < nb; ++i) t += part[(size_t)i * 3 + threadIdx.x];
        out[threadIdx.x] = t;
    }
}

// r = a * r + c * (u1 - u0) [+ d * v]   (u0, v optional)
// (u1 may be r itself)
__global__ void k_update(long long n, float* r, double a, double c, const float* u1, const float* __restrict__ u0,
                         double d, const float* __restrict__ v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double u = (double)u1[i] - (u0 ? (double)u0[i] : 0.0);
        double t = (a != 0.0 ? a * (double)r[i] : 0.0) + c * u;  // a = 0: r is write-only
        if (v) t += d * (double)v[i];
        r[i] = (float)t;
    }
}

// one axis of a separable filter: field (n1, n2, n3), axis stride `st`, length `len`
__global__ void k_smooth_axis(const float* __restrict__ in, float* __restrict__ out, long long n, long long st, int len,
                              const float* __restrict__ w, int rad) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)((i / st) % len);
        const long long base = i - (long long)p * st;
        float acc = 0.f;
        for (int k = -rad; k <= rad; ++k) {
            const int q = min(max(p + k, 0), len - 1);
            acc += w[k + rad] * in[base + (long long)q * st];
        }
        out[i] = acc;
    }
}

__global__ void k_taper(float* __restrict__ f, long long n, int n1, int n2, int n3, int a1, int b1, int a2, int b2,
                        int a3, int b3) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(i % n1);
        const int i2 = (int)((i / n1) % n2);
        const int i3 = (int)(i / ((long long)n1 * n2));
        auto ramp = [](int j, int l) -> float {
            if (j >= l) return 1.f;
            const double t = (double)j / (double)l;
            return (float)(0.42 - 0.5 * cospi(t) + 0.08 * cospi(2.0 * t));
        };
        float w = 1.f;  // axes of one sample are left alone
        if (n1 > 1) w *= ramp(i1, a1) * ramp(n1 - 1 - i1, b1);
        if (n2 > 1) w *= ramp(i2, a2) * ramp(n2 - 1 - i2, b2);
        if (n3 > 1) w *= ramp(i3, a3) * ramp(n3 - 1 - i3, b3);
        f[i] *= w;
    }
}

__global__ void k_mul(float* __restrict__ f, long long n, const float* __restrict__ m, float c) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        f[i] = (m ? f[i] * m[i] : f[i]) * c;
}

__global__ void k_max_part(const float* __restrict__ f, long long n, float* __restrict__ part) {
    float m = -INFINITY;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, f[i]);
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = red[0];
        for (int i = 1; i < 8; ++i) t = fmaxf(t, red[i]);
        part[blockIdx.x] = t;
    }
}

// sum of squares of each slice along an axis (one CTA per slice, FP64)
__global__ void k_slice_sumsq(const float* __restrict__ f, int n1, int n2, int n3, int axis, double* __restrict__ out) {
    const int j = blockIdx.x;
    const long long m = axis == 0 ? (long long)n2 * n3 : axis == 1 ? (long long)n1 * n3 : (long long)n1 * n2;
    double acc = 0.0;
    for (long long e = threadIdx.x; e < m; e += blockDim.x) {
        long long i1, i2, i3;
        if (axis == 0) { i1 = j; i2 = e % n2; i3 = e / n2; }
        else if (axis == 1) { i1 = e % n1; i2 = j; i3 = e / n1; }
        else { i1 = e % n1; i2 = e / n1; i3 = j; }
        const double v = f[(i3 * n2 + i2) * n1 + i1];
        acc += v * v;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = red[0];
}

// each element divided by the norm of its slice's window; NaN / Inf -> 0
__global__ void k_div_slice(float* __restrict__ f, long long n, int n1, int n2, int axis, const float* __restrict__ nrm) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long j = axis == 0 ? i % n1 : axis == 1 ? (i / n1) % n2 : i / ((long long)n1 * n2);
        const float v = f[i] / nrm[j];
        f[i] = isfinite(v) ? v : 0.f;
    }
}

// median of the (2 h1 + 1) x (2 h2 + 1) x (2 h3 + 1) window, truncated at the ends
__device__ float select_kth(float* a, int n, int k) {  // k-th smallest (0-based), a is reordered
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const float piv = a[(lo + hi) / 2];
        int i = lo, j = hi;
        while (i <= j) {
            while (a[i] < piv) ++i;
            while (a[j] > piv) --j;
            if (i <= j) {
                const float t = a[i]; a[i] = a[j]; a[j] = t;
                ++i; --j;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else return a[k];
    }
    return a[k];
}

__global__ void k_median(const float* __restrict__ in, float* __restrict__ out, int n1, int n2, int n3, int h1, int h2,
                         int h3) {
    const long long n = (long long)n1 * n2 * n3;
    float w[343];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(i % n1), i2 = (int)((i / n1) % n2), i3 = (int)(i / ((long long)n1 * n2));
        int c = 0;
        for (int a3 = max(0, i3 - h3); a3 <= min(n3 - 1, i3 + h3); ++a3)
            for (int a2 = max(0, i2 - h2); a2 <= min(n2 - 1, i2 + h2); ++a2)
                for (int a1 = max(0, i1 - h1); a1 <= min(n1 - 1, i1 + h1); ++a1)
                    w[c++] = in[((long long)a3 * n2 + a2) * n1 + a1];
        float v;
        if (c & 1) {
            v = select_kth(w, c, c / 2);
        } else {
            const float hi = select_kth(w, c, c / 2);
            float lo = w[0];  // after the selection, the largest of w[0 .. c/2 - 1] is the (c/2 - 1)-th
            for (int k = 1; k < c / 2; ++k) lo = fmaxf(lo, w[k]);
            v = 0.5f * (lo + hi);
        }
        out[i] = v;
    }
}

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, RED_BLOCKS)); }

// (s.q, y.s, y.y) on the device, returned to the host
struct Dots {
    DevBuf<double> part, out;
    double v[3];
    void run(long long n, const float* x1, const float* x0, const float* g1, const float* g0, const float* q,
             cudaStream_t s) {
        const int nb = blocks_for(n);
        part.reserve((size_t)nb * 3);
        out.reserve(3);
        k_dots<<<nb, 256, 0, s>>>(n, x1, x0, g1, g0, q, part.p);
        k_sum_parts<<<1, 32, 0, s>>>(part.p, nb, out.p);
        OWL_LAUNCH_CHECK();
        OWL_CUDA(cudaMemcpyAsync(v, out.p, sizeof(v), cudaMemcpyDeviceToHost, s));
        OWL_CUDA(cudaStreamSynchronize(s));
    }
};

void update(long long n, float* r, double a, double c, const float* u1, const float* u0, double d, const float* v,
            cudaStream_t s) {
    k_update<<<blocks_for(n), 256, 0, s>>>(n, r, a, c, u1, u0, d, v);
    OWL_LAUNCH_CHECK();
}

}  // namespace

// models[0..nm-1] oldest first, grads alike; srch written. All device pointers.
void search_direction(int method, long long n, int nm, const float* const* x, const float* const* g,
                      const float* prev_srch, float* srch, cudaStream_t s) {
    Dots dots;
    const float* gk = g[nm - 1];
    if (method == OWL_SEARCH_SD || nm < 2) {
        update(n, srch, 0.0, -1.0, gk, nullptr, 0.0, nullptr, s);
        return;
    }
    if (method == OWL_SEARCH_CG) {
        // Polak-Ribiere: beta = max(0, g.(g - gp) / gp.gp), srch = -g + beta srch_prev
        OWL_CHECK(prev_srch, OWL_ERR_INVALID, "conjugate gradient needs the previous search direction");
        const float* gp = g[nm - 2];
        dots.run(n, nullptr, nullptr, gp, nullptr, nullptr, s);
        const double s1 = dots.v[2];
        dots.run(n, nullptr, nullptr, gk, gp, gk, s);  // y = g - gp, q = g: c = y.g
        const double s2 = dots.v[2];
        const double beta = s1 == 0.0 ? 0.0 : std::max(0.0, s2 / s1);
        update(n, srch, 0.0, -1.0, gk, nullptr, beta, prev_srch, s);
        return;
    }
    // L-BFGS two-loop recursion over the pairs (x_{i+1} - x_i, g_{i+1} - g_i), newest first
    const int np = nm - 1;
    std::vector<double> alpha(np, 0.0), ys(np, 0.0);
    OWL_CUDA(cudaMemcpyAsync(srch, gk, n * sizeof(float), cudaMemcpyDeviceToDevice, s));  // q = g_k
    for (int i = np - 1; i >= 0; --i) {
        dots.run(n, x[i + 1], x[i], g[i + 1], g[i], srch, s);  // a = s.q, b = y.s
        ys[i] = dots.v[1];
        alpha[i] = ys[i] == 0.0 ? 0.0 : dots.v[0] / ys[i];
        update(n, srch, 1.0, -alpha[i], g[i + 1], g[i], 0.0, nullptr, s);  // q -= alpha y
    }
    // initial scaling (s.y) / (y.y) of the newest pair
    dots.run(n, x[np], x[np - 1], g[np], g[np - 1], nullptr, s);
    const double gamma = dots.v[2] == 0.0 ? 0.0 : dots.v[1] / dots.v[2];
    update(n, srch, gamma, 0.0, srch, nullptr, 0.0, nullptr, s);
    for (int i = 0; i < np; ++i) {
        dots.run(n, nullptr, nullptr, g[i + 1], g[i], srch, s);  // c = y.r
        const double beta = ys[i] == 0.0 ? 0.0 : dots.v[2] / ys[i];
        update(n, srch, 1.0, alpha[i] - beta, x[i + 1], x[i], 0.0, nullptr, s);  // r += s (alpha - beta)
    }
    update(n, srch, -1.0, 0.0, srch, nullptr, 0.0, nullptr, s);
}

void grad_process(int op, int n1, int n2, int n3, const float* param, const float* mask, float* f, cudaStream_t s) {
    const long long n = (long long)n1 * n2 * n3;
    if (n == 0) return;
    const int nb = blocks_for(n);
    switch (op) {
        case OWL_GRAD_SMOOTH: {
            DevBuf<float> tmp, w;
            tmp.reserve(n);
            const int len[3] = {n1, n2, n3};
            const long long st[3] = {1, n1, (long long)n1 * n2};
            for (int ax = 0; ax < 3; ++ax) {
                const double sg = param[ax];
                if (!(sg > 0.0) || len[ax] < 2) continue;
                const int rad = std::max(1, (int)std::ceil(3.0 * sg));
                std::vector<float> hw(2 * rad + 1);
                double tot = 0.0;
                std::vector<double> dw(2 * rad + 1);
                for (int k = -rad; k <= rad; ++k) tot += dw[k + rad] = std::exp(-0.5 * (double)k * k / (sg * sg));
                for (int k = 0; k <= 2 * rad; ++k) hw[k] = (float)(dw[k] / tot);
                w.upload(hw.data(), hw.size(), s);
                k_smooth_axis<<<nb, 256, 0, s>>>(f, tmp.p, n, st[ax], len[ax], w.p, rad);
                OWL_LAUNCH_CHECK();
                OWL_CUDA(cudaMemcpyAsync(f, tmp.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
                OWL_CUDA(cudaStreamSynchronize(s));  // hw is reused by the next axis
            }
            break;
        }
        case OWL_GRAD_TAPER: {
            int l[6];
            for (int i = 0; i < 6; ++i) l[i] = std::max(0, (int)std::lround(param[i]));
            k_taper<<<nb, 256, 0, s>>>(f, n, n1, n2, n3, l[0], l[1], l[2], l[3], l[4], l[5]);
            OWL_LAUNCH_CHECK();
            break;
        }
        case OWL_GRAD_MASK:
            OWL_CHECK(mask, OWL_ERR_INVALID, "mask needs a mask field");
            k_mul<<<nb, 256, 0, s>>>(f, n, mask, 1.f);
            OWL_LAUNCH_CHECK();
            break;
        case OWL_GRAD_SCALE:
            k_mul<<<nb, 256, 0, s>>>(f, n, nullptr, param[0]);
            OWL_LAUNCH_CHECK();
            break;
        case OWL_GRAD_MAX_BALANCE: {
            DevBuf<float> part;
            part.reserve(nb);
            k_max_part<<<nb, 256, 0, s>>>(f, n, part.p);
            OWL_LAUNCH_CHECK();
            std::vector<float> hp(nb);
            OWL_CUDA(cudaMemcpyAsync(hp.data(), part.p, nb * sizeof(float), cudaMemcpyDeviceToHost, s));
            OWL_CUDA(cudaStreamSynchronize(s));
            const float m = *std::max_element(hp.begin(), hp.end());
            if (m != 0.f) {
                k_mul<<<nb, 256, 0, s>>>(f, n, nullptr, 1.f / m);
                OWL_LAUNCH_CHECK();
            }
            break;
        }
        case OWL_GRAD_RMS_BALANCE: {
            DevBuf<double> part, tot;
            part.reserve(1);
            k_slice_sumsq<<<1, 256, 0, s>>>(f, 1, (int)n, 1, 0, part.p);  // the whole field as one slice
            OWL_LAUNCH_CHECK();
            double ss = 0.0;
            OWL_CUDA(cudaMemcpyAsync(&ss, part.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            OWL_CUDA(cudaStreamSynchronize(s));
            const double rms = std::sqrt(ss / (double)n);
            if (rms != 0.0) {
                k_mul<<<nb, 256, 0, s>>>(f, n, nullptr, (float)(1.0 / rms));
                OWL_LAUNCH_CHECK();
            }
            break;
        }
        case OWL_GRAD_RMS_BALANCE_AXIS: {
            const int axis = (int)std::lround(param[0]) - 1;
            OWL_CHECK(axis >= 0 && axis <= 2, OWL_ERR_INVALID, "rms balance axis must be 1, 2 or 3");
            int wn = (int)std::lround(param[1]);
            if (wn % 2 == 0) --wn;
            OWL_CHECK(wn >= 1, OWL_ERR_INVALID, "rms balance window must be at least 1 cell");
            const int len[3] = {n1, n2, n3};
            const int L = len[axis];
            DevBuf<double> ss;
            ss.reserve(L);
            k_slice_sumsq<<<L, 256, 0, s>>>(f, n1, n2, n3, axis, ss.p);
            OWL_LAUNCH_CHECK();
            std::vector<double> hs(L);
            OWL_CUDA(cudaMemcpyAsync(hs.data(), ss.p, L * sizeof(double), cudaMemcpyDeviceToHost, s));
            OWL_CUDA(cudaStreamSynchronize(s));
            std::vector<float> hn(L);
            const int hw = (wn - 1) / 2;
            for (int j = 0; j < L; ++j) {
                double acc = 0.0;
                for (int k = std::max(0, j - hw); k <= std::min(L - 1, j + hw); ++k) acc += hs[k];
                hn[j] = (float)std::sqrt(acc);
            }
            DevBuf<float> dn;
            dn.upload(hn.data(), L, s);
            k_div_slice<<<nb, 256, 0, s>>>(f, n, n1, n2, axis, dn.p);
            OWL_LAUNCH_CHECK();
            OWL_CUDA(cudaStreamSynchronize(s));
            break;
        }
        case OWL_GRAD_MEDIAN: {
            int h[3];
            for (int i = 0; i < 3; ++i) h[i] = std::max(0, (int)std::lround(param[i]));
            if (n1 == 1) h[0] = 0;
            if (n2 == 1) h[1] = 0;
            if (n3 == 1) h[2] = 0;
            OWL_CHECK((2 * h[0] + 1) * (2 * h[1] + 1) * (2 * h[2] + 1) <= 343, OWL_ERR_INVALID,
                      "median window above 343 cells");
            DevBuf<float> tmp;
            tmp.reserve(n);
            k_median<<<nb, 256, 0, s>>>(f, tmp.p, n1, n2, n3, h[0], h[1], h[2]);
            OWL_LAUNCH_CHECK();
            OWL_CUDA(cudaMemcpyAsync(f, tmp.p, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
            break;
        }
        default:
            throw OwlError(OWL_ERR_INVALID, "bad gradient processing op");
    }
    OWL_CUDA(cudaStreamSynchronize(s));
}

}  // namespace owl
