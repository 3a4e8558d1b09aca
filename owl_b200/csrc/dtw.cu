// dtw.cu -- dynamic-time-warping misfit and adjoint source on the GPU
// (compute_adjsrc_dtw and solve_gdtw, src/inverse/module_inversion_adjoint_source.f90:73-234, 715-980).
//
// Per gather (one shot's one component), for every kept trace:
//   1. obs and syn are normalised by their own L2 norms (single precision);
//   2. the generalized DTW of Deriso & Boyd finds the shift tau(t) with
//      obs(t + tau) ~ syn(t): a dynamic program over n samples x m candidate
//      shifts per iteration, the candidate band shrinking around the previous
//      path (dtw_niter iterations at most). One CTA per trace, one thread per
//      candidate; the double-precision arithmetic of the program uses
//      explicitly rounded operations (no fused multiply-add) so that every
//      comparison matches the FP64 restatement in the oracle;
//   3. a quality weight q(t) from the windowed normalised correlation of syn and
//      the warped obs (|q|^0.2, 7-sample median, Gaussian of 3 samples,
//      normalised, rescaled to [0, 1]);
//   4. misfit sum q tau^2 and adjoint q tau d/dt(warped obs) ('phase'), the
//      warped residual ('amp'), or both ('phase+amp').
#include <algorithm>
#include <cmath>

#include "adjsrc.cuh"

namespace owl {

namespace {

constexpr double DTW_SMIN = 1.0e-8, DTW_SMAX = 1.0e2, DTW_ETA = 0.15, DTW_DELTA = 1.0e-10;
constexpr double DTW_HUGE = 1.7976931348623157e308;

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

struct DtwArgs {
    int n, m, ntr, ngather, niter, trc, form;
    int vc;               // components per receiver: 1, or the ncomp consecutive gathers of a shot (dtw-vector)
    const double* vnrm;   // per row: obs and syn norms over the receiver's kept components
    const int* gptr;
    const unsigned char* live;
    const float* syn;
    const float* obs;
    const double* nrm;    // per trace: obs norm, syn norm
    double* dsn;          // normalised syn (ntr x n)
    double* dob;          // normalised obs
    float* tau;           // shift in seconds (ntr x n)
    float* q;             // quality weight
    float* dw;            // warped normalised obs (ntr x n)
    unsigned short* path; // per CTA: n x m back-pointers
    double* band;         // per CTA: l, u, tau (3 n)
    double rinst, rcuml, epsabs, epsrel, power;
    float dd, amp_weight, tlag;
    float* adj;
    double* tm;
};

// gather of trace r (gptr ascending)
__device__ int gather_of(const DtwArgs& a, int r) {
    int lo = 0, hi = a.ngather - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (a.gptr[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// row of component c of the receiver of row r (dtw-vector; c = the row's own
// component when vc = 1), and the gather bounds of that component
__device__ __forceinline__ int comp_row(const DtwArgs& a, int g, int r, int c, int& lo, int& hi) {
    const int sg = g / a.vc, gc = sg * a.vc + c;
    lo = a.gptr[gc];
    hi = a.gptr[gc + 1];
    return lo + (r - a.gptr[g]);
}

// obs / syn norms of each row's receiver over its kept components
__global__ void k_dtw_vnorm(DtwArgs a, double* vn) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.ntr) return;
    const int g = gather_of(a, r);
    double so = 0.0, ss = 0.0;
    for (int c = 0; c < a.vc; ++c) {
        int lo, hi;
        const int rc = comp_row(a, g, r, c, lo, hi);
        if (rc < hi && a.live[rc]) {
            so += a.nrm[2 * rc] * a.nrm[2 * rc];
            ss += a.nrm[2 * rc + 1] * a.nrm[2 * rc + 1];
        }
    }
    vn[2 * r] = sqrt(so);
    vn[2 * r + 1] = sqrt(ss);
}

__device__ double block_sum_d(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    __syncthreads();
    return t;
}

__device__ double block_minmax_d(double v, double* red, bool is_max) {
    for (int o = 16; o; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_max ? fmax(v, w) : fmin(v, w);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = red[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) t = is_max ? fmax(t, red[i]) : fmin(t, red[i]);
    __syncthreads();
    return t;
}

// normalised traces (:761-775): obs / norm2(obs), syn / norm2(syn) in single
// precision, stored as doubles; discarded traces stay zero
__global__ void k_dtw_normalise(DtwArgs a) {
    const size_t tot = (size_t)a.ntr * a.n;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < tot; o += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(o / a.n);
        const bool lv = a.live[r] != 0;
        const double* nr = a.vc > 1 ? a.vnrm : a.nrm;
        const float no = (float)nr[2 * r], ns = (float)nr[2 * r + 1];
        a.dob[o] = lv ? (double)(a.obs[o] / no) : 0.0;
        a.dsn[o] = lv ? (double)(a.syn[o] / ns) : 0.0;
    }
}

__device__ __forceinline__ double grid_t(int i, int n) { return (double)i / (double)(n - 1); }

// linear interpolation of column x (uniform grid i / (n-1)) at q, clamped to the ends
__device__ double interp_clamped(const double* x, int n, double q) {
    if (q <= 0.0) return x[0];
    if (q >= grid_t(n - 1, n)) return x[n - 1];
    int i0 = min((int)floor(dmul(q, (double)(n - 1))), n - 2);
    i0 = max(i0, 0);
    while (i0 > 0 && grid_t(i0, n) > q) --i0;
    while (i0 < n - 2 && grid_t(i0 + 1, n) <= q) ++i0;
    const double t0 = grid_t(i0, n), t1 = grid_t(i0 + 1, n);
    const double w = dsub(q, t0) / dsub(t1, t0);
    return dadd(dmul(x[i0], dsub(1.0, w)), dmul(x[i0 + 1], w));
}

__device__ __forceinline__ double powabs(double d, double p) {
    const double v = fabs(d);
    if (p == 0.5) return __dsqrt_rn(v);
    if (p == 1.0) return v;
    if (p == 2.0) return dmul(v, v);
    return pow(v, p);
}

// solve_gdtw (:73-234), one CTA per kept trace (grid-strided over traces)
__global__ void __launch_bounds__(256) k_dtw_solve(DtwArgs a) {
    extern __shared__ double sh[];
    const int n = a.n, m = a.m, jc = (m - 1) / 2;
    double* lin = sh;
    double* fa = sh + m;
    double* fb = sh + 2 * m;
    __shared__ double s_cost;
    unsigned short* path = a.path + (size_t)blockIdx.x * n * m;
    double* L = a.band + (size_t)blockIdx.x * 3 * n;
    double* U = L + n;
    double* T = U + n;
    const double dt = 1.0 / ((double)n - 1.0);
    for (int j = threadIdx.x; j < m; j += blockDim.x) lin[j] = (double)j / (double)(m - 1);
    for (int r = blockIdx.x; r < a.ntr; r += gridDim.x) {
        const int g = gather_of(a, r);
        if (g % a.vc != 0) continue;  // dtw-vector: the receiver is solved from its first component's row
        bool lv = false;
        for (int c = 0; c < a.vc; ++c) {
            int lo, hi;
            const int rc = comp_row(a, g, r, c, lo, hi);
            lv = lv || (rc < hi && a.live[rc]);
        }
        if (!lv) {
            for (int c = 0; c < a.vc; ++c) {
                int lo, hi;
                const int rc = comp_row(a, g, r, c, lo, hi);
                if (rc < hi)
                    for (int i = threadIdx.x; i < n; i += blockDim.x) a.tau[(size_t)rc * n + i] = 0.f;
            }
            continue;
        }
        // distance columns: components outer, the trc neighbours on each side inner
        // (the reference's reshape of (nn, 2 trc + 1, nc))
        const int nc = (2 * a.trc + 1) * a.vc;
        auto col_row = [&](int c, int& rc) {
            const int comp = c / (2 * a.trc + 1), off = c - comp * (2 * a.trc + 1) - a.trc;
            int lo, hi;
            rc = comp_row(a, g, r, comp, lo, hi) + off;
            return rc >= lo && rc < hi;
        };
        double cost_prev = 1.1754943508222875e-38;  // single-precision tiny
        __syncthreads();
        for (int it = 0; it < a.niter; ++it) {
            // search band (:112-130)
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const double t = grid_t(i, n);
                const double u0 = fmin(fmin(0.0 + dmul(DTW_SMAX, t), dsub(1.0, dmul(DTW_SMIN, dsub(1.0, t)))), 1.0);
                const double l0 = fmax(fmax(dmul(DTW_SMIN, t), dsub(1.0, dmul(DTW_SMAX, dsub(1.0, t)))), 0.0);
                if (it == 0) {
                    U[i] = u0;
                    L[i] = l0;
                } else {
                    const double rng = dmul(DTW_ETA, dsub(U[i], L[i])) / 2.0;
                    U[i] = fmin(dadd(T[i], rng), u0);
                    L[i] = fmax(dsub(T[i], rng), l0);
                }
            }
            __syncthreads();
            // row 0: only the centre candidate (bc_start_stop)
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                double v = DTW_HUGE;
                if (k == jc) {
                    const double tg = dadd(L[0], dmul(dsub(U[0], L[0]), lin[k]));
                    double dist = 0.0;
                    for (int c = 0; c < nc; ++c) {
                        int rc;
                        const bool in = col_row(c, rc);
                        const double xv = in ? interp_clamped(a.dob + (size_t)rc * n, n, tg) : 0.0;
                        const double yv = in ? a.dsn[(size_t)rc * n] : 0.0;
                        dist = dadd(dist, powabs(dsub(xv, yv), a.power));
                    }
                    const double d = dsub(tg, 0.0);
                    v = dadd(dist, dmul(a.rcuml, dmul(d, d)));
                }
                fa[k] = v;
            }
            __syncthreads();
            double* fcur = fa;
            double* fnext = fb;
            for (int i = 0; i < n - 1; ++i) {
                const double li = L[i], dui = dsub(U[i], L[i]);
                const double ln = L[i + 1], dun = dsub(U[i + 1], L[i + 1]);
                const double tn = grid_t(i + 1, n);
                for (int k = threadIdx.x; k < m; k += blockDim.x) {
                    const double tgk = dadd(ln, dmul(dun, lin[k]));
                    double dist = 0.0;
                    for (int c = 0; c < nc; ++c) {
                        int rc;
                        const bool in = col_row(c, rc);
                        const double xv = in ? interp_clamped(a.dob + (size_t)rc * n, n, tgk) : 0.0;
                        const double yv = in ? a.dsn[(size_t)rc * n + i + 1] : 0.0;
                        dist = dadd(dist, powabs(dsub(xv, yv), a.power));
                    }
                    const double d = dsub(tgk, tn);
                    const double nu = dadd(dist, dmul(a.rcuml, dmul(d, d)));
                    // candidates j with s_min - delta <= slope <= s_max + delta form one run
                    // (the slope falls as j grows); walk it in ascending j as the reference does
                    auto slope_of = [&](int j) { return dsub(tgk, dadd(li, dmul(dui, lin[j]))) / dt; };
                    int j = 0;
                    if (dui > 0.0) {
                        const double est = (tgk - (DTW_SMAX + DTW_DELTA) * dt - li) / dui * (double)(m - 1);
                        j = est <= 0.0 ? 0 : (est >= (double)(m - 1) ? m - 1 : (int)est);
                        j = max(0, j - 2);
                        while (j > 0 && !(slope_of(j - 1) > DTW_SMAX + DTW_DELTA)) --j;
                    }
                    while (j < m && slope_of(j) > DTW_SMAX + DTW_DELTA) ++j;
                    double best = DTW_HUGE;
                    int bj = 0;
                    for (; j < m; ++j) {
                        const double s = slope_of(j);
                        if (s < DTW_SMIN - DTW_DELTA) break;
                        const double fj = fcur[j];
                        if (!(fj < DTW_HUGE)) continue;
                        const double pc = dadd(fj, dmul(dt, dadd(dmul(a.rinst, dmul(s, s)), nu)));
                        if (pc < best) {
                            best = pc;
                            bj = j;
                        }
                    }
                    fnext[k] = best;
                    path[(size_t)(i + 1) * m + k] = (unsigned short)bj;
                }
                __syncthreads();
                double* tmp = fcur;
                fcur = fnext;
                fnext = tmp;
            }
            // traceback (:196-209)
            if (threadIdx.x == 0) {
                const double cost = fcur[jc];
                int j = jc;
                for (int i = n - 1; i >= 0; --i) {
                    T[i] = dadd(L[i], dmul(dsub(U[i], L[i]), lin[j]));
                    if (i > 0) j = path[(size_t)i * m + j];
                }
                s_cost = cost;
            }
            __syncthreads();
            const double cost = s_cost;
            if (fabs(cost - cost_prev) <= a.epsabs + a.epsrel * cost_prev) break;
            cost_prev = cost;
            __syncthreads();
        }
        // tau = (tau - linspace(0, 1, n)) (n - 1), in seconds (:232, :810), on every component's row
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double lin32 = (double)((float)i / (float)(n - 1));
            const float v = (float)dmul(dmul(dsub(T[i], lin32), (double)(n - 1)), (double)a.dd);
            for (int c = 0; c < a.vc; ++c) {
                int lo, hi;
                const int rc = comp_row(a, g, r, c, lo, hi);
                if (rc < hi) a.tau[(size_t)rc * n + i] = v;
            }
        }
        __syncthreads();
    }
}

// single-precision linear interpolation on the grid i dd, zero outside
__device__ float interp_zero_f(const double* x, int n, float dd, float q) {
    const float tl = (float)(n - 1) * dd;
    if (q < 0.f || q > tl) return 0.f;
    int i0 = min(max((int)floorf(q / dd), 0), n - 2);
    while (i0 > 0 && (float)i0 * dd > q) --i0;
    while (i0 < n - 2 && (float)(i0 + 1) * dd <= q) ++i0;
    const float t0 = (float)i0 * dd, t1 = (float)(i0 + 1) * dd;
    const float w = (q - t0) / (t1 - t0);
    return (float)x[i0] * (1.f - w) + (float)x[i0 + 1] * w;
}

// quality weights (:838-905), one CTA per trace (dtw-vector: per receiver, the
// components' windowed correlations summed before |q|^0.2, q on every component's row)
__global__ void __launch_bounds__(256) k_dtw_quality(DtwArgs a) {
    __shared__ double red[32];
    const int r = blockIdx.x, n = a.n;
    const int g = gather_of(a, r);
    if (g % a.vc != 0) return;
    bool lv = false;
    for (int c = 0; c < a.vc; ++c) {
        int lo, hi;
        const int rc = comp_row(a, g, r, c, lo, hi);
        lv = lv || (rc < hi && a.live[rc]);
    }
    float* q = a.q + (size_t)r * n;
    float* dw = a.dw + (size_t)r * n;
    auto spread = [&]() {  // copy q to the other components' rows
        __syncthreads();
        for (int c = 1; c < a.vc; ++c) {
            int lo, hi;
            const int rc = comp_row(a, g, r, c, lo, hi);
            if (rc < hi)
                for (int i = threadIdx.x; i < n; i += blockDim.x) a.q[(size_t)rc * n + i] = q[i];
        }
    };
    if (!lv || a.form == 1) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = 1.f;
        spread();
        return;
    }
    const int nw = (int)floor(fabs((double)(a.tlag / a.dd)) + 0.5);  // nint(tlag_max / dd)
    for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = 0.f;
    for (int c = 0; c < a.vc; ++c) {
        int lo, hi;
        const int rc = comp_row(a, g, r, c, lo, hi);
        if (rc >= hi || !a.live[rc]) continue;  // a dropped component is a zero trace: it adds nothing
        const double* ds = a.dsn + (size_t)rc * n;
        const double* dob = a.dob + (size_t)rc * n;
        const float* tau = a.tau + (size_t)rc * n;
        float* dwc = a.dw + (size_t)rc * n;
        double s1 = 0.0, s2 = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float tg = (float)i * a.dd;
            const float v = interp_zero_f(dob, n, a.dd, tau[i] + tg);
            dwc[i] = v;
            s1 += ds[i] * ds[i];
            s2 += (double)v * (double)v;
        }
        s1 = block_sum_d(s1, red);
        s2 = block_sum_d(s2, red);
        float eta = (float)(fmax(sqrt(s1), sqrt(s2)) * (double)1.0e-2f);
        if (eta == 0.f) eta = 1.0e-9f;
        __syncthreads();
        // windowed normalised correlation, summed over the components
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int l0 = max(0, j - nw), l1 = min(n - 1, j + nw);
            double uv = 0.0, uu = 0.0, vv = 0.0;
            for (int i = l0; i <= l1; ++i) {
                const double u = (double)(float)ds[i], v = (double)dwc[i];
                uv += u * v;
                uu += u * u;
                vv += v * v;
            }
            q[j] += (float)(uv / (sqrt(uu) * sqrt(vv) + (double)eta));
        }
        __syncthreads();
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) q[j] = powf(fabsf(q[j]), 0.2f);
    __syncthreads();
    // 7-sample median (truncated at the ends) into dw
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        float w[7];
        const int lo = max(0, j - 3), hi = min(n - 1, j + 3), c = hi - lo + 1;
        for (int i = 0; i < c; ++i) w[i] = q[lo + i];
        for (int i = 1; i < c; ++i) {
            const float v = w[i];
            int k = i - 1;
            while (k >= 0 && w[k] > v) { w[k + 1] = w[k]; --k; }
            w[k + 1] = v;
        }
        dw[j] = (c & 1) ? w[c / 2] : 0.5f * (w[c / 2 - 1] + w[c / 2]);
    }
    __syncthreads();
    // Gaussian of 3 samples truncated at 9, end samples replicated (double),
    // normalised by its L2 norm, rescaled to [0, 1]; NaN / Inf -> 0
    double wsum = 0.0;
    for (int k = -9; k <= 9; ++k) wsum += exp(-0.5 * (double)(k * k) / 9.0);
    auto gauss = [&](int j) {
        double acc = 0.0;
        for (int k = -9; k <= 9; ++k) acc += exp(-0.5 * (double)(k * k) / 9.0) / wsum * (double)dw[min(max(j + k, 0), n - 1)];
        return acc;
    };
    double sq = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double g = gauss(j);
        sq += g * g;
    }
    const double nrm = sqrt(block_sum_d(sq, red));
    double lo = DTW_HUGE, hi = -DTW_HUGE;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double v = gauss(j) / nrm;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    lo = block_minmax_d(lo, red, false);
    hi = block_minmax_d(hi, red, true);
    double qmax = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double v = (gauss(j) / nrm - lo) / (hi - lo);
        if (!isfinite(v)) v = 0.0;
        const float f = (float)v;
        q[j] = f;
        qmax = fmax(qmax, (double)fabsf(f));
    }
    __syncthreads();
    qmax = block_minmax_d(qmax, red, true);
    if (qmax == 0.0)
        for (int j = threadIdx.x; j < n; j += blockDim.x) q[j] = 1.f;
    spread();
}

// interp_to(x, nn, 'cubic') of the normalised traces (:765-768): Keys cubic
// convolution (a = -1/2; indices clamped to the trace, zero outside it, 1e-4
// snap to a node) in float64 without fused multiply-adds, rounded to single
// precision as the reference's traces are
__global__ void k_dtw_resample(const double* __restrict__ in, int n, double din, double* __restrict__ out, int nn,
                               double dout, int ntr) {
    const size_t tot = (size_t)ntr * nn;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < tot; o += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(o / nn), i = (int)(o % nn);
        double x = __ddiv_rn(dmul((double)i, dout), din);
        const double xr = rint(x);
        if (fabs(dsub(x, xr)) <= 1e-4) x = xr;
        double v = 0.0;
        if (x >= 0.0 && x <= (double)(n - 1)) {
            const int j0 = (int)floor(x);
            const double u = dsub(x, (double)j0), u2 = dmul(u, u), u3 = dmul(u2, u);
            const double w0 = dmul(0.5, dsub(dadd(-u3, dmul(2.0, u2)), u));
            const double w1 = dmul(0.5, dadd(dsub(dmul(3.0, u3), dmul(5.0, u2)), 2.0));
            const double w2 = dmul(0.5, dadd(dadd(dmul(-3.0, u3), dmul(4.0, u2)), u));
            const double w3 = dmul(0.5, dsub(u3, u2));
            const double* row = in + (size_t)r * n;
            v = dadd(dadd(dadd(dmul(w0, row[max(j0 - 1, 0)]), dmul(w1, row[j0])), dmul(w2, row[min(j0 + 1, n - 1)])),
                     dmul(w3, row[min(j0 + 2, n - 1)]));
        }
        out[o] = (double)(float)v;
    }
}

__device__ __forceinline__ int sgn(double v) { return (v > 0.0) - (v < 0.0); }

// slope of the monotone cubic at node k of a row on the unit grid: the harmonic
// mean of the neighbouring secants inside (zero where they differ in sign or one
// is zero), the three-point formula at the ends limited to keep the secant's
// sign and at most three times it (Fritsch and Carlson 1980)
__device__ double pchip_slope(const float* r, int nn, int k) {
    if (nn == 2) return dsub((double)r[1], (double)r[0]);
    if (k == 0 || k == nn - 1) {
        const double a = k == 0 ? dsub((double)r[1], (double)r[0]) : dsub((double)r[nn - 1], (double)r[nn - 2]);
        const double b = k == 0 ? dsub((double)r[2], (double)r[1]) : dsub((double)r[nn - 2], (double)r[nn - 3]);
        const double a3 = dmul(3.0, a);
        const double d = __ddiv_rn(dsub(a3, b), 2.0);
        if (sgn(d) != sgn(a)) return 0.0;
        if (sgn(a) != sgn(b) && fabs(d) > fabs(a3)) return a3;
        return d;
    }
    const double a = dsub((double)r[k], (double)r[k - 1]), b = dsub((double)r[k + 1], (double)r[k]);
    if (a == 0.0 || b == 0.0 || (a > 0.0) != (b > 0.0)) return 0.0;
    return __ddiv_rn(2.0, dadd(__ddiv_rn(1.0, a), __ddiv_rn(1.0, b)));
}

// interp_to(x, [n, nr], method=['pchip', 'nearest']) (:907-911): rows of nn
// samples at din onto n samples at dout (x = i dout / din, 1e-4 snap to a node,
// clamped to the grid), float64 without fused multiply-adds, single-precision out
__global__ void k_dtw_pchip(const float* __restrict__ in, int nn, double din, float* __restrict__ out, int n,
                            double dout, int ntr) {
    const size_t tot = (size_t)ntr * n;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < tot; o += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(o / n), i = (int)(o % n);
        double x = __ddiv_rn(dmul((double)i, dout), din);
        const double xr = rint(x);
        if (fabs(dsub(x, xr)) <= 1e-4) x = xr;
        x = fmin(fmax(x, 0.0), (double)(nn - 1));
        const int j0 = min((int)floor(x), nn - 2);
        const double u = dsub(x, (double)j0), w = dsub(1.0, u), ww = dmul(w, w), uu = dmul(u, u);
        const double h00 = dmul(dadd(1.0, dmul(2.0, u)), ww), h10 = dmul(u, ww);
        const double h01 = dmul(uu, dsub(3.0, dmul(2.0, u))), h11 = dmul(uu, dsub(u, 1.0));
        const float* row = in + (size_t)r * nn;
        const double v = dadd(dadd(dadd(dmul(h00, (double)row[j0]), dmul(h10, pchip_slope(row, nn, j0))),
                                   dmul(h01, (double)row[j0 + 1])),
                              dmul(h11, pchip_slope(row, nn, j0 + 1)));
        out[o] = (float)v;
    }
}

__device__ __forceinline__ double keys_at(const float* x, int n, double p) {
    if (fabs(p - rint(p)) <= 1e-4) p = rint(p);
    if (p < 0.0 || p > (double)(n - 1)) return 0.0;
    const int j0 = (int)floor(p);
    const double u = p - j0, u2 = u * u, u3 = u2 * u;
    const double w0 = 0.5 * (-u3 + 2 * u2 - u), w1 = 0.5 * (3 * u3 - 5 * u2 + 2);
    const double w2 = 0.5 * (-3 * u3 + 4 * u2 + u), w3 = 0.5 * (u3 - u2);
    return w0 * x[max(j0 - 1, 0)] + w1 * x[j0] + w2 * x[min(j0 + 1, n - 1)] + w3 * x[min(j0 + 2, n - 1)];
}

// adjoint source and misfit (:917-978), one CTA per trace; warped obs staged in dw
__global__ void __launch_bounds__(256) k_dtw_adjoint(DtwArgs a) {
    __shared__ double red[32];
    const int r = blockIdx.x, n = a.n;
    float* adj = a.adj ? a.adj + (size_t)r * n : nullptr;
    const int g = gather_of(a, r);
    bool lv = false;
    for (int c = 0; c < a.vc; ++c) {
        int lo, hi;
        const int rc = comp_row(a, g, r, c, lo, hi);
        lv = lv || (rc < hi && a.live[rc]);
    }
    if (!a.live[r]) {
        // a dropped trace (dtw-vector: a dropped component of a kept receiver is a
        // zero trace: no adjoint, its share of the receiver's phase misfit)
        if (adj)
            for (int i = threadIdx.x; i < n; i += blockDim.x) adj[i] = 0.f;
        double mph = 0.0;
        if (lv && a.form != 1) {
            const float* tau = a.tau + (size_t)r * n;
            const float* q = a.q + (size_t)r * n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) mph += (double)q[i] * (double)tau[i] * (double)tau[i];
            mph = block_sum_d(mph, red);
        }
        if (threadIdx.x == 0 && a.tm)
            a.tm[r] = !lv ? 0.0 : a.form == 0 ? mph / a.vc : a.form == 1 ? 0.0 : mph * (1.0 + (double)a.amp_weight);
        return;
    }
    const float* obs = a.obs + (size_t)r * n;
    const float* syn = a.syn + (size_t)r * n;
    const float* tau = a.tau + (size_t)r * n;
    const float* q = a.q + (size_t)r * n;
    float* dw = a.dw + (size_t)r * n;
    double mph = 0.0, ma = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float pos = (tau[i] + (float)i * a.dd) / a.dd;
        const double w = keys_at(obs, n, (double)pos);
        dw[i] = (float)w;
        const double ti = tau[i];
        mph += (double)q[i] * ti * ti;
        const double rr = (double)syn[i] - w;
        ma += rr * rr;
    }
    mph = block_sum_d(mph, red);
    ma = block_sum_d(ma, red);
    // dtw-vector: the receiver's phase misfit is shared by its component rows
    if (threadIdx.x == 0 && a.tm)
        a.tm[r] = a.form == 0 ? mph / a.vc : a.form == 1 ? ma : mph * (1.0 + (double)a.amp_weight);
    if (!adj) return;
    const double dd = a.dd;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        // the warped trace is recomputed in double for the derivative's neighbours
        auto wv = [&](int k) {
            const float pos = (tau[k] + (float)k * a.dd) / a.dd;
            return keys_at(obs, n, (double)pos);
        };
        double der;
        if (i == 0) der = wv(1) - wv(0);
        else if (i == n - 1) der = wv(n - 1) - wv(n - 2);
        else der = (wv(i + 1) - wv(i - 1)) * 0.5;
        const double ph = (double)q[i] * (double)tau[i] * der / dd;
        const double res = (double)syn[i] - wv(i);
        double v;
        if (a.form == 0) v = ph;
        else if (a.form == 1) v = res;
        else v = ph + (double)a.amp_weight * mph / (ma + 1.1754943508222875e-38) * res;
        adj[i] = (float)v;
    }
}

}  // namespace

void AdjointSource::run_dtw(const owl_misfit_opts& o, int ngather, int nt, int ntr, const float* syn, const float* obs,
                            float* adj, double* tm, float* tau_out, cudaStream_t s) {
    OWL_CHECK(o.dt > 0.f, OWL_ERR_INVALID, "the DTW misfit needs the sample interval dt");
    OWL_CHECK(nt >= 3 && nt <= 16384, OWL_ERR_INVALID, "DTW traces must have 3 .. 16384 samples");
    const float tlag = o.tlag_max > 0.f ? o.tlag_max : 0.1f * (float)(nt - 1) * o.dt;
    // adj_nt (:744-750): the shifts and quality weights are computed on the
    // normalised traces resampled to ns samples over the same span
    const bool rs = o.adj_nt > 0 && o.adj_nt != nt;
    const int ns = rs ? o.adj_nt : nt;
    OWL_CHECK(ns >= 3 && ns <= 16384, OWL_ERR_INVALID, "DTW: adj_nt must lie in 3 .. 16384");
    const float dds = rs ? ((float)(nt - 1) * o.dt) / (float)(ns - 1) : o.dt;
    // m = nint(2 tlag_max / dd) + 1, odd (:795, solve_gdtw :92-96)
    const float x = (2.0f * tlag) / dds;
    int m = (int)std::floor(std::fabs((double)x) + 0.5) + 1;
    if (m % 2 == 0) ++m;
    OWL_CHECK(m >= 3 && m <= 4095, OWL_ERR_INVALID, "DTW: 2 tlag_max / dt + 1 must lie in 3 .. 4095 candidates");
    OWL_CHECK(o.dtw_form >= 0 && o.dtw_form <= 2, OWL_ERR_INVALID, "bad dtw_form");
    OWL_CHECK(o.dtw_trc >= 0 && o.dtw_niter >= 0, OWL_ERR_INVALID, "bad DTW options");
    DtwArgs a{};
    a.n = nt;
    a.m = m;
    a.ntr = ntr;
    a.ngather = ngather;
    a.niter = o.dtw_niter > 0 ? o.dtw_niter : 5;
    a.trc = o.dtw_trc;
    a.form = o.dtw_form;
    a.gptr = gptr.p;
    a.live = live.p;
    a.syn = syn;
    a.obs = obs;
    a.nrm = nrm.p;
    a.vc = o.misfit == OWL_MISFIT_DTW_VECTOR ? std::max(1, o.ncomp) : 1;
    auto dflt = [](float v, float d) { return v == 0.f ? (double)d : (v < 0.f ? 0.0 : (double)v); };
    a.rinst = dflt(o.dtw_rinst, 0.1f);
    a.rcuml = dflt(o.dtw_rcuml, 1.0f);
    a.epsabs = dflt(o.dtw_epsabs, 1.0e-2f);
    a.epsrel = dflt(o.dtw_epsrel, 1.0e-3f);
    a.power = o.dtw_loss_power > 0.f ? (double)o.dtw_loss_power : 0.5;
    a.amp_weight = o.dtw_amp_weight != 0.f ? std::max(0.f, o.dtw_amp_weight) : 1.0f;
    a.dd = o.dt;
    a.tlag = tlag;
    const size_t nn = (size_t)ntr * nt;
    dsn.reserve(nn);
    dob.reserve(nn);
    qw.reserve(nn);
    warp.reserve((size_t)ntr * std::max(nt, ns));
    DevBuf<float> tmp_tau;
    if (!tau_out) {
        tmp_tau.reserve(nn);
        tau_out = tmp_tau.p;
    }
    a.dsn = dsn.p;
    a.dob = dob.p;
    a.q = qw.p;
    a.dw = warp.p;
    a.tau = tau_out;
    a.adj = adj;
    a.tm = tm;
    int dev_id = 0, nsm = 0;
    OWL_CUDA(cudaGetDevice(&dev_id));
    OWL_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id));
    // back-pointer tables of the traces solved at once: at most 2 GiB
    const size_t per = (size_t)ns * m * sizeof(unsigned short);
    const size_t cap = std::max<size_t>(1, ((size_t)2 << 30) / per);
    const int grid = (int)std::max<size_t>(1, std::min<size_t>({(size_t)ntr, (size_t)nsm * 4, cap}));
    path.reserve((size_t)grid * ns * m);
    band.reserve((size_t)grid * 3 * ns);
    a.path = path.p;
    a.band = band.p;
    if (a.vc > 1) {
        vnrm.reserve(2 * (size_t)ntr);
        k_dtw_vnorm<<<(ntr + 127) / 128, 128, 0, s>>>(a, vnrm.p);
        a.vnrm = vnrm.p;
        launches++;
    }
    k_dtw_normalise<<<(int)std::min<size_t>((nn + 255) / 256, (size_t)nsm * 32), 256, 0, s>>>(a);
    // the shift computation's view: ns samples at dds
    DtwArgs b = a;
    DevBuf<double> rsn, rob;
    DevBuf<float> rtau, rq;
    if (rs) {
        const size_t nr = (size_t)ntr * ns;
        rsn.reserve(nr);
        rob.reserve(nr);
        rtau.reserve(nr);
        rq.reserve(nr);
        const int gr = (int)std::min<size_t>((nr + 255) / 256, (size_t)nsm * 32);
        k_dtw_resample<<<gr, 256, 0, s>>>(dsn.p, nt, (double)o.dt, rsn.p, ns, (double)dds, ntr);
        k_dtw_resample<<<gr, 256, 0, s>>>(dob.p, nt, (double)o.dt, rob.p, ns, (double)dds, ntr);
        launches += 2;
        b.n = ns;
        b.dd = dds;
        b.dsn = rsn.p;
        b.dob = rob.p;
        b.tau = rtau.p;
        b.q = rq.p;
    }
    const size_t smem = (size_t)3 * m * sizeof(double);
    OWL_CUDA(cudaFuncSetAttribute(k_dtw_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_dtw_solve<<<grid, 256, smem, s>>>(b);
    k_dtw_quality<<<ntr, 256, 0, s>>>(b);
    if (rs) {
        // shifts and weights back to the trace length (:907-911)
        const int gr = (int)std::min<size_t>((nn + 255) / 256, (size_t)nsm * 32);
        k_dtw_pchip<<<gr, 256, 0, s>>>(rtau.p, ns, (double)dds, a.tau, nt, (double)o.dt, ntr);
        k_dtw_pchip<<<gr, 256, 0, s>>>(rq.p, ns, (double)dds, a.q, nt, (double)o.dt, ntr);
        launches += 2;
    }
    k_dtw_adjoint<<<ntr, 256, 0, s>>>(a);
    OWL_LAUNCH_CHECK();
    launches += 4;
    OWL_CUDA(cudaStreamSynchronize(s));
}

}  // namespace owl
