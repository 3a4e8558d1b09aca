// vec4.cuh -- helpers of the four-cell-per-thread stencil kernels (2D): a
// thread owns cells x .. x + 3 of one row, x - R a multiple of 4, so every row
// access is one 16-byte float4.
#pragma once

#include <cuda_runtime.h>

namespace owl {

// f[x - R .. x + R + 3] as R / 2 + 1 float4 loads (f points at cell x): the x
// arms of the four cells' stencils, P-type (x + k, x + 1 - k) and M-type
// (x + k - 1, x - k) alike
template <int R>
__device__ __forceinline__ void win4(const float* f, float* w) {
#pragma unroll
    for (int q = 0; q < R / 2 + 1; ++q) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(f - R + 4 * q));
        w[4 * q] = t.x; w[4 * q + 1] = t.y; w[4 * q + 2] = t.z; w[4 * q + 3] = t.w;
    }
}
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float f4at(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ void f4set(float4& v, int c, float s) {
    if (c == 0) v.x = s; else if (c == 1) v.y = s; else if (c == 2) v.z = s; else v.w = s;
}
// all four cells, or the first n one by one
__device__ __forceinline__ void st4n(float* p, const float4& v, int n) {
    if (n == 4) {
        *reinterpret_cast<float4*>(p) = v;
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (c < n) p[c] = f4at(v, c);
    }
}

// the same with evict-first (streaming) stores and loads, for data written once
// and read once a segment later (the stored stencil terms): they pass through
// L2 without displacing the wavefields that stay resident there between launches
__device__ __forceinline__ void st4n_cs(float* p, const float4& v, int n) {
    if (n == 4) {
        __stcs(reinterpret_cast<float4*>(p), v);
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (c < n) __stcs(p + c, f4at(v, c));
    }
}
__device__ __forceinline__ float4 ldcs4(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }

}  // namespace owl
