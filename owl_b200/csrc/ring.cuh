// ring.cuh -- asynchronous-copy helpers of the z-marching stencil kernels:
// 16-byte cp.async copies into a shared-memory ring and the per-thread copy
// slots of a tile (computed once per CTA, reused on every plane).
#pragma once

#include <cuda_runtime.h>

namespace owl {

__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = pred ? 16 : 0;  // 0: zero-fill the 16 bytes
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The copies of a tile are the same on every plane but for the plane offset:
// thread t owns elements e = t + 256 k of a ROWS x CH grid of 16-byte chunks,
// stored at dst + 4 e. Their in-plane offsets (-1: outside the field, zero
// fill) are computed once per CTA, so a plane costs one cp.async per element.
template <int ROWS, int CH>
struct TileSlots {
    static constexpr int N = (ROWS * CH + 255) / 256;
    int off[N];
    __device__ __forceinline__ void init(int x0, int y0, int pitch, int NYs) {
        const int tid = threadIdx.y * 32 + threadIdx.x;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int e = tid + 256 * k;
            const int r = e / CH, c = e - r * CH;
            const int xx = x0 + 4 * c, yy = y0 + r;
            const bool ok = e < ROWS * CH && yy >= 0 && yy < NYs && xx >= 0 && xx + 3 < pitch;
            off[k] = ok ? yy * pitch + xx : -1;
        }
    }
    __device__ __forceinline__ void copy(float* dst, const float* plane) const {
        const int tid = threadIdx.y * 32 + threadIdx.x;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int e = tid + 256 * k;
            if (e < ROWS * CH) cp16(dst + 4 * e, off[k] >= 0 ? plane + off[k] : plane, off[k] >= 0);
        }
    }
};

}  // namespace owl
