// tma.cuh -- tiled TMA loads into shared memory with mbarrier completion, for
// the z-marching stencil kernels (sm_100a).
//
// Every load is a plain per-CTA cp.async.bulk.tensor of this GPU's own memory
// into the issuing CTA's shared memory (no cluster multicast). A plane's tiles
// complete on one mbarrier per ring stage: one thread arms it with the bytes of
// the plane's tiles (arrive.expect_tx) and issues the loads; every thread waits
// on the stage's phase. Each wait is bounded: after TMA_SPIN_LIMIT polls it
// records the failure in a device flag and returns false, and the kernel then
// drains what it issued (bounded again) and leaves; the host turns the flag into
// OWL_ERR_TIMEOUT.
//
// The innermost (x) coordinate of every load is a multiple of 4 floats (16
// bytes) and the box's x extent a multiple of 16 bytes; the host checks the
// tensor maps' bases and strides (16-byte multiples) when it encodes them.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace owl {

constexpr unsigned TMA_SPIN_LIMIT = 1u << 20;  // polls of one wait (each try_wait may suspend for a while)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the async proxy (TMA)
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the phase `parity` of a barrier; false (and *err set) when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err) {
    for (unsigned i = 0; i < TMA_SPIN_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, 1);
    return false;
}

// 3D / 4D / 5D tiled loads (coordinates innermost first) completing on `bar`
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// ---- host side: tensor maps of float32 arrays ------------------------------
// rank <= 5 dimensions (innermost first), byte strides of dimensions 1..rank-1,
// box extents; out-of-range elements load as zero
CUtensorMap make_tensor_map_f32(const float* base, int rank, const uint64_t* dims, const uint64_t* stride_bytes,
                                const uint32_t* box);

}  // namespace owl
