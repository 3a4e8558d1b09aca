// common.cuh -- shared host/device utilities of the B200 SSG library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/owl_ssg.h"

namespace owl {

// ----------------------------------------------------------------------------
// errors: every failure becomes an OwlError carrying an ABI status code; the
// C entry points catch it and return the code (never abort the process).
// ----------------------------------------------------------------------------
struct OwlError : std::runtime_error {
    int code;
    OwlError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define OWL_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? OWL_ERR_OOM : OWL_ERR_CUDA;          \
            throw ::owl::OwlError(code_, std::string(#call) + ": " + cudaGetErrorString(e_) +    \
                                             " (" __FILE__ ":" + std::to_string(__LINE__) + ")"); \
        }                                                                                        \
    } while (0)

#define OWL_CHECK(cond, code, msg)                              \
    do {                                                        \
        if (!(cond)) throw ::owl::OwlError((code), (msg));      \
    } while (0)

#define OWL_LAUNCH_CHECK() OWL_CUDA(cudaGetLastError())

// ----------------------------------------------------------------------------
// Programmatic dependent launch: a kernel launched with launch_pdl may start
// while the kernel before it on the stream drains; it must call pdl_prologue()
// before its first global read (griddepcontrol.wait returns once the previous
// grid has completed and its writes are visible), and the call also lets the
// next kernel be scheduled. OWL_NO_PDL=1 in the environment launches plainly.
// ----------------------------------------------------------------------------
__device__ __forceinline__ void pdl_prologue() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

bool pdl_enabled();

template <typename... KArgs, typename... Args>
void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    OWL_CUDA(cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...));
}

// ----------------------------------------------------------------------------
// grow-only device buffer. Keeping the pointer stable across calls lets the
// captured CUDA graphs be replayed without re-instantiation.
// ----------------------------------------------------------------------------
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;  // capacity in elements
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // returns true if the pointer changed
    bool reserve(size_t count) {
        if (count <= n && p) return false;
        release();
        size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        const cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            // a failed allocation leaves the handle usable: clear the runtime's
            // last error so that the next launch check does not report it again
            p = nullptr;
            (void)cudaGetLastError();
            OWL_CUDA(e);
        }
        n = std::max<size_t>(count, 1);
        return true;
    }
    void zero(cudaStream_t s, size_t count) { OWL_CUDA(cudaMemsetAsync(p, 0, count * sizeof(T), s)); }
    void upload(const T* h, size_t count, cudaStream_t s) {
        reserve(count);
        if (count) OWL_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// ----------------------------------------------------------------------------
// point operators (source injection, receiver sampling, adjoint-source
// injection) in CSR form. Each item (a source of one shot, a receiver, a
// unique target cell) owns a contiguous run of taps (field slot, offset, w).
// ----------------------------------------------------------------------------
struct Tap {
    int field;   // field slot within the medium's state (e.g. 0 = p, 1 = vx, 2 = vz)
    int shot;    // shot index inside the batch
    int64_t off; // offset inside one shot's field (z * pitch + x)
    float w;     // weight
    int item;    // owning item for scatter tables (receiver / source index)
};

struct HostCSR {
    std::vector<int> ptr{0};
    std::vector<int> field, shot, item;
    std::vector<long long> off;
    std::vector<float> w;
    void push(const Tap& t) {
        field.push_back(t.field);
        shot.push_back(t.shot);
        item.push_back(t.item);
        off.push_back(t.off);
        w.push_back(t.w);
    }
    void close_item() { ptr.push_back((int)field.size()); }
    int nitems() const { return (int)ptr.size() - 1; }
    int ntaps() const { return (int)field.size(); }
};

struct DevCSR {
    DevBuf<int> ptr, field, shot, item;
    DevBuf<long long> off;
    DevBuf<float> w;
    int nitems = 0, ntaps = 0;
    void upload(const HostCSR& h, cudaStream_t s) {
        nitems = h.nitems();
        ntaps = h.ntaps();
        ptr.upload(h.ptr.data(), h.ptr.size(), s);
        field.upload(h.field.data(), h.field.size(), s);
        shot.upload(h.shot.data(), h.shot.size(), s);
        item.upload(h.item.data(), h.item.size(), s);
        off.upload(h.off.data(), h.off.size(), s);
        w.upload(h.w.data(), h.w.size(), s);
    }
};

// device view of a CSR table
struct CSRView {
    const int* ptr;
    const int* field;
    const int* shot;
    const int* item;
    const long long* off;
    const float* w;
    int nitems;
};

inline CSRView view(const DevCSR& d) {
    return CSRView{d.ptr.p, d.field.p, d.shot.p, d.item.p, d.off.p, d.w.p, d.nitems};
}

// FD coefficients of the optimised staggered scheme (src/lib/module_fdcoef.f90:23-30, 59-62)
inline const float* fd_coefs(int half) {
    static const float c4[4] = {0.1217990e+1f, -0.9382142e-1f, 0.1507536e-1f, -0.1700324e-2f};
    static const float c8[8] = {0.1259312e+1f, -0.1280347e+0f, 0.3841945e-1f, -0.1473229e-1f,
                                0.5924913e-2f, -0.2248618e-2f, 0.7179226e-3f, -0.1400855e-3f};
    return half == 8 ? c8 : c4;
}

// CFS-PML coefficient of one node, damp_coef (src/solver/acoustic_iso_2d/module_cfspml.f90:37-56),
// evaluated in single precision in the reference's operation order.
void damp_coef(float bdvp, float d, float dist, int pml, float dt, float alphamax, float& a, float& b);

// 1D CFS-PML coefficients at integer and half nodes over the padded compute
// range [-pml+1, n+pml] (module_cfspml.f90:95-131), mapped to storage index
// i + pml + R - 1 with length `len`.
struct Pml1DHost {
    std::vector<float> ai, bi, ah, bh;
};
Pml1DHost build_pml_1d(int n, int pml, int R, int len, float d, float dt, float pmlvp, float alphamax);

int nint_f(float v);  // Fortran nint

// device-time measurement of a call
struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit EventTimer(cudaStream_t st) : s(st) {
        OWL_CUDA(cudaEventCreate(&a));
        OWL_CUDA(cudaEventCreate(&b));
        OWL_CUDA(cudaEventRecord(a, s));
    }
    double stop_ms() {
        OWL_CUDA(cudaEventRecord(b, s));
        OWL_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        OWL_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// simple cached CUDA graph of a launch sequence
struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> sig;
    ~GraphCache() { reset(); }
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        sig.clear();
    }
};

}  // namespace owl
