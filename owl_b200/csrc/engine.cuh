// engine.cuh -- medium-independent engine interface and shared kernels.
#pragma once

#include <vector>

#include "common.cuh"

namespace owl {

// internal adjoint-source kind of Engine::gradient: a data-domain misfit given
// by Engine::mopts (owl_ssg_gradient_misfit)
constexpr int ADJ_MISFIT = 100;

struct Engine {
    owl_ssg_desc desc{};
    owl_misfit_opts mopts{};
    cudaStream_t stream = nullptr;
    float dt_stable_ = 0.f;
    bool model_set = false;
    virtual ~Engine() {}
    virtual void set_model(int nparam, const float* const* fields) = 0;
    virtual void forward(int nshots, const owl_shot* shots, const owl_run_opts& o, float* seis, int mem,
                         owl_run_info& info) = 0;
    virtual void gradient(int nshots, const owl_shot* shots, const float* data, int adj_kind,
                          const owl_run_opts& o, double* misfit, float* grad, float* seis_out, int mem,
                          owl_run_info& info) = 0;
    virtual void kernel_time(int id, int nlaunch, double* avg_ms, double* alg_bytes) = 0;
    virtual void misfit(int nshots, const owl_shot* shots, const float* obs, const owl_run_opts& o, double* misfit,
                        double* trace_misfit, float* seis_out, int mem, owl_run_info& info) = 0;
    virtual void source_gradient(int nshots, const owl_shot* shots, const float* adj, const owl_run_opts& o,
                                 float* stf_grad, int mem, owl_run_info& info) = 0;
    // seismogram sampling of the data (forward output, observed data, adjoint
    // sources): data_nt samples at data_dt from t = 0; data_nt <= 0: the time axis
    int data_nt = 0;
    float data_dt = 0.f;
    // M-PML face ratios of the model (elastic 3D; null elsewhere), the layout of owl_ssg_mpml_ratios
    virtual const std::vector<float>* mpml_faces() const { return nullptr; }
};

Engine* make_ac2d_engine(const owl_ssg_desc& d);
Engine* make_ac3d_engine(const owl_ssg_desc& d);
Engine* make_el2d_engine(const owl_ssg_desc& d);
Engine* make_el3d_engine(const owl_ssg_desc& d);
// refine_nz of the depth-refined free-surface mesh from the model's surface row (el2d.cu)
int el2d_refine_rows(const owl_ssg_desc& d, int nparam, const float* const* fields, float f0_min);
int el3d_refine_rows(const owl_ssg_desc& d, int nparam, const float* const* fields, float f0_min);  // el3d.cu

// -------- shared device helpers (defined in shared.cu) ----------------------

// Kahan-compensated accumulation of v into (s, c)
__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

// one-thread-per-CTA tick of the step counter after all CTAs of a launch have
// read it: the last CTA to finish applies `delta` (the threadfence-reduction
// pattern; no CTA ever waits on another).
__device__ __forceinline__ void tick_last_block(int* d_step, int* d_done, int delta) {
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        __threadfence();
        int prev = atomicAdd(d_done, 1);
        if (prev == (int)(gridDim.x * gridDim.y * gridDim.z) - 1) {
            *d_step += delta;
            *d_done = 0;
            __threadfence();
        }
    }
}

// launches of shared kernels (shared.cu)
void launch_transpose_rec_to_seis(const float* rec, float* seis, int nt, int rtot, cudaStream_t s);
void launch_transpose_seis_to_rec(const float* seis, float* rec, int nt, int rtot, cudaStream_t s);
// residual = syn - obs on live traces (weight != 0); misfit[shot] = sum (obs - syn)^2 (FP64,
// deterministic per-shot block reduction). Traces are indexed by the global receiver id.
void launch_residual_l2(const float* syn, const float* obs, float* res, const unsigned char* live,
                        const int* shot_rec_ptr, int nshots, int nt, int rtot, double* misfit,
                        cudaStream_t s);
void launch_check_finite(const float* f, size_t n, int* flag, cudaStream_t s);
// per-trace FP64 L2 misfits (trace_misfit[rtot]) and their per-shot sums (misfit[nshots])
void launch_trace_misfit(const float* syn, const float* obs, const unsigned char* live, const int* shot_rec_ptr,
                         int nshots, int nt, int rtot, double* trace_misfit, double* misfit, cudaStream_t s);
void launch_fill_f64(double* p, size_t n, double v, cudaStream_t s);
// cubic-convolution resampling of ntr rows (nin samples at din from oin) to nout samples at dout from oout
void launch_resample_rows(const float* in, int nin, double din, double oin, float* out, int nout, double dout,
                          double oout, int ntr, cudaStream_t s);
// per-shot sums of per-trace misfits, in trace order
void launch_shot_misfit(const double* trace_misfit, const int* shot_rec_ptr, int nshots, double* misfit,
                        cudaStream_t s);
// SU records <-> trace rows (su.cu); header: one 240-byte host template; dev: data buffers on the device
void su_encode(const unsigned char* header, const float* traces, int ntr, int ns, unsigned char* out, bool dev,
               cudaStream_t s);
void su_decode(const unsigned char* in, int ntr, int ns, float* traces, bool dev, cudaStream_t s);
// search directions / gradient processing (optim.cu), device pointers
void search_direction(int method, long long n, int nm, const float* const* x, const float* const* g,
                      const float* prev_srch, float* srch, cudaStream_t s);
void grad_process(int op, int n1, int n2, int n3, const float* param, const float* mask, float* f, cudaStream_t s);
// out[i] = (w[i] != 0) (adjsrc.cu)
void launch_nonzero(const float* w, int n, unsigned char* out, cudaStream_t s);

}  // namespace owl
