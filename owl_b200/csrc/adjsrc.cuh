// adjsrc.cuh -- data-domain misfits and adjoint sources on the GPU
// (compute_adjoint_source, src/inverse/module_inversion_adjoint_source.f90:985-1277).
#pragma once

#include "common.cuh"

namespace owl {

// Bluestein tables of a length-N DFT computed as an M-point power-of-two
// circular convolution (M >= 2N - 1): chirp c_n = exp(-i pi n^2 / N), the
// M-point FFT of the conjugate chirp filter, and the M/2 twiddles exp(-2 pi i j / M).
struct DftTables {
    int N = 0, M = 0, logM = 0;
    DevBuf<float2> chirp, bf, tw;
    void build(int n, cudaStream_t s);
};

struct AdjointSource {
    DftTables hil, awi, awl;  // awl: the local and space-time adaptive misfits
    DevBuf<int> gptr;
    DevBuf<unsigned char> live;
    DevBuf<double> nrm, gmax;
    DevBuf<float> pen, ramp, scratch;
    DevBuf<float2> cscratch;
    DevBuf<double> dsn, dob, band, vnrm;  // DTW: normalised traces, per-CTA search bands, receiver norms
    DevBuf<float> qw, warp;         // DTW: quality weights, warped traces
    DevBuf<unsigned short> path;    // DTW: per-CTA back-pointers of the dynamic program
    long long launches = 0;

    // Misfit and adjoint source of every trace (rows of nt samples) of ngather
    // contiguous gathers, all pointers on the device except h_gather_ptr.
    // weight_live: per-trace 0 / 1 (or nullptr = all live) before the discard
    // rule. adj, tm (per trace), gm (per gather) may be nullptr; tau (DTW only,
    // may be nullptr) receives the time shifts in seconds, rows like syn.
    void run(const owl_misfit_opts& o, int ngather, const int* h_gather_ptr, int nt, const float* syn,
             const float* obs, const unsigned char* weight_live, float* adj, double* tm, double* gm,
             cudaStream_t s, float* tau = nullptr);
    // the DTW part of run (dtw.cu), after the norms and the discard rule
    void run_dtw(const owl_misfit_opts& o, int ngather, int nt, int ntr, const float* syn, const float* obs,
                 float* adj, double* tm, float* tau, cudaStream_t s);
};

// smallest m >= n with no prime factor above 5 (FLIT next_power_235)
int next_power_235(int n);

}  // namespace owl
