// su.cu -- SU trace records (240-byte header + ns float32 samples, native
// byte order) assembled and taken apart on the GPU, so that seismograms and
// adjoint sources move between files and device memory in one copy each
// (the su type's output / load, src/lib/module_su.f90).
//
// A record is 60 + ns four-byte words: the header, then the samples; the
// header of every trace is the same template (ns at byte 114, dt in
// microseconds at 116, d1 at 180, as the Python writer sets them).
#include "engine.cuh"

namespace owl {

namespace {

__global__ void k_su_encode(const unsigned* __restrict__ hdr, const unsigned* __restrict__ data, int ntr, int ns,
                            unsigned* __restrict__ out) {
    const long long nw = (long long)ntr * (60 + ns);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / (60 + ns);
        const int w = (int)(i - r * (60 + ns));
        out[i] = w < 60 ? hdr[w] : data[r * ns + (w - 60)];
    }
}

__global__ void k_su_decode(const unsigned* __restrict__ in, int ntr, int ns, unsigned* __restrict__ data) {
    const long long n = (long long)ntr * ns;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / ns;
        data[i] = in[r * (60 + ns) + 60 + (i - r * ns)];
    }
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

}  // namespace

void su_encode(const unsigned char* header, const float* traces, int ntr, int ns, unsigned char* out, bool dev,
               cudaStream_t s) {
    const size_t rec = 240 + 4 * (size_t)ns, n = (size_t)ntr * rec;
    DevBuf<unsigned> h, d, o;
    h.upload(reinterpret_cast<const unsigned*>(header), 60, s);  // the template is host memory
    const unsigned* pd = reinterpret_cast<const unsigned*>(traces);
    unsigned* po = reinterpret_cast<unsigned*>(out);
    if (!dev) {
        d.upload(pd, (size_t)ntr * ns, s);
        o.reserve(n / 4);
        pd = d.p;
        po = o.p;
    }
    k_su_encode<<<grid_for((long long)(n / 4)), 256, 0, s>>>(h.p, pd, ntr, ns, po);
    OWL_LAUNCH_CHECK();
    if (!dev) OWL_CUDA(cudaMemcpyAsync(out, po, n, cudaMemcpyDeviceToHost, s));
    OWL_CUDA(cudaStreamSynchronize(s));
}

void su_decode(const unsigned char* in, int ntr, int ns, float* traces, bool dev, cudaStream_t s) {
    const size_t rec = 240 + 4 * (size_t)ns, n = (size_t)ntr * rec;
    DevBuf<unsigned> i, d;
    const unsigned* pi = reinterpret_cast<const unsigned*>(in);
    unsigned* pd = reinterpret_cast<unsigned*>(traces);
    if (!dev) {
        i.upload(pi, n / 4, s);
        d.reserve((size_t)ntr * ns);
        pi = i.p;
        pd = d.p;
    }
    k_su_decode<<<grid_for((long long)ntr * ns), 256, 0, s>>>(pi, ntr, ns, pd);
    OWL_LAUNCH_CHECK();
    if (!dev) OWL_CUDA(cudaMemcpyAsync(traces, pd, (size_t)ntr * ns * 4, cudaMemcpyDeviceToHost, s));
    OWL_CUDA(cudaStreamSynchronize(s));
}

}  // namespace owl
