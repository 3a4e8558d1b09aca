// capi.cu -- extern "C" entry points declared in include/owl_ssg.h.
#include <algorithm>
#include <memory>
#include <mutex>

#include "adjsrc.cuh"
#include "engine.cuh"
#include "vmesh.hpp"

struct owl_ssg {
    std::unique_ptr<owl::Engine> eng;
};

namespace owl {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

template <typename F>
static int guarded(F&& f) {
    try {
        f();
        return OWL_OK;
    } catch (const OwlError& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return OWL_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return OWL_ERR_INVALID;
    }
}

static void check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw OwlError(OWL_ERR_NO_DEVICE, "no CUDA device available");
    }
}

static owl_run_opts opts_or_default(const owl_run_opts* o) {
    owl_run_opts r{};
    if (o) r = *o;
    return r;
}

}  // namespace owl

using namespace owl;

extern "C" {

int owl_ssg_abi_version(void) { return OWL_SSG_ABI_VERSION; }

const char* owl_last_error(void) { return g_last_error.c_str(); }

int owl_ssg_nparam(int medium) {
    switch (medium) {
        case OWL_ACOUSTIC_ISO_2D:
        case OWL_ACOUSTIC_ISO_3D: return 2;
        case OWL_ELASTIC_VHTIORT_2D: return 3;
        case OWL_ELASTIC_VHTIORT_3D: return 10;
        default: return -1;
    }
}

int owl_ssg_desc_nparam(const owl_ssg_desc* d) {
    if (!d) return -1;
    if (d->medium == OWL_ELASTIC_VHTIORT_3D)
        return d->aniso == OWL_ANISO_ISO ? 3 : d->aniso == OWL_ANISO_THOMSEN ? 8 : d->aniso == OWL_ANISO_CIJ ? 10 : -1;
    if (d->medium != OWL_ELASTIC_VHTIORT_2D) return owl_ssg_nparam(d->medium);
    switch (d->aniso) {
        case OWL_ANISO_ISO: return 3;
        case OWL_ANISO_THOMSEN:
        case OWL_ANISO_AT: return 6;
        case OWL_ANISO_CIJ: return 5;
        default: return -1;
    }
}

int owl_ssg_ncomp(int medium) {
    switch (medium) {
        case OWL_ACOUSTIC_ISO_2D:
        case OWL_ACOUSTIC_ISO_3D: return 1;
        case OWL_ELASTIC_VHTIORT_2D: return 2;
        case OWL_ELASTIC_VHTIORT_3D: return 3;
        default: return -1;
    }
}

int owl_vertical_mesh(const owl_ssg_desc* desc, int* nz_mesh, float* z_i, float* z_h, float* dz_i, float* dz_h) {
    return guarded([&] {
        OWL_CHECK(desc && nz_mesh, OWL_ERR_INVALID, "null argument");
        OWL_CHECK(desc->nz >= 1 && desc->pml >= 0 && desc->dz > 0, OWL_ERR_INVALID, "bad grid");
        VMesh m;
        try {
            m = build_vmesh(*desc);
        } catch (const std::invalid_argument& e) {
            throw OwlError(OWL_ERR_INVALID, e.what());
        }
        *nz_mesh = m.nz;
        const int P = desc->pml;
        const size_t L = (size_t)m.nz + 2 * P + 2;
        for (int j = -P; j <= m.nz + P + 1; ++j) {
            const size_t o = (size_t)(j + P);
            if (m.refined) {
                if (z_i) z_i[o] = m.zi[o];
                if (z_h) z_h[o] = m.zh[o];
                if (dz_i) dz_i[o] = m.dzi[o];
                if (dz_h) dz_h[o] = m.dzh[o];
            } else {
                // the uniform grid: row j at (j - 1) dz, half row at (j - 1.5) dz
                if (z_i) z_i[o] = (float)(j - 1) * desc->dz;
                if (z_h) z_h[o] = ((float)(j - 1) - 0.5f) * desc->dz;
                if (dz_i) dz_i[o] = desc->dz;
                if (dz_h) dz_h[o] = desc->dz;
            }
        }
        (void)L;
    });
}

int owl_free_surface_refine_rows(const owl_ssg_desc* desc, int nparam, const float* const* fields, float f0_min,
                                 int* refine_rows) {
    return guarded([&] {
        OWL_CHECK(desc && fields && refine_rows, OWL_ERR_INVALID, "null argument");
        OWL_CHECK(f0_min > 0, OWL_ERR_INVALID, "f0_min must be positive");
        OWL_CHECK(desc->medium == OWL_ELASTIC_VHTIORT_2D || desc->medium == OWL_ELASTIC_VHTIORT_3D,
                  OWL_ERR_UNSUPPORTED, "the refined free-surface mesh belongs to the elastic media");
        *refine_rows = desc->medium == OWL_ELASTIC_VHTIORT_2D ? el2d_refine_rows(*desc, nparam, fields, f0_min)
                                                              : el3d_refine_rows(*desc, nparam, fields, f0_min);
    });
}

int owl_ssg_device_ok(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return 0;
    return p.major == 10 ? 1 : 0;
}

int owl_ssg_create(const owl_ssg_desc* desc, owl_ssg** out) {
    return guarded([&] {
        OWL_CHECK(desc && out, OWL_ERR_INVALID, "null argument");
        *out = nullptr;
        check_device();
        std::unique_ptr<owl_ssg> h(new owl_ssg);
        switch (desc->medium) {
            case OWL_ACOUSTIC_ISO_2D: h->eng.reset(make_ac2d_engine(*desc)); break;
            case OWL_ACOUSTIC_ISO_3D: h->eng.reset(make_ac3d_engine(*desc)); break;
            case OWL_ELASTIC_VHTIORT_2D: h->eng.reset(make_el2d_engine(*desc)); break;
            case OWL_ELASTIC_VHTIORT_3D: h->eng.reset(make_el3d_engine(*desc)); break;
            default: throw OwlError(OWL_ERR_UNSUPPORTED, "medium not built");
        }
        *out = h.release();
    });
}

int owl_ssg_set_model(owl_ssg* h, int nparam, const float* const* fields) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        h->eng->set_model(nparam, fields);
    });
}

int owl_ssg_forward(owl_ssg* h, int nshots, const owl_shot* shots, const owl_run_opts* opts, float* seis,
                    int mem_kind, owl_run_info* info) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(nshots >= 0 && (nshots == 0 || shots), OWL_ERR_INVALID, "bad shots");
        OWL_CHECK(seis || nshots == 0, OWL_ERR_INVALID, "null seismogram buffer");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        owl_run_info tmp{};
        h->eng->forward(nshots, shots, opts_or_default(opts), seis, mem_kind, info ? *info : tmp);
    });
}

int owl_ssg_gradient(owl_ssg* h, int nshots, const owl_shot* shots, const float* data, int adj_kind,
                     const owl_run_opts* opts, double* misfit, float* grad, float* seis_out, int mem_kind,
                     owl_run_info* info) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(nshots >= 0 && (nshots == 0 || shots), OWL_ERR_INVALID, "bad shots");
        OWL_CHECK(data || nshots == 0, OWL_ERR_INVALID, "null data buffer");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        owl_run_info tmp{};
        h->eng->gradient(nshots, shots, data, adj_kind, opts_or_default(opts), misfit, grad, seis_out, mem_kind,
                         info ? *info : tmp);
    });
}

int owl_ssg_source_gradient(owl_ssg* h, int nshots, const owl_shot* shots, const float* adj, const owl_run_opts* opts,
                            float* stf_grad, int mem_kind, owl_run_info* info) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(nshots >= 0 && (nshots == 0 || shots) && adj && stf_grad, OWL_ERR_INVALID, "bad arguments");
        owl_run_info tmp{};
        h->eng->source_gradient(nshots, shots, adj, opts_or_default(opts), stf_grad, mem_kind, info ? *info : tmp);
    });
}

int owl_ssg_misfit(owl_ssg* h, int nshots, const owl_shot* shots, const float* obs, const owl_run_opts* opts,
                   double* misfit, double* trace_misfit, float* seis_out, int mem_kind, owl_run_info* info) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(nshots >= 0 && (nshots == 0 || shots), OWL_ERR_INVALID, "bad shots");
        OWL_CHECK(obs || nshots == 0, OWL_ERR_INVALID, "null data buffer");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        owl_run_info tmp{};
        h->eng->misfit(nshots, shots, obs, opts_or_default(opts), misfit, trace_misfit, seis_out, mem_kind,
                       info ? *info : tmp);
    });
}

int owl_ssg_gradient_misfit(owl_ssg* h, int nshots, const owl_shot* shots, const float* obs,
                            const owl_misfit_opts* mopts, const owl_run_opts* opts, double* misfit, float* grad,
                            float* seis_out, int mem_kind, owl_run_info* info) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(mopts, OWL_ERR_INVALID, "null misfit options");
        OWL_CHECK(nshots >= 0 && (nshots == 0 || shots), OWL_ERR_INVALID, "bad shots");
        OWL_CHECK(obs || nshots == 0, OWL_ERR_INVALID, "null data buffer");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        OWL_CHECK(mopts->misfit >= OWL_MISFIT_WAVEFORM && mopts->misfit <= OWL_MISFIT_DTW_VECTOR, OWL_ERR_INVALID,
                  "bad misfit type");
        h->eng->mopts = *mopts;
        if (h->eng->mopts.dt <= 0.f) h->eng->mopts.dt = h->eng->desc.dt;
        owl_run_info tmp{};
        h->eng->gradient(nshots, shots, obs, ADJ_MISFIT, opts_or_default(opts), misfit, grad, seis_out, mem_kind,
                         info ? *info : tmp);
    });
}

int owl_ssg_set_data_sampling(owl_ssg* h, int data_nt, float data_dt) {
    return guarded([&] {
        OWL_CHECK(h && h->eng, OWL_ERR_INVALID, "null handle");
        OWL_CHECK(data_nt <= 0 || data_dt > 0.f, OWL_ERR_INVALID, "data_dt must be positive");
        h->eng->data_nt = data_nt > 0 ? data_nt : 0;
        h->eng->data_dt = data_nt > 0 ? data_dt : 0.f;
    });
}

int owl_resample_traces(int ntr, int nin, float din, float oin, const float* in, int nout, float dout, float oout,
                        float* out, int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(ntr >= 0 && nin >= 1 && nout >= 0 && din > 0.f && dout > 0.f, OWL_ERR_INVALID,
                  "bad resampling geometry");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        if (ntr == 0 || nout == 0) return;
        OWL_CHECK(in && out, OWL_ERR_INVALID, "null trace buffer");
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        DevBuf<float> din_b, dout_b;
        const float* pi = in;
        float* po = out;
        if (mem_kind == OWL_MEM_HOST) {
            din_b.upload(in, (size_t)ntr * nin, c.s);
            dout_b.reserve((size_t)ntr * nout);
            pi = din_b.p;
            po = dout_b.p;
        }
        launch_resample_rows(pi, nin, din, oin, po, nout, dout, oout, ntr, c.s);
        if (mem_kind == OWL_MEM_HOST)
            OWL_CUDA(cudaMemcpyAsync(out, po, (size_t)ntr * nout * sizeof(float), cudaMemcpyDeviceToHost, c.s));
        OWL_CUDA(cudaStreamSynchronize(c.s));
    });
}

int owl_su_encode(int ntr, int ns, const unsigned char* header, const float* traces, unsigned char* out,
                  int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(ntr >= 0 && ns >= 1 && ns <= 32767, OWL_ERR_INVALID, "bad SU geometry (1 <= ns <= 32767)");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        if (ntr == 0) return;
        OWL_CHECK(header && traces && out, OWL_ERR_INVALID, "null buffer");
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        su_encode(header, traces, ntr, ns, out, mem_kind == OWL_MEM_DEVICE, c.s);
    });
}

int owl_su_decode(int ntr, int ns, const unsigned char* in, float* traces, int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(ntr >= 0 && ns >= 1 && ns <= 32767, OWL_ERR_INVALID, "bad SU geometry (1 <= ns <= 32767)");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        if (ntr == 0) return;
        OWL_CHECK(in && traces, OWL_ERR_INVALID, "null buffer");
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        su_decode(in, ntr, ns, traces, mem_kind == OWL_MEM_DEVICE, c.s);
    });
}

int owl_search_direction(int method, long long n, int nm, const float* const* models, const float* const* grads,
                         const float* prev_srch, float* srch, int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(method >= OWL_SEARCH_SD && method <= OWL_SEARCH_LBFGS, OWL_ERR_INVALID, "bad search method");
        OWL_CHECK(n >= 0 && nm >= 1 && models && grads && srch, OWL_ERR_INVALID, "bad search-direction arguments");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        for (int i = 0; i < nm; ++i) OWL_CHECK(grads[i] && (models[i] || method != OWL_SEARCH_LBFGS),
                                                 OWL_ERR_INVALID, "null model / gradient");
        if (n == 0) return;
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        std::vector<const float*> x(nm), g(nm);
        const float* ps = prev_srch;
        float* out = srch;
        std::vector<std::unique_ptr<DevBuf<float>>> keep;
        auto dev = [&](const float* h) -> const float* {
            if (!h || mem_kind == OWL_MEM_DEVICE) return h;
            keep.emplace_back(new DevBuf<float>());
            keep.back()->upload(h, (size_t)n, c.s);
            return keep.back()->p;
        };
        for (int i = 0; i < nm; ++i) {
            x[i] = dev(models[i]);
            g[i] = dev(grads[i]);
        }
        ps = dev(prev_srch);
        DevBuf<float> dsrch;
        if (mem_kind == OWL_MEM_HOST) {
            dsrch.reserve((size_t)n);
            out = dsrch.p;
        }
        search_direction(method, n, nm, x.data(), g.data(), ps, out, c.s);
        if (mem_kind == OWL_MEM_HOST)
            OWL_CUDA(cudaMemcpyAsync(srch, out, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, c.s));
        OWL_CUDA(cudaStreamSynchronize(c.s));
    });
}

int owl_grad_process(int op, int n1, int n2, int n3, const float* param, const float* mask, float* field,
                     int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(op >= OWL_GRAD_SMOOTH && op <= OWL_GRAD_MEDIAN, OWL_ERR_INVALID, "bad gradient processing op");
        OWL_CHECK(n1 >= 1 && n2 >= 1 && n3 >= 1 && field, OWL_ERR_INVALID, "bad field");
        OWL_CHECK(param || op == OWL_GRAD_MASK || op == OWL_GRAD_MAX_BALANCE, OWL_ERR_INVALID, "null param");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        const size_t n = (size_t)n1 * n2 * n3;
        DevBuf<float> df, dm;
        float* f = field;
        const float* m = mask;
        if (mem_kind == OWL_MEM_HOST) {
            df.upload(field, n, c.s);
            f = df.p;
            if (mask) {
                dm.upload(mask, n, c.s);
                m = dm.p;
            }
        }
        grad_process(op, n1, n2, n3, param, m, f, c.s);
        if (mem_kind == OWL_MEM_HOST) OWL_CUDA(cudaMemcpyAsync(field, f, n * sizeof(float), cudaMemcpyDeviceToHost, c.s));
        OWL_CUDA(cudaStreamSynchronize(c.s));
    });
}

// owl_adjoint_source and owl_dtw_time_shifts: host or device traces in, the
// requested outputs back in the same memory kind
static int adjoint_source_impl(const owl_misfit_opts* mopts, int ngather, const int* gather_ptr, int nt,
                               const float* syn, const float* obs, const float* weight, float* adj,
                               double* trace_misfit, double* gather_misfit, float* tau, int mem_kind) {
    return guarded([&] {
        check_device();
        OWL_CHECK(mopts, OWL_ERR_INVALID, "null misfit options");
        OWL_CHECK(ngather >= 0 && (ngather == 0 || gather_ptr) && nt >= 1, OWL_ERR_INVALID, "bad trace layout");
        OWL_CHECK(mem_kind == OWL_MEM_HOST || mem_kind == OWL_MEM_DEVICE, OWL_ERR_INVALID, "bad mem_kind");
        const int ntr = ngather ? gather_ptr[ngather] : 0;
        OWL_CHECK(ntr >= 0 && (ntr == 0 || (syn && obs)), OWL_ERR_INVALID, "null trace buffer");
        struct Ctx {
            cudaStream_t s = nullptr;
            ~Ctx() {
                if (s) cudaStreamDestroy(s);
            }
        } c;
        OWL_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        AdjointSource as;
        const size_t n = (size_t)ntr * nt;
        DevBuf<float> dsyn, dobs, dadj, dw, dtau;
        DevBuf<double> dtm, dgm;
        DevBuf<unsigned char> dlive;
        const bool dev = mem_kind == OWL_MEM_DEVICE;
        const float* ps = syn;
        const float* po = obs;
        float* pa = adj;
        double* ptm = trace_misfit;
        double* pgm = gather_misfit;
        float* ptau = tau;
        if (!dev && ntr) {
            dsyn.upload(syn, n, c.s);
            dobs.upload(obs, n, c.s);
            ps = dsyn.p;
            po = dobs.p;
            if (adj) { dadj.reserve(n); pa = dadj.p; }
            if (trace_misfit) { dtm.reserve(ntr); ptm = dtm.p; }
            if (tau) { dtau.reserve(n); ptau = dtau.p; }
        }
        if (!dev && gather_misfit && ngather) { dgm.reserve(ngather); pgm = dgm.p; }
        const unsigned char* wl = nullptr;
        if (weight && ntr) {
            const float* pw = weight;
            if (!dev) { dw.upload(weight, ntr, c.s); pw = dw.p; }
            dlive.reserve(ntr);
            launch_nonzero(pw, ntr, dlive.p, c.s);
            wl = dlive.p;
        }
        as.run(*mopts, ngather, gather_ptr, nt, ps, po, wl, pa, ptm, pgm, c.s, ptau);
        if (!dev) {
            if (adj && ntr) OWL_CUDA(cudaMemcpyAsync(adj, pa, n * sizeof(float), cudaMemcpyDeviceToHost, c.s));
            if (tau && ntr) OWL_CUDA(cudaMemcpyAsync(tau, ptau, n * sizeof(float), cudaMemcpyDeviceToHost, c.s));
            if (trace_misfit && ntr)
                OWL_CUDA(cudaMemcpyAsync(trace_misfit, ptm, ntr * sizeof(double), cudaMemcpyDeviceToHost, c.s));
            if (gather_misfit && ngather)
                OWL_CUDA(cudaMemcpyAsync(gather_misfit, pgm, ngather * sizeof(double), cudaMemcpyDeviceToHost, c.s));
        }
        OWL_CUDA(cudaStreamSynchronize(c.s));
    });
}

int owl_adjoint_source(const owl_misfit_opts* mopts, int ngather, const int* gather_ptr, int nt, const float* syn,
                       const float* obs, const float* weight, float* adj, double* trace_misfit,
                       double* gather_misfit, int mem_kind) {
    return adjoint_source_impl(mopts, ngather, gather_ptr, nt, syn, obs, weight, adj, trace_misfit, gather_misfit,
                               nullptr, mem_kind);
}

int owl_dtw_time_shifts(const owl_misfit_opts* mopts, int ngather, const int* gather_ptr, int nt, const float* syn,
                        const float* obs, const float* weight, float* tau, int mem_kind) {
    if (!mopts || (mopts->misfit != OWL_MISFIT_DTW && mopts->misfit != OWL_MISFIT_DTW_VECTOR) || !tau)
        return guarded([&] { OWL_CHECK(false, OWL_ERR_INVALID, "owl_dtw_time_shifts needs the DTW misfit and a tau buffer"); });
    return adjoint_source_impl(mopts, ngather, gather_ptr, nt, syn, obs, weight, nullptr, nullptr, nullptr, tau,
                               mem_kind);
}

int owl_ssg_kernel_time(owl_ssg* h, int kernel_id, int nlaunch, double* avg_ms, double* alg_bytes) {
    return guarded([&] {
        OWL_CHECK(h && h->eng && avg_ms && alg_bytes && nlaunch > 0, OWL_ERR_INVALID, "bad arguments");
        h->eng->kernel_time(kernel_id, nlaunch, avg_ms, alg_bytes);
    });
}

int owl_ssg_mpml_ratios(const owl_ssg* h, float* faces) {
    return guarded([&] {
        OWL_CHECK(h && h->eng && faces, OWL_ERR_INVALID, "bad arguments");
        const std::vector<float>* f = h->eng->mpml_faces();
        OWL_CHECK(f && h->eng->model_set, OWL_ERR_INVALID, "M-PML ratios exist for an elastic 3D handle after set_model");
        std::copy(f->begin(), f->end(), faces);
    });
}

void owl_ssg_destroy(owl_ssg* h) {
    if (!h) return;
    try {
        if (h->eng) cudaStreamSynchronize(h->eng->stream);
    } catch (...) {
    }
    delete h;
}

float owl_ssg_dt_stable(const owl_ssg* h) { return (h && h->eng) ? h->eng->dt_stable_ : 0.f; }

}  // extern "C"
