// ssg_base.cu -- medium-independent host engine and point / checkpoint kernels.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <map>

#include "ssg_base.cuh"

namespace owl {

// ------------------------------ point operators ----------------------------
// Grid (shots, NB). Forward: add_source(t) by the CTAs of row 0 (sources in
// order, taps of one source in parallel, as the reference's loops), then the
// receivers of step t+1 (each trace a sequential sum over its taps) spread over
// the NB CTAs of the shot. With NB > 1 injection and sampling are two launches
// (the sampling must see every injected tap). The last CTA to finish advances
// the device step counter, so one captured graph serves every segment.
__global__ void k_point_fwd(PointDev a, int mode) {
    pdl_prologue();
    const int s = blockIdx.x;
    const int cur = *a.d_step;
    const int t = cur + 1;
    if ((mode & PT_INJECT) && blockIdx.y == 0) {
        for (int it = a.inj_shot_ptr[s]; it < a.inj_shot_ptr[s + 1]; ++it) {
            const float A = a.amp[(size_t)it * a.nt + (t - 1)];
            if (A != 0.f) {
                for (int j = a.inj.ptr[it] + threadIdx.x; j < a.inj.ptr[it + 1]; j += blockDim.x) {
                    float* f = a.fld[a.inj.field[j]] + s * a.sstride + a.inj.off[j];
                    *f = *f + A * a.inj.w[j];
                }
            }
            __syncthreads();
        }
    }
    if (mode & PT_SAMPLE) {
        const int tr = (mode & PT_NEXT) ? t + 1 : t;
        if (tr <= a.nt) {
            const int step = gridDim.y * blockDim.x;
            for (int r = a.rec_shot_ptr[s] + blockIdx.y * blockDim.x + threadIdx.x; r < a.rec_shot_ptr[s + 1]; r += step) {
                float acc = 0.f;
                for (int j = a.smp.ptr[r]; j < a.smp.ptr[r + 1]; ++j)
                    acc = acc + a.fld[a.smp.field[j]][s * a.sstride + a.smp.off[j]] * a.smp.w[j];
                a.rec[(size_t)(tr - 1) * a.rtot + r] = acc;
            }
        }
    }
    if (mode & PT_TICK) tick_last_block(a.d_step, a.d_done, 1);
}

// Adjoint of the sampling of step t (residual into the adjoint fields, one
// thread per distinct target node, contributions summed in a fixed order),
// then the source-side adjoint taps . lambda_{t-1}; the last CTA steps back.
// Same split as the forward when a shot has many target nodes.
__global__ void k_point_adj(PointDev a, int mode) {
    pdl_prologue();
    const int s = blockIdx.x;
    const int t = *a.d_step;
    if (mode & PA_SCATTER) {
        const int step = gridDim.y * blockDim.x;
        for (int it = a.sct_shot_ptr[s] + blockIdx.y * blockDim.x + threadIdx.x; it < a.sct_shot_ptr[s + 1]; it += step) {
            float acc = 0.f;
            const int j0 = a.sct.ptr[it], j1 = a.sct.ptr[it + 1];
            for (int j = j0; j < j1; ++j) acc = acc + a.res[(size_t)(t - 1) * a.rtot + a.sct.item[j]] * a.sct.w[j];
            float* f = a.fld[a.sct.field[j0]] + s * a.sstride + a.sct.off[j0];
            *f = *f + acc;
        }
    }
    if ((mode & PA_SRC) && blockIdx.y == 0) {
        __syncthreads();
        if (a.src_adj && t - 1 >= 1) {
            for (int it = a.inj_shot_ptr[s] + threadIdx.x; it < a.inj_shot_ptr[s + 1]; it += blockDim.x) {
                float acc = 0.f;
                for (int j = a.inj.ptr[it]; j < a.inj.ptr[it + 1]; ++j)
                    acc = acc + a.fld[a.inj.field[j]][s * a.sstride + a.inj.off[j]] * a.inj.w[j];
                a.src_adj[(size_t)it * a.nt + (t - 2)] = acc;
            }
        }
    }
    if ((mode & PA_SRC_NOW) && blockIdx.y == 0 && a.src_adj && t >= 1) {
        for (int it = a.inj_shot_ptr[s] + threadIdx.x; it < a.inj_shot_ptr[s + 1]; it += blockDim.x) {
            float acc = 0.f;
            for (int j = a.inj.ptr[it]; j < a.inj.ptr[it + 1]; ++j)
                acc = acc + a.fld[a.inj.field[j]][s * a.sstride + a.inj.off[j]] * a.inj.w[j];
            a.src_adj[(size_t)it * a.nt + (t - 1)] = acc;
        }
    }
    if (mode & PA_TICK) tick_last_block(a.d_step, a.d_done, -1);
}

void launch_point_fwd(const PointDev& q, int S, int nb, int mode, cudaStream_t s) {
    launch_pdl(k_point_fwd, dim3(S, nb), dim3(256), 0, s, q, mode);
}
void launch_point_adj(const PointDev& q, int S, int nb, int mode, cudaStream_t s) {
    launch_pdl(k_point_adj, dim3(S, nb), dim3(256), 0, s, q, mode);
}

// ------------------------- compressed checkpoints ---------------------------
// Per (shot, state field) scale = max |x|; values stored as x / scale in FP16 or
// BF16. Blocks: (segment, shot); each block loops over its segment.
struct SegDev {
    const long long* off;
    const long long* len;
    int nseg;
};

__global__ void k_absmax(const float* __restrict__ st, long long sstride, SegDev sg, float* __restrict__ scale) {
    const int g = blockIdx.x, s = blockIdx.y;
    const float* p = st + s * sstride + sg.off[g];
    const long long n = sg.len[g];
    float m = 0.f;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fabsf(p[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmaxf(r, red[w]);
        scale[s * sg.nseg + g] = r;
    }
}

template <bool BF16>
__global__ void k_pack(const float* __restrict__ st, long long sstride, SegDev sg, const float* __restrict__ scale,
                       unsigned short* __restrict__ out) {
    const int g = blockIdx.x, s = blockIdx.y;
    const float* p = st + s * sstride + sg.off[g];
    unsigned short* q = out + s * sstride + sg.off[g];
    const long long n = sg.len[g];
    const float sc = scale[s * sg.nseg + g];
    // a field whose largest value is below the smallest normal float is stored as
    // zero: 1 / sc would overflow and turn its zeros into NaN
    const float inv = sc >= FLT_MIN ? 1.0f / sc : 0.f;
    for (long long i = blockIdx.z * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.z * blockDim.x) {
        float v = p[i] * inv;
        if (BF16) {
            __nv_bfloat16 h = __float2bfloat16_rn(v);
            q[i] = *reinterpret_cast<unsigned short*>(&h);
        } else {
            __half h = __float2half_rn(v);
            q[i] = *reinterpret_cast<unsigned short*>(&h);
        }
    }
}

template <bool BF16>
__global__ void k_unpack(const unsigned short* __restrict__ in, long long sstride, SegDev sg,
                         const float* __restrict__ scale, float* __restrict__ st) {
    const int g = blockIdx.x, s = blockIdx.y;
    float* p = st + s * sstride + sg.off[g];
    const unsigned short* q = in + s * sstride + sg.off[g];
    const long long n = sg.len[g];
    const float sc = scale[s * sg.nseg + g];
    for (long long i = blockIdx.z * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.z * blockDim.x) {
        unsigned short u = q[i];
        float v;
        if (BF16) v = __bfloat162float(*reinterpret_cast<__nv_bfloat16*>(&u));
        else v = __half2float(*reinterpret_cast<__half*>(&u));
        p[i] = sc >= FLT_MIN ? v * sc : 0.f;
    }
}

// ------------------------------ fold ----------------------------------------
// Padded-grid FP64 gradient -> model cells (adjoint of pad_array's edge
// replication), output (nz[,ny],nx) with z fastest.
__global__ void k_fold(const double* __restrict__ gp, int nxq, int nyq, int P, int nx, int ny, int nz, int dim,
                       float* __restrict__ out) {
    const long long n = (long long)nx * ny * nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int iz = (int)(q % nz) + 1;
        const long long r = q / nz;
        const int iy = (int)(r % ny) + 1, ix = (int)(r / ny) + 1;
        const int xa = ix == 1 ? -P : ix, xb = ix == nx ? nx + P + 1 : ix;
        const int za = iz == 1 ? -P : iz, zb = iz == nz ? nz + P + 1 : iz;
        int ya = 0, yb = 0;
        if (dim == 3) { ya = iy == 1 ? -P : iy; yb = iy == ny ? ny + P + 1 : iy; }
        double acc = 0;
        for (int k = za; k <= zb; ++k)
            for (int j = ya; j <= yb; ++j)
                for (int i = xa; i <= xb; ++i)
                    acc += gp[((long long)(k + P) * nyq + (dim == 3 ? j + P : 0)) * nxq + (i + P)];
        out[q] = (float)acc;
    }
}

void launch_fold(const double* gp, int nxq, int nyq, int P, int nx, int ny, int nz, int dim, float* out,
                 cudaStream_t s) {
    k_fold<<<148 * 4, 256, 0, s>>>(gp, nxq, nyq, P, nx, ny, nz, dim, out);
    OWL_LAUNCH_CHECK();
}

__global__ void k_add_points_f64(double* g, const long long* idx, const double* val, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[idx[i]] += val[i];
}

// ============================================================================
// host side
// ============================================================================
SsgBase::SsgBase(const owl_ssg_desc& d, int dim_) {
    desc = d;
    dim = dim_;
    OWL_CHECK(d.nx >= 8 && d.nz >= 8 && (dim == 2 || d.ny >= 8), OWL_ERR_INVALID, "grid dimensions must be >= 8");
    OWL_CHECK(d.fdhalf == 4 || d.fdhalf == 8, OWL_ERR_INVALID, "fdhalf must be 4 or 8");
    OWL_CHECK(d.pml >= 1, OWL_ERR_INVALID, "pml must be >= 1");
    OWL_CHECK(d.dx > 0 && d.dz > 0 && (dim == 2 || d.dy > 0) && d.dt > 0 && d.nt >= 1, OWL_ERR_INVALID,
              "dx, dy, dz, dt, nt must be positive");
    nx = d.nx; ny = dim == 3 ? d.ny : 1; nz = d.nz;
    P = d.pml; R = d.fdhalf; pr = P + R;
    NXp = nx + 2 * P; NYp = dim == 3 ? ny + 2 * P : 1; NZp = nz + 2 * P;
    NXs = NXp + 2 * R; NYs = dim == 3 ? NYp + 2 * R : 1; NZs = NZp + 2 * R;
    // rows of 128-byte multiples; in 2D at least four floats past the last
    // column, so that the four-cell kernels' float4 windows stay in their row
    pitch = (NXs + (dim == 2 ? 4 : 0) + 31) / 32 * 32;
    plane = (long long)pitch * NYs;
    fs = plane * NZs;
    dt = d.dt;
    OWL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    // step counter, CTA count of the last-block tick, non-finite flag, timeout flag
    ctr.reserve(4);
    OWL_CUDA(cudaMemsetAsync(ctr.p, 0, 4 * sizeof(int), stream));
}

void SsgBase::check_timeout() {
    int flag = 0;
    OWL_CUDA(cudaMemcpyAsync(&flag, ctr.p + 3, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OWL_CUDA(cudaStreamSynchronize(stream));
    if (flag) {
        OWL_CUDA(cudaMemsetAsync(ctr.p + 3, 0, sizeof(int), stream));
        throw OwlError(OWL_ERR_TIMEOUT, "a bounded wait (TMA copies or a grid barrier) gave up; the results are invalid");
    }
}

SsgBase::~SsgBase() {
    invalidate_graphs();
    if (stream) cudaStreamDestroy(stream);
}

void SsgBase::invalidate_graphs() {
    g_fwd.reset();
    g_rec.reset();
    g_adj.reset();
    g_fst.reset();
}

DevBuf<long long>& SsgBase::seg_off() {
    const size_t n = st_segments.size();
    if (segbuf.n < 2 * n || !segbuf.p) {
        std::vector<long long> h(2 * n);
        for (size_t i = 0; i < n; ++i) { h[i] = st_segments[i].first; h[n + i] = st_segments[i].second; }
        segbuf.upload(h.data(), h.size(), stream);
    }
    return segbuf;
}

void SsgBase::set_step(int v) {
    int h[2] = {v, 0};
    OWL_CUDA(cudaMemcpyAsync(ctr.p, h, 2 * sizeof(int), cudaMemcpyHostToDevice, stream));
}

void SsgBase::build_tables(int S, const owl_shot* shots, bool need_sct) {
    HostCSR hinj, hsmp, hsct;
    std::vector<int> hinj_ptr(1, 0), hrec_ptr(1, 0), hsct_ptr(1, 0);
    h_gather_ptr.assign(1, 0);
    std::vector<float> hamp;
    std::vector<unsigned char> hlive;
    std::vector<int4> hbox;
    std::vector<float> hbw;
    const size_t boxn = dim == 3 ? (size_t)BOX_W * BOX_W * BOX_W : (size_t)BOX_W * BOX_W;
    bool fuse = fuse_supported();
    item_src.clear(); item_comp.clear(); item_shot.clear(); item_rho_cell.clear(); item_rho.clear();
    const int nt = desc.nt;
    std::vector<TapPt> taps, mapped;
    rtot = 0;
    for (int s = 0; s < S; ++s) {
        const owl_shot& sh = shots[s];
        OWL_CHECK(sh.nsrc >= 0 && sh.nrec >= 0 && (sh.nsrc == 0 || sh.src) && (sh.nrec == 0 || sh.rec),
                  OWL_ERR_INVALID, "bad shot arrays");
        for (int kk = 0; kk < sh.nsrc; ++kk) {
            const owl_source& q = sh.src[kk];
            OWL_CHECK(q.nt_stf >= 0 && (q.nt_stf == 0 || q.stf), OWL_ERR_INVALID, "bad source STF");
            const int nc = src_ncomp(q);
            for (int comp = 0; comp < nc; ++comp) {
                taps.clear();
                long long rc = -1;
                float rv = 0.f;
                src_taps(q, comp, taps, rc, rv);
                int bi = 1 << 30, bj = 1 << 30, bk = 1 << 30, bf = -1;
                for (const TapPt& t : taps) {
                    if (t.w == 0.f) continue;
                    OWL_CHECK(in_wavefield(t.i, t.j, t.k), OWL_ERR_INVALID, "source tap outside the padded grid");
                    hinj.push(Tap{t.field, s, soff(t.i, t.j, t.k), t.w, 0});
                    bi = std::min(bi, t.i); bj = std::min(bj, t.j); bk = std::min(bk, t.k);
                    if (bf < 0) bf = t.field;
                    if (bf != t.field) fuse = false;
                }
                hinj.close_item();
                {
                    const size_t base = hbw.size();
                    hbw.resize(base + boxn, 0.f);
                    if (bf < 0) { bi = bj = bk = -(1 << 20); bf = 0; }
                    hbox.push_back(int4{bf, bi + pr - 1, dim == 3 ? bj + pr - 1 : 0, bk + pr - 1});
                    for (const TapPt& t : taps) {
                        if (t.w == 0.f) continue;
                        const int dx = t.i - bi, dy = dim == 3 ? t.j - bj : 0, dz = t.k - bk;
                        if (dx >= BOX_W || dy >= BOX_W || dz >= BOX_W) { fuse = false; continue; }
                        hbw[base + ((size_t)dz * (dim == 3 ? BOX_W : 1) + dy) * BOX_W + dx] = t.w;
                        fuse &= fuse_tap_ok(t.field, t.i + pr - 1, dim == 3 ? t.j + pr - 1 : 0, t.k + pr - 1, false);
                    }
                }
                item_src.push_back(kk); item_comp.push_back(comp); item_shot.push_back(s);
                item_rho_cell.push_back(rc); item_rho.push_back(rv);
                size_t base = hamp.size();
                hamp.resize(base + nt, 0.f);
                for (int t = std::max(1, q.nbeg); t <= q.nbeg + q.nt_stf - 1 && t <= nt; ++t)
                    hamp[base + t - 1] = q.stf[t - q.nbeg] * q.amp * dt;
            }
        }
        hinj_ptr.push_back(hinj.nitems());
        std::map<std::pair<int, long long>, std::vector<std::pair<int, float>>> cells;
        for (int comp = 0; comp < ncomp; ++comp) {
            for (int r = 0; r < sh.nrec; ++r) {
                const owl_receiver& q = sh.rec[r];
                const int rg = rtot + comp * sh.nrec + r;
                hlive.push_back(q.weight != 0.f);
                if (q.weight != 0.f) {
                    taps.clear();
                    rec_taps(q, comp, taps);
                    for (const TapPt& t : taps) {
                        if (t.w == 0.f) continue;
                        OWL_CHECK(in_wavefield(t.i, t.j, t.k), OWL_ERR_INVALID, "receiver tap outside the padded grid");
                        hsmp.push(Tap{t.field, s, soff(t.i, t.j, t.k), t.w, rg});
                        fuse &= fuse_tap_ok(t.field, t.i + pr - 1, dim == 3 ? t.j + pr - 1 : 0, t.k + pr - 1, true);
                        if (need_sct) {
                            mapped.clear();
                            scatter_map(t, mapped);
                            for (const TapPt& m : mapped) {
                                cells[{m.field, soff(m.i, m.j, m.k)}].push_back({rg, m.w});
                                fuse &= fuse_tap_ok(m.field, m.i + pr - 1, dim == 3 ? m.j + pr - 1 : 0, m.k + pr - 1,
                                                    true);
                            }
                        }
                    }
                }
                hsmp.close_item();
            }
        }
        for (auto& kv : cells) {
            for (auto& e : kv.second) hsct.push(Tap{kv.first.first, s, kv.first.second, e.second, e.first});
            hsct.close_item();
        }
        for (int comp = 0; comp < ncomp; ++comp) h_gather_ptr.push_back(rtot + (comp + 1) * sh.nrec);
        rtot += ncomp * sh.nrec;
        hrec_ptr.push_back(rtot);
        hsct_ptr.push_back(hsct.nitems());
    }
    int mr = 0, ms = 0;
    for (size_t i = 0; i + 1 < hrec_ptr.size(); ++i) mr = std::max(mr, hrec_ptr[i + 1] - hrec_ptr[i]);
    for (size_t i = 0; i + 1 < hsct_ptr.size(); ++i) ms = std::max(ms, hsct_ptr[i + 1] - hsct_ptr[i]);
    nb_rec = std::max(1, std::min(1024, (mr + 255) / 256));
    nb_sct = std::max(1, std::min(1024, (ms + 255) / 256));
    inj.upload(hinj, stream);
    smp.upload(hsmp, stream);
    sct.upload(hsct, stream);
    inj_shot_ptr.upload(hinj_ptr.data(), hinj_ptr.size(), stream);
    rec_shot_ptr.upload(hrec_ptr.data(), hrec_ptr.size(), stream);
    sct_shot_ptr.upload(hsct_ptr.data(), hsct_ptr.size(), stream);
    amp.upload(hamp.data(), hamp.size(), stream);
    live.upload(hlive.data(), hlive.size(), stream);
    inj_fmask = 0;
    for (const int4& b : hbox)
        if (b.x >= 0 && b.x < 30) inj_fmask |= 1 << b.x;
    {
        std::vector<int4> bb(2 * (size_t)std::max(S, 1), int4{0, 0, 0, 0});
        for (int s = 0; s < S; ++s)
            for (int it = hinj_ptr[s]; it < hinj_ptr[s + 1]; ++it) {
                const int4 b = hbox[it];
                if (b.x < 0 || b.y < -(1 << 19)) continue;  // no taps
                int4& u = bb[2 * s + (b.x == 0 ? 0 : 1)];
                const int4 nb{b.y, b.y + BOX_W, b.w, b.w + BOX_W};
                if (u.x == u.y) u = nb;
                else u = int4{std::min(u.x, nb.x), std::max(u.y, nb.y), std::min(u.z, nb.z), std::max(u.w, nb.w)};
            }
        inj_bbox.upload(bb.data(), bb.size(), stream);
    }
    if (hbox.empty()) { hbox.push_back(int4{-1, 0, 0, 0}); hbw.resize(boxn, 0.f); }
    inj_box.upload(hbox.data(), hbox.size(), stream);
    inj_bw.upload(hbw.data(), hbw.size(), stream);
    // the point work inside the stencil kernels where the medium supports it:
    // the adjoint's residual scatter by default; OWL_FUSE=1 also the forward's
    // injection and sampling (measured 3 % slower on the 32-shot gradient than
    // the separate point kernel, whose one small launch per step costs less
    // than the extra work of the stencil CTAs), OWL_FUSE=0 neither
    const char* fz = std::getenv("OWL_FUSE");
    fuse_on = fuse && !(fz && fz[0] == '0' && fz[1] == 0);
    fuse_fwd = fuse_on && fz && fz[0] == '1' && fz[1] == 0;
}

void SsgBase::ensure_state(int S, int k, bool grad) {
    st.reserve((size_t)sst * S);
    if (grad) {
        ad.reserve((size_t)sad * S);
        G.reserve((size_t)2 * ngrad * S * fs);
        Sbuf.reserve((size_t)nS * k * S * fs);
    }
}

PointDev SsgBase::pdev(int S, bool adjoint, bool want_src_adj) {
    PointDev q{};
    for (int f = 0; f < MAX_PT_FIELDS; ++f) q.fld[f] = nullptr;
    for (int f = 0; f < MAX_PT_FIELDS; ++f) {
        float* p = adjoint ? ad_field(f) : st_field(f);
        if (!p) break;
        q.fld[f] = p;
    }
    q.sstride = adjoint ? sad : sst;
    q.nt = desc.nt;
    q.rtot = rtot;
    q.inj = view(inj); q.inj_shot_ptr = inj_shot_ptr.p; q.amp = amp.p;
    q.smp = view(smp); q.rec_shot_ptr = rec_shot_ptr.p; q.rec = rec.p;
    q.sct = view(sct); q.sct_shot_ptr = sct_shot_ptr.p; q.res = res.p;
    q.src_adj = want_src_adj ? src_adj.p : nullptr;
    q.d_step = ctr.p; q.d_done = ctr.p + 1;
    return q;
}

// kind 0: forward step; 1: recomputed step storing the stencil terms; 2:
// adjoint step; 3: forward step storing the stencil terms (the last segment of
// a gradient's forward, whose recompute it replaces)
int SsgBase::step_launches(int kind) const {
    if (kind == 2 && fuse_on) return want_src_now ? 3 : 2;
    if (kind != 2 && fuse_fwd) return 2;
    if (kind == 1) return 3;
    if (kind != 2) return nb_rec <= 4 ? 3 : 4;
    return nb_sct <= 4 ? 3 : 4;
}

void SsgBase::launch_step(int kind, int S, const PointDev& q) {
    if ((kind == 2 && fuse_on) || (kind != 2 && fuse_fwd)) {
        // the stencil kernels inject, sample / scatter and advance the step counter
        if (kind != 2) {
            fz_mode = FZ_INJ | FZ_TICK | (kind == 1 ? 0 : FZ_SMP);
            launch_kernel(OWL_K_FWD_P, S, kind == 1 || kind == 3);
            launch_kernel(OWL_K_FWD_V, S, kind == 1 || kind == 3);
        } else {
            fz_mode = FZ_SCT | (want_src_now ? 0 : FZ_TICK);
            launch_kernel(OWL_K_ADJ_P, S, false);
            launch_kernel(OWL_K_ADJ_V, S, false);
            if (want_src_now) launch_point_adj(q, S, 1, PA_SRC | PA_TICK, stream);
        }
        fz_mode = 0;
        launches += step_launches(kind);
        return;
    }
    // point operators of shots with more than 1024 traces / target nodes use
    // NB CTAs per shot and a separate launch for the dependent phase
    if (kind != 2) {
        launch_kernel(OWL_K_FWD_P, S, kind == 1 || kind == 3);
        launch_kernel(OWL_K_FWD_V, S, kind == 1 || kind == 3);
        if (kind == 1) {
            launch_point_fwd(q, S, 1, PT_INJECT | PT_TICK, stream);
            launches += 3;
        } else if (nb_rec <= 4) {
            launch_point_fwd(q, S, 1, PT_INJECT | PT_SAMPLE | PT_NEXT | PT_TICK, stream);
            launches += 3;
        } else {
            launch_point_fwd(q, S, 1, PT_INJECT, stream);
            launch_point_fwd(q, S, nb_rec, PT_SAMPLE | PT_NEXT | PT_TICK, stream);
            launches += 4;
        }
    } else {
        launch_kernel(OWL_K_ADJ_P, S, false);
        launch_kernel(OWL_K_ADJ_V, S, false);
        if (nb_sct <= 4) {
            launch_point_adj(q, S, 1, PA_SCATTER | PA_SRC | PA_TICK, stream);
            launches += 3;
        } else {
            launch_point_adj(q, S, nb_sct, PA_SCATTER, stream);
            launch_point_adj(q, S, 1, PA_SRC | PA_TICK, stream);
            launches += 4;
        }
    }
}

void SsgBase::run_steps(int kind, int n, int S, const PointDev& q, bool graph) {
    if (n <= 0) return;
    if (run_steps_persistent(kind, n, S)) return;
    if (!graph) {
        for (int i = 0; i < n; ++i) launch_step(kind, S, q);
        OWL_LAUNCH_CHECK();
        return;
    }
    GraphCache& gc = kind == 0 ? g_fwd : kind == 1 ? g_rec : kind == 3 ? g_fst : g_adj;
    std::vector<uintptr_t> sig = {(uintptr_t)n, (uintptr_t)S, (uintptr_t)spt_f, (uintptr_t)spt_a, (uintptr_t)tz_f,
                                  (uintptr_t)tz_a, (uintptr_t)cur_k, (uintptr_t)tile_x, (uintptr_t)st.p,
                                  (uintptr_t)ad.p, (uintptr_t)Sbuf.p, (uintptr_t)G.p, (uintptr_t)rec.p,
                                  (uintptr_t)res.p, (uintptr_t)q.src_adj, (uintptr_t)inj.ptr.p, (uintptr_t)inj.w.p,
                                  (uintptr_t)inj.off.p, (uintptr_t)smp.ptr.p, (uintptr_t)smp.w.p, (uintptr_t)smp.off.p,
                                  (uintptr_t)sct.ptr.p, (uintptr_t)sct.w.p, (uintptr_t)sct.off.p, (uintptr_t)amp.p,
                                  (uintptr_t)inj_shot_ptr.p, (uintptr_t)rec_shot_ptr.p, (uintptr_t)sct_shot_ptr.p,
                                  (uintptr_t)q.rtot, (uintptr_t)nb_rec, (uintptr_t)nb_sct, (uintptr_t)inj_box.p,
                                  (uintptr_t)inj_bw.p, (uintptr_t)fuse_on, (uintptr_t)fuse_fwd,
                                  (uintptr_t)want_src_now};
    if (!gc.exec || gc.sig != sig) {
        gc.reset();
        cudaGraph_t g;
        OWL_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        long long l0 = launches;
        for (int i = 0; i < n; ++i) launch_step(kind, S, q);
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        OWL_CUDA(e1);
        OWL_CUDA(e2);
        launches = l0;
        cudaError_t e3 = cudaGraphInstantiate(&gc.exec, g, 0);
        cudaGraphDestroy(g);
        OWL_CUDA(e3);
        gc.sig = sig;
    }
    OWL_CUDA(cudaGraphLaunch(gc.exec, stream));
    launches += (long long)n * step_launches(kind);
}

double SsgBase::batch_bytes(int S, int k, bool grad, int rec_per_shot) const {
    const double f4 = 4.0, nt = desc.nt;
    const double rtotS = (double)rec_per_shot * ncomp * S;
    double b = f4 * sst * S + f4 * nt * std::max(rtotS, 1.0) * (grad ? 5.0 : 2.0) + f4 * nparam * (double)nx * ny * nz;
    if (grad) {
        const int kk = std::max(1, std::min(k, desc.nt));
        const double nseg = std::ceil(nt / kk);
        const double ck = ckpt_prec == OWL_CKPT_FP32 ? 4.0 : 2.0;
        b += f4 * sad * S                          // adjoint state
             + f4 * 2.0 * ngrad * S * (double)fs   // Kahan sums, one group per shot at most
             + f4 * nS * (double)kk * S * fs       // stencil terms of a segment
             + nseg * ck * sst * S                 // checkpoints
             + 8.0 * grad_planes() * (double)npad();  // FP64 padded gradient
    }
    return b;
}

double SsgBase::held_bytes() const {
    return 4.0 * ((double)st.n + ad.n + G.n + Sbuf.n + ckpt.n + rec.n + res.n + obs_t.n + seis_tmp.n) +
           2.0 * (double)ckpt16.n + 8.0 * (double)gpad.n;
}

// Options of one call. Shots per batch: opts.shots_per_launch, else the
// largest count up to max_shots whose buffers fit the device. Checkpoint
// interval: opts.checkpoint_interval (0: 50); < 0 the whole run when the
// stored stencil terms of every step fit (nothing is recomputed), else the
// longest interval that fits. "Fit" counts every buffer of the batch (state,
// adjoint state, Kahan sums, the segment's stencil terms, checkpoints, traces)
// against 92 % of the free device memory plus what the handle already holds
// (OWL_MEM_BUDGET_MB in the environment caps that figure).
void SsgBase::resolve_opts(const owl_run_opts& o, int nshots, const owl_shot* shots, bool grad, int& B, int& k,
                           bool& graph) {
    // tile_z: 0 = autotuned; > 0 explicit tile height (3D forward: rows per
    // thread); < 0 in 3D: one thread per cell for the forward kernels
    tune = o.shots_per_cta <= 0 && o.tile_z == 0;
    OWL_CHECK(o.checkpoint_precision >= OWL_CKPT_FP32 && o.checkpoint_precision <= OWL_CKPT_BF16, OWL_ERR_INVALID,
              "bad checkpoint precision");
    ckpt_prec = o.checkpoint_precision;
    const int Bmax = std::min(o.shots_per_launch > 0 ? o.shots_per_launch : std::max(1, desc.max_shots),
                              std::max(1, nshots));
    int recs = 1;
    for (int i = 0; i < nshots && shots; ++i) recs = std::max(recs, shots[i].nrec);
    size_t fr = 0, tot = 0;
    OWL_CUDA(cudaMemGetInfo(&fr, &tot));
    double budget = 0.92 * (double)fr + held_bytes();
    if (const char* e = std::getenv("OWL_MEM_BUDGET_MB")) budget = std::min(budget, std::atof(e) * 1048576.0);
    const bool auto_k = o.checkpoint_interval < 0;
    const int k_fixed = std::min(o.checkpoint_interval > 0 ? o.checkpoint_interval : 50, desc.nt);
    // the longest interval that fits S shots, 0 if none
    auto fit_k = [&](int S) {
        if (!auto_k) return batch_bytes(S, k_fixed, grad, recs) <= budget ? k_fixed : 0;
        if (!grad) return batch_bytes(S, desc.nt, false, recs) <= budget ? desc.nt : 0;
        for (int kk = desc.nt; kk >= 1; --kk)
            if (batch_bytes(S, kk, true, recs) <= budget) return kk;
        return 0;
    };
    B = Bmax;
    k = fit_k(B);
    if (o.shots_per_launch <= 0) {
        while (k == 0 && B > 1) k = fit_k(--B);
    }
    if (k == 0) {
        // nothing fits: the interval of least memory (the allocation reports OWL_ERR_OOM)
        k = k_fixed;
        if (auto_k && grad) {
            double best = 1e300;
            for (int kk = 1; kk <= desc.nt; ++kk) {
                const double b = batch_bytes(B, kk, true, recs);
                if (b < best) { best = b; k = kk; }
            }
        }
    }
    k = std::max(1, std::min(k, desc.nt));
    plan_k = k;
    plan_B = B;
    spt_f = spt_a = std::min(o.shots_per_cta > 0 ? o.shots_per_cta : 1, B);
    graph = o.use_graph >= 0;
    launch_params(o);
}

// Times the stencil kernels of one step for each (shots per CTA, tile height)
// candidate on this batch's buffers, forward pair and adjoint pair separately,
// and keeps the fastest. Cached per (batch size, gradient). The buffers'
// contents are reset by the caller afterwards.
void SsgBase::launch_params(const owl_run_opts& o) {
    tile_x = o.tile_x > 0 ? o.tile_x : 32;
    tz_f = tz_a = o.tile_z > 0 ? o.tile_z : (dim == 3 ? 4 : 8);
    if (dim == 3 && o.tile_z < 0) tz_f = 0;
    OWL_CHECK(tile_x % 32 == 0 && tz_a >= 1 && tile_x * tz_a <= 512 && (tz_f >= 1 || dim == 3), OWL_ERR_INVALID,
              "tile_x must be a multiple of 32 and tile_x * tile_z <= 512");
}

std::vector<int> SsgBase::tune_spt(int) const { return {1, 2, 4, 8, 16, 32}; }

// 3D forward kernels take rows per thread (1, 2, 4; 0 = the per-cell kernel), 3D adjoint kernels a
// tile height (2, 4, 8; 1 = the ring kernels); 2D kernels a tile height
std::vector<int> SsgBase::tune_tz(int pass) const {
    if (dim == 3) return pass == 0 ? std::vector<int>{0, 1, 2, 4} : std::vector<int>{1, 2, 4, 8};
    return {4, 8, 16};
}

void SsgBase::autotune(int S, int k, bool grad) {
    auto key = std::make_pair(S, grad ? 1 : 0);
    auto it = tune_cache.find(key);
    if (it != tune_cache.end()) {
        spt_f = it->second[0]; tz_f = it->second[1]; spt_a = it->second[2]; tz_a = it->second[3];
        tune_extra(S, k, grad);
        return;
    }
    cur_k = k;
    set_step(k);
    // the forward pass's choice is shared by the forward-only and the gradient
    // entries of S: the forwards of a misfit and of a gradient of one handle
    // run the same kernels (their seismograms equal to the bit)
    const auto other = tune_cache.find(std::make_pair(S, grad ? 0 : 1));
    const bool have_fwd = other != tune_cache.end();
    if (have_fwd) { spt_f = other->second[0]; tz_f = other->second[1]; }
    for (int pass = 0; pass < (grad ? 2 : 1); ++pass) {
        if (pass == 0 && have_fwd) continue;
        const std::vector<int> tzs = tune_tz(pass);
        float best = 1e30f;
        int bs = 1, bt = tzs[std::min<size_t>(1, tzs.size() - 1)];
        for (int spt : tune_spt(pass)) {
            if (spt > S) break;
            for (int tz : tzs) {
                if (pass == 0) { spt_f = spt; tz_f = tz; } else { spt_a = spt; tz_a = tz; }
                // the forward variants the time loop launches (the fused injection,
                // without the sampling CTAs and the step counter); the adjoint's
                // fused work is the residual scatter of extra CTAs, whose residual
                // buffer does not exist yet: its stencil kernels are timed alone
                auto run = [&]() {
                    if (pass == 0) {
                        fz_mode = fuse_fwd ? FZ_INJ : 0;
                        launch_kernel(OWL_K_FWD_P, S, false);
                        launch_kernel(OWL_K_FWD_V, S, false);
                    } else {
                        launch_kernel(OWL_K_ADJ_P, S, false);
                        launch_kernel(OWL_K_ADJ_V, S, false);
                    }
                    fz_mode = 0;
                };
                run();
                run();
                OWL_LAUNCH_CHECK();
                EventTimer tm(stream);
                for (int i = 0; i < 8; ++i) run();
                float ms = (float)tm.stop_ms();
                launches += 20;
                if (ms < best) { best = ms; bs = spt; bt = tz; }
            }
        }
        if (pass == 0) { spt_f = bs; tz_f = bt; } else { spt_a = bs; tz_a = bt; }
    }
    tune_cache[key] = {spt_f, tz_f, spt_a, tz_a};
    tune_extra(S, k, grad);
}

void SsgBase::save_ckpt(int slot, int S) {
    const size_t n = (size_t)sst * S;
    if (ckpt_prec == OWL_CKPT_FP32) {
        OWL_CUDA(cudaMemcpyAsync(ckpt.p + slot * n, st.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream));
        return;
    }
    const int nseg = (int)st_segments.size();
    DevBuf<long long>& so = seg_off();
    SegDev sg{so.p, so.p + nseg, nseg};
    float* sc = ck_scale.p + (size_t)slot * S * nseg;
    dim3 g1(nseg, S);
    k_absmax<<<g1, 256, 0, stream>>>(st.p, sst, sg, sc);
    dim3 g2(nseg, S, 64);
    if (ckpt_prec == OWL_CKPT_BF16) k_pack<true><<<g2, 256, 0, stream>>>(st.p, sst, sg, sc, ckpt16.p + slot * n);
    else k_pack<false><<<g2, 256, 0, stream>>>(st.p, sst, sg, sc, ckpt16.p + slot * n);
    OWL_LAUNCH_CHECK();
    launches += 2;
}

void SsgBase::restore_ckpt(int slot, int S) {
    const size_t n = (size_t)sst * S;
    if (ckpt_prec == OWL_CKPT_FP32) {
        OWL_CUDA(cudaMemcpyAsync(st.p, ckpt.p + slot * n, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream));
        return;
    }
    const int nseg = (int)st_segments.size();
    DevBuf<long long>& so = seg_off();
    SegDev sg{so.p, so.p + nseg, nseg};
    const float* sc = ck_scale.p + (size_t)slot * S * nseg;
    dim3 g2(nseg, S, 64);
    if (ckpt_prec == OWL_CKPT_BF16) k_unpack<true><<<g2, 256, 0, stream>>>(ckpt16.p + slot * n, sst, sg, sc, st.p);
    else k_unpack<false><<<g2, 256, 0, stream>>>(ckpt16.p + slot * n, sst, sg, sc, st.p);
    OWL_LAUNCH_CHECK();
    launches += 1;
}

// save: a checkpoint at the start of every segment; store_last: the last
// segment's steps store their stencil terms (slot t % k, as its recompute
// would) and get no checkpoint
void SsgBase::forward_batch(int S, int k, bool graph, bool save, bool store_last) {
    const int nt = desc.nt;
    cur_k = k;
    PointDev q = pdev(S, false, false);
    OWL_CUDA(cudaMemsetAsync(st.p, 0, sizeof(float) * sst * S, stream));
    set_step(0);
    launch_point_fwd(q, S, nb_rec, PT_SAMPLE, stream);
    OWL_LAUNCH_CHECK();
    launches++;
    const int nseg = (nt + k - 1) / k;
    for (int sg = 0; sg < nseg; ++sg) {
        const bool last = store_last && sg == nseg - 1;
        if (save && !last) save_ckpt(sg, S);
        const int n = std::min(k, nt - sg * k);
        run_steps(last ? 3 : 0, n, S, q, graph && n == k);
    }
}

void SsgBase::check_nonfinite(const float* f, size_t n) {
    OWL_CUDA(cudaMemsetAsync(ctr.p + 2, 0, sizeof(int), stream));
    launch_check_finite(f, n, ctr.p + 2, stream);
    launches++;
    int flag = 0;
    OWL_CUDA(cudaMemcpyAsync(&flag, ctr.p + 2, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OWL_CUDA(cudaStreamSynchronize(stream));
    if (flag) throw OwlError(OWL_ERR_NONFINITE, "non-finite values in the wavefield");
}

void SsgBase::copy_out(void* dst, const void* src, size_t bytes, int mem) {
    OWL_CUDA(cudaMemcpyAsync(dst, src, bytes,
                             mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream));
}

void SsgBase::fill_info(owl_run_info& info, int nshots, int batches, bool grad) {
    info.gpu_launches = launches;
    // a gradient: forward, recompute of all but the last segment, adjoint
    const int kk = std::max(1, std::min(cur_k, desc.nt));
    const double passes = grad ? 2.0 + (double)((desc.nt + kk - 1) / kk - 1) * kk / desc.nt : 1.0;
    info.steps_cell_updates = passes * (double)NXp * NYp * NZp * desc.nt * nshots;
    info.dt_used = dt;
    info.dt_stable = dt_stable_;
    info.shots_per_cta = grad ? spt_a : spt_f;
    info.tile_x = tile_x;
    info.tile_z = grad ? tz_a : tz_f;
    info.batches = batches;
    info.checkpoint_interval = grad ? plan_k : 0;
    info.shots_per_launch = plan_B;
    info.tile_z_forward = tz_f;
    info.shots_per_cta_forward = spt_f;
}

void SsgBase::forward(int nshots, const owl_shot* shots, const owl_run_opts& o, float* seis, int mem,
                      owl_run_info& info) {
    OWL_CHECK(model_set, OWL_ERR_INVALID, "set_model must be called first");
    int B, k;
    bool graph;
    resolve_opts(o, nshots, shots, false, B, k, graph);
    launches = 0;
    EventTimer tm(stream);
    size_t out_off = 0;
    int batches = 0;
    for (int b0 = 0; b0 < nshots; b0 += B) {
        const int S = std::min(B, nshots - b0);
        build_tables(S, shots + b0, false);
        ensure_state(S, k, false);
        cur_S = S;
        if (tune) autotune(S, k, false);
        const size_t nrt = (size_t)desc.nt * std::max(rtot, 1);
        rec.reserve(nrt);
        OWL_CUDA(cudaMemsetAsync(rec.p, 0, sizeof(float) * nrt, stream));
        forward_batch(S, k, graph, false);
        if (o.check_every > 0) check_nonfinite(st.p, (size_t)S * sst);
        const size_t n = (size_t)rtot * dnt();
        if (n) {
            seis_tmp.reserve(n);
            syn_to_data(seis_tmp.p);
            copy_out(seis + out_off, seis_tmp.p, n * sizeof(float), mem);
        }
        out_off += n;
        batches++;
    }
    info.elapsed_ms = tm.stop_ms();
    check_timeout();
    fill_info(info, nshots, batches, false);
}

// Misfit-only batched forward (the trial forwards of the step-length search,
// src/inverse/module_inversion_step_size.f90:263-592): no checkpoints, no
// seismogram round trip unless asked for.
void SsgBase::misfit(int nshots, const owl_shot* shots, const float* obs, const owl_run_opts& o, double* misfit,
                     double* trace_misfit, float* seis_out, int mem, owl_run_info& info) {
    OWL_CHECK(model_set, OWL_ERR_INVALID, "set_model must be called first");
    int B, k;
    bool graph;
    resolve_opts(o, nshots, shots, false, B, k, graph);
    launches = 0;
    EventTimer tm(stream);
    size_t data_off = 0, tr_off = 0;
    int batches = 0, shot0 = 0;
    for (int b0 = 0; b0 < nshots; b0 += B) {
        const int S = std::min(B, nshots - b0);
        build_tables(S, shots + b0, false);
        ensure_state(S, k, false);
        cur_S = S;
        if (tune) autotune(S, k, false);
        const size_t nrt = (size_t)desc.nt * std::max(rtot, 1);
        rec.reserve(nrt);
        obs_t.reserve(nrt);
        OWL_CUDA(cudaMemsetAsync(rec.p, 0, sizeof(float) * nrt, stream));
        forward_batch(S, k, graph, false);
        if (o.check_every > 0) check_nonfinite(st.p, (size_t)S * sst);
        const int tn = dnt();
        const size_t n = (size_t)rtot * tn;
        misfit_d.reserve(S);
        trace_d.reserve(std::max(rtot, 1));
        obs_t.reserve(std::max(nrt, n));
        if (n) {
            seis_tmp.reserve(n);
            OWL_CUDA(cudaMemcpyAsync(seis_tmp.p, obs + data_off, n * sizeof(float),
                                     mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
            launch_transpose_seis_to_rec(seis_tmp.p, obs_t.p, tn, rtot, stream);
            launches++;
        }
        const float* syn_i = rec.p;  // synthetics at the data sampling, (tn, rtot)
        if (resampled() && n) {
            dat_a.reserve(n);
            dat_b.reserve(n);
            syn_to_data(dat_a.p);
            launch_transpose_seis_to_rec(dat_a.p, dat_b.p, tn, rtot, stream);
            launches++;
            syn_i = dat_b.p;
        }
        launch_trace_misfit(syn_i, obs_t.p, live.p, rec_shot_ptr.p, S, tn, rtot, trace_d.p, misfit_d.p, stream);
        launches += 2;
        if (misfit) copy_out(misfit + shot0, misfit_d.p, sizeof(double) * S, mem);
        if (trace_misfit && rtot) copy_out(trace_misfit + tr_off, trace_d.p, sizeof(double) * rtot, mem);
        if (seis_out && n) {
            if (resampled()) {
                copy_out(seis_out + data_off, dat_a.p, n * sizeof(float), mem);
            } else {
                launch_transpose_rec_to_seis(rec.p, seis_tmp.p, desc.nt, rtot, stream);
                launches++;
                copy_out(seis_out + data_off, seis_tmp.p, n * sizeof(float), mem);
            }
        }
        OWL_CUDA(cudaStreamSynchronize(stream));
        data_off += n;
        tr_off += (size_t)rtot;
        shot0 += S;
        batches++;
    }
    info.elapsed_ms = tm.stop_ms();
    check_timeout();
    fill_info(info, nshots, batches, false);
}

void SsgBase::fold_out(float* grad, int mem) {
    const size_t nm = (size_t)nx * ny * nz;
    seis_tmp.reserve((size_t)nparam * nm);
    for (int p = 0; p < nparam; ++p) {
        k_fold<<<148 * 4, 256, 0, stream>>>(gpad.p + (size_t)p * npad(), nxq(), nyq(), P, nx, ny, nz, dim,
                                            seis_tmp.p + (size_t)p * nm);
        launches++;
    }
    OWL_LAUNCH_CHECK();
    copy_out(grad, seis_tmp.p, (size_t)nparam * nm * sizeof(float), mem);
}

void SsgBase::syn_to_data(float* out) {
    if (!resampled()) {
        launch_transpose_rec_to_seis(rec.p, out, desc.nt, rtot, stream);
        launches++;
        return;
    }
    syn_t.reserve((size_t)rtot * desc.nt);
    launch_transpose_rec_to_seis(rec.p, syn_t.p, desc.nt, rtot, stream);
    launch_resample_rows(syn_t.p, desc.nt, dt, 0.0, out, data_nt, data_dt, 0.0, rtot, stream);
    launches += 2;
}

void SsgBase::data_to_res(const float* rows) {
    if (!resampled()) {
        launch_transpose_seis_to_rec(rows, res.p, desc.nt, rtot, stream);
        launches++;
        return;
    }
    adj_t.reserve((size_t)rtot * desc.nt);
    launch_resample_rows(rows, data_nt, data_dt, 0.0, adj_t.p, desc.nt, dt, 0.0, rtot, stream);
    launch_transpose_seis_to_rec(adj_t.p, res.p, desc.nt, rtot, stream);
    launches += 2;
}

// Adjoint source of a batch whose data are sampled off the time axis, as the
// reference orders it: synthetics resampled to the data sampling
// (submodule_forward_modeling.f90:124-125), the adjoint source computed there,
// and resampled back to the time axis before injection
// (submodule_fwi_gradient.f90:46).
void SsgBase::data_adjoint_source(const float* data, int adj_kind, int mem, int S, float* seis_out) {
    const int tn = dnt();
    const size_t n = (size_t)rtot * tn;
    seis_tmp.reserve(n);
    OWL_CUDA(cudaMemcpyAsync(seis_tmp.p, data, n * sizeof(float),
                             mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
    dat_a.reserve(n);
    dat_b.reserve(n);
    syn_to_data(dat_a.p);
    if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
        obs_t.reserve(n);
        syn_t.reserve(std::max(n, (size_t)rtot * desc.nt));
        launch_transpose_seis_to_rec(seis_tmp.p, obs_t.p, tn, rtot, stream);
        launch_transpose_seis_to_rec(dat_a.p, dat_b.p, tn, rtot, stream);
        launch_residual_l2(dat_b.p, obs_t.p, syn_t.p, live.p, rec_shot_ptr.p, S, tn, rtot, misfit_d.p, stream);
        launch_transpose_rec_to_seis(syn_t.p, dat_b.p, tn, rtot, stream);
        launches += 4;
        data_to_res(dat_b.p);
    } else if (adj_kind == ADJ_MISFIT) {
        owl_misfit_opts mo = mopts;
        mo.dt = data_dt;
        if (mo.ncomp <= 0) mo.ncomp = ncomp;  // dtw-vector: the components of a shot are its ncomp gathers
        // adj_nt defaults to the time axis' nt (module_parameters.f90:552): the misfit of data
        // sampled differently is taken on traces resampled to nt samples (DTW: its shifts)
        if (mo.adj_nt <= 0) mo.adj_nt = desc.nt;
        trace_d.reserve(std::max(rtot, 1));
        adjsrc.launches = 0;
        adjsrc.run(mo, (int)h_gather_ptr.size() - 1, h_gather_ptr.data(), tn, dat_a.p, seis_tmp.p, live.p, dat_b.p,
                   trace_d.p, nullptr, stream);
        launch_shot_misfit(trace_d.p, rec_shot_ptr.p, S, misfit_d.p, stream);
        launches += adjsrc.launches + 1;
        data_to_res(dat_b.p);
    } else {
        data_to_res(seis_tmp.p);
    }
    if (seis_out) copy_out(seis_out, dat_a.p, n * sizeof(float), mem);
}

void SsgBase::gradient_impl(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                            double* misfit, float* grad, float* seis_out, float* stf_grad, int mem,
                            owl_run_info& info) {
    OWL_CHECK(model_set, OWL_ERR_INVALID, "set_model must be called first");
    OWL_CHECK(adj_kind == OWL_ADJ_L2_RESIDUAL || adj_kind == OWL_ADJ_GIVEN || adj_kind == ADJ_MISFIT,
              OWL_ERR_INVALID, "bad adj_kind");
    int B, k;
    bool graph;
    resolve_opts(o, nshots, shots, true, B, k, graph);
    launches = 0;
    const int nt = desc.nt;
    EventTimer tm(stream);
    gpad.reserve((size_t)grad_planes() * npad());
    OWL_CUDA(cudaMemsetAsync(gpad.p, 0, sizeof(double) * grad_planes() * npad(), stream));
    size_t data_off = 0, stf_off = 0;
    int batches = 0, shot0 = 0;
    for (int b0 = 0; b0 < nshots; b0 += B) {
        const int S = std::min(B, nshots - b0);
        const owl_shot* sh = shots + b0;
        build_tables(S, sh, true);
        ensure_state(S, k, true);
        cur_S = S;
        cur_k = k;
        if (tune) autotune(S, k, true);
        const int groups = (S + spt_a - 1) / spt_a;
        const int nseg = (nt + k - 1) / k;
        if (ckpt_prec == OWL_CKPT_FP32) {
            ckpt.reserve((size_t)nseg * sst * S);
        } else {
            ckpt16.reserve((size_t)nseg * sst * S);
            ck_scale.reserve((size_t)nseg * S * st_segments.size());
        }
        const size_t nrt = (size_t)nt * std::max(rtot, 1);
        rec.reserve(nrt);
        res.reserve(nrt);
        obs_t.reserve(nrt);
        OWL_CUDA(cudaMemsetAsync(rec.p, 0, sizeof(float) * nrt, stream));
        bool want_src = stf_grad != nullptr;
        for (long long rc : item_rho_cell) want_src |= rc >= 0;
        const size_t nitems = item_src.size();
        src_adj.reserve(std::max<size_t>(1, nitems * nt));
        if (want_src) OWL_CUDA(cudaMemsetAsync(src_adj.p, 0, sizeof(float) * std::max<size_t>(1, nitems * nt), stream));
        // 1. forward with checkpoints; the last segment stores its stencil terms
        // the forward stores the last segment's stencil terms (no recompute of
        // it); OWL_NO_STORE_LAST=1 checkpoints and recomputes it like the others
        // (the tests compare the two)
        const bool store_last = std::getenv("OWL_NO_STORE_LAST") == nullptr;
        forward_batch(S, k, graph, true, store_last);
        if (o.check_every > 0) check_nonfinite(st.p, (size_t)S * sst);
        // 2. adjoint source and misfit
        const size_t n = (size_t)rtot * dnt();
        misfit_d.reserve(S);
        OWL_CUDA(cudaMemsetAsync(misfit_d.p, 0, sizeof(double) * S, stream));
        if (n && resampled()) {
            data_adjoint_source(data + data_off, adj_kind, mem, S, seis_out ? seis_out + data_off : nullptr);
        } else if (n) {
            seis_tmp.reserve(n);
            OWL_CUDA(cudaMemcpyAsync(seis_tmp.p, data + data_off, n * sizeof(float),
                                     mem == OWL_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
            launch_transpose_seis_to_rec(seis_tmp.p, obs_t.p, nt, rtot, stream);
            launches++;
            if (adj_kind == OWL_ADJ_L2_RESIDUAL) {
                launch_residual_l2(rec.p, obs_t.p, res.p, live.p, rec_shot_ptr.p, S, nt, rtot, misfit_d.p, stream);
                launches++;
            } else if (adj_kind == ADJ_MISFIT) {
                // compute_adjoint_source on the trace-major gathers of the batch
                // (seis_tmp holds the observed traces as uploaded)
                syn_t.reserve(n);
                adj_t.reserve(n);
                trace_d.reserve(rtot);
                launch_transpose_rec_to_seis(rec.p, syn_t.p, nt, rtot, stream);
                adjsrc.launches = 0;
                owl_misfit_opts mo = mopts;
                if (mo.ncomp <= 0) mo.ncomp = ncomp;  // dtw-vector: the components of a shot are its ncomp gathers
                adjsrc.run(mo, (int)h_gather_ptr.size() - 1, h_gather_ptr.data(), nt, syn_t.p, seis_tmp.p,
                           live.p, adj_t.p, trace_d.p, nullptr, stream);
                launch_shot_misfit(trace_d.p, rec_shot_ptr.p, S, misfit_d.p, stream);
                launch_transpose_seis_to_rec(adj_t.p, res.p, nt, rtot, stream);
                launches += adjsrc.launches + 3;
            } else {
                OWL_CUDA(cudaMemcpyAsync(res.p, obs_t.p, n * sizeof(float), cudaMemcpyDeviceToDevice, stream));
            }
            if (seis_out) {
                launch_transpose_rec_to_seis(rec.p, seis_tmp.p, nt, rtot, stream);
                launches++;
                copy_out(seis_out + data_off, seis_tmp.p, n * sizeof(float), mem);
            }
        }
        if (misfit) copy_out(misfit + shot0, misfit_d.p, sizeof(double) * S, mem);
        // 3. reverse sweep: restore a checkpoint, recompute its segment storing
        //    the stencil terms, run the exact adjoint back through it (the last
        //    segment's terms are already stored by the forward)
        OWL_CUDA(cudaMemsetAsync(ad.p, 0, sizeof(float) * sad * S, stream));
        OWL_CUDA(cudaMemsetAsync(G.p, 0, sizeof(float) * 2 * ngrad * groups * fs, stream));
        PointDev qf = pdev(S, false, false);
        PointDev qa = pdev(S, true, want_src);
        want_src_now = want_src;
        for (int sg = nseg - 1; sg >= 0; --sg) {
            const int n0 = sg * k, nn = std::min(k, nt - n0);
            if (sg == nseg - 1 && store_last) {
                set_step(nt);
            } else {
                restore_ckpt(sg, S);
                set_step(n0);
                run_steps(1, nn, S, qf, graph && nn == k);
            }
            run_steps(2, nn, S, qa, graph && nn == k);
        }
        want_src_now = false;
        if (o.check_every > 0) check_nonfinite(ad.p, (size_t)S * sad);
        // 4. chain rule (FP64) into the padded accumulators
        chain_rule(S, groups);
        // 5. source-side terms: rho of force sources, STF gradient
        if (want_src && nitems) {
            std::vector<float> hsa(nitems * nt), hamp(nitems * nt);
            OWL_CUDA(cudaMemcpyAsync(hsa.data(), src_adj.p, sizeof(float) * nitems * nt, cudaMemcpyDeviceToHost, stream));
            OWL_CUDA(cudaMemcpyAsync(hamp.data(), amp.p, sizeof(float) * nitems * nt, cudaMemcpyDeviceToHost, stream));
            OWL_CUDA(cudaStreamSynchronize(stream));
            std::map<long long, double> pts;
            for (size_t it = 0; it < nitems; ++it) {
                if (item_rho_cell[it] < 0) continue;
                double acc = 0;
                for (int t = 0; t < nt; ++t) acc += (double)hamp[it * nt + t] * (double)hsa[it * nt + t];
                // the force weights carry 1/rho: d/drho (A w lambda) = -A w lambda / rho
                pts[item_rho_cell[it] + (long long)rho_param() * (long long)npad()] += -acc / (double)item_rho[it];
            }
            if (!pts.empty()) {
                std::vector<long long> hi;
                std::vector<double> hv;
                for (auto& kv : pts) { hi.push_back(kv.first); hv.push_back(kv.second); }
                DevBuf<long long> didx;
                didx.upload(hi.data(), hi.size(), stream);
                pt_val.upload(hv.data(), hv.size(), stream);
                k_add_points_f64<<<(int)(hi.size() + 127) / 128, 128, 0, stream>>>(gpad.p, didx.p, pt_val.p,
                                                                                   (int)hi.size());
                OWL_LAUNCH_CHECK();
                OWL_CUDA(cudaStreamSynchronize(stream));
                launches++;
            }
            if (stf_grad) {
                for (int s = 0; s < S; ++s) {
                    const owl_shot& shs = sh[s];
                    for (int kk = 0; kk < shs.nsrc; ++kk)
                        std::fill(stf_grad + stf_off + (size_t)kk * nt, stf_grad + stf_off + (size_t)(kk + 1) * nt, 0.f);
                    for (size_t it = 0; it < nitems; ++it) {
                        if (item_shot[it] != s) continue;
                        const owl_source& q = shs.src[item_src[it]];
                        float* outk = stf_grad + stf_off + (size_t)item_src[it] * nt;
                        for (int t = 0; t < nt; ++t)
                            outk[t] += (float)((double)hsa[it * nt + t] * (double)q.amp * (double)dt);
                    }
                    stf_off += (size_t)shs.nsrc * nt;
                }
            }
        }
        data_off += n;
        shot0 += S;
        batches++;
    }
    if (grad) fold_out(grad, mem);
    info.elapsed_ms = tm.stop_ms();
    check_timeout();
    fill_info(info, nshots, batches, true);
}

void SsgBase::gradient(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                       double* misfit, float* grad, float* seis_out, int mem, owl_run_info& info) {
    gradient_impl(nshots, shots, data, adj_kind, o, misfit, grad, seis_out, nullptr, mem, info);
}

void SsgBase::source_gradient(int nshots, const owl_shot* shots, const float* adj, const owl_run_opts& o,
                              float* stf_grad, int mem, owl_run_info& info) {
    OWL_CHECK(mem == OWL_MEM_HOST, OWL_ERR_UNSUPPORTED, "source_gradient takes host buffers");
    gradient_impl(nshots, shots, adj, OWL_ADJ_GIVEN, o, nullptr, nullptr, nullptr, stf_grad, mem, info);
}

void SsgBase::kernel_time(int id, int nlaunch, double* avg_ms, double* bytes) {
    OWL_CHECK(cur_S > 0, OWL_ERR_INVALID, "no batch has run on this handle");
    OWL_CHECK(id >= OWL_K_FWD_P && id <= OWL_K_FWD_V_STORE, OWL_ERR_INVALID, "bad kernel id");
    const int S = cur_S;
    const bool store = id == OWL_K_FWD_P_STORE || id == OWL_K_FWD_V_STORE;
    const int kid = store ? id - OWL_K_FWD_P_STORE : id;
    OWL_CHECK((kid < OWL_K_ADJ_P && !store) ||
                  (ad.p && G.p && Sbuf.p && ad.n >= (size_t)sad * S && Sbuf.n >= (size_t)nS * cur_k * S * fs),
              OWL_ERR_INVALID, "adjoint kernels and store variants need a gradient call first");
    set_step(cur_k);
    // the variant the time loop launches, without advancing the step counter
    const int fz = kid < OWL_K_ADJ_P ? (fuse_fwd ? FZ_INJ : 0) : (fuse_on ? FZ_SCT : 0);
    fz_mode = fz;
    for (int i = 0; i < 3; ++i) launch_kernel(kid, S, store);
    OWL_LAUNCH_CHECK();
    if (kid >= OWL_K_ADJ_P || store) {
        // kernels that read or write the segment's stored stencil terms: each
        // launch at another step of the segment, so that the terms stream from
        // HBM as in the time loop (the same slot every launch would stay in L2);
        // each launch timed alone, the step counter set between them
        std::vector<cudaEvent_t> ev(2 * (size_t)nlaunch);
        for (auto& e : ev) OWL_CUDA(cudaEventCreate(&e));
        for (int i = 0; i < nlaunch; ++i) {
            const int slot = i % std::max(1, cur_k);
            set_step(kid >= OWL_K_ADJ_P ? cur_k - slot : slot);
            OWL_CUDA(cudaEventRecord(ev[2 * (size_t)i], stream));
            launch_kernel(kid, S, store);
            OWL_CUDA(cudaEventRecord(ev[2 * (size_t)i + 1], stream));
        }
        fz_mode = 0;
        OWL_LAUNCH_CHECK();
        OWL_CUDA(cudaEventSynchronize(ev.back()));
        double tot = 0;
        for (int i = 0; i < nlaunch; ++i) {
            float ms = 0;
            OWL_CUDA(cudaEventElapsedTime(&ms, ev[2 * (size_t)i], ev[2 * (size_t)i + 1]));
            tot += ms;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        *avg_ms = tot / nlaunch;
    } else {
        EventTimer tm(stream);
        for (int i = 0; i < nlaunch; ++i) launch_kernel(kid, S, store);
        fz_mode = 0;
        OWL_LAUNCH_CHECK();
        *avg_ms = tm.stop_ms() / nlaunch;
    }
    check_timeout();
    *bytes = alg_bytes(kid, S, (S + spt_a - 1) / spt_a);
    if (store) {
        const int terms = kid == OWL_K_FWD_P ? n_store_p() : nS - n_store_p();
        *bytes += 4.0 * terms * (double)S * NXp * NYp * NZp;
    }
}

}  // namespace owl
