// ssg_base.cuh -- medium-independent host engine of the SSG solvers.
//
// A medium (2D/3D acoustic, 2D/3D elastic) supplies its stencil kernels, its
// source / receiver taps and its chain rule; this base supplies everything
// around them: point-operator tables (source injection, receiver sampling,
// adjoint-source injection), the shot-batched state, every-k-step checkpoints
// (FP32 or FP16 / BF16 with a per-field, per-shot scale), the device step
// counter and CUDA-graph capture of the time loop, the gradient driver
// (forward -> FP64 misfit / residual -> reverse sweep with segment
// recomputation -> FP64 chain rule -> fold onto the model cells), the
// autotuner and kernel timing.
//
// Layouts. Storage index of the reference's node (i, j, k) (x, y, z; 1-based,
// padded range [-pml-R+1, n+pml+R]) is x = i + pml + R - 1 (same for y, z);
// a field is (NZs, NYs, pitch) floats with x fastest (NYs = 1 in 2D). The
// forward state and the adjoint state are shot-major: shot s of field f lives
// at base + s * shot_stride + field_offset[f].
#pragma once

#include <array>
#include <map>
#include <vector>

#include "adjsrc.cuh"
#include "engine.cuh"

namespace owl {

constexpr int MAX_PT_FIELDS = 10;

struct PointDev {
    float* fld[MAX_PT_FIELDS];
    long long sstride;  // shot stride of the fields
    int nt, rtot;
    CSRView inj;
    const int* inj_shot_ptr;
    const float* amp;
    CSRView smp;
    const int* rec_shot_ptr;
    float* rec;
    CSRView sct;
    const int* sct_shot_ptr;
    const float* res;
    float* src_adj;
    int* d_step;
    int* d_done;
};

enum { PT_INJECT = 1, PT_SAMPLE = 2, PT_TICK = 4, PT_NEXT = 8 };  // forward point kernel phases
// point work fused into a medium's stencil kernels (media that support it):
// FZ_INJ source injection by the owner of each tap node, FZ_SMP receiver
// sampling by extra CTAs of the velocity kernel, FZ_TICK the step counter
// advanced by the last CTA, FZ_SCT the residual scatter by extra CTAs of the
// adjoint velocity-node kernel
enum { FZ_INJ = 1, FZ_SMP = 2, FZ_TICK = 4, FZ_SCT = 8 };
constexpr int BOX_W = 9;  // taps of a source along each axis (the 9-tap Kaiser sinc)
// adjoint point kernel phases. PA_SRC records the source-side adjoint of step
// t-1 after the scatter; PA_SRC_NOW records that of step t from the fields as
// they are (media whose adjoint kernels interleave with the source terms)
enum { PA_SCATTER = 1, PA_SRC = 2, PA_TICK = 4, PA_SRC_NOW = 8 };

void launch_point_fwd(const PointDev& q, int S, int nb, int mode, cudaStream_t s);
void launch_point_adj(const PointDev& q, int S, int nb, int mode, cudaStream_t s);
// padded-grid FP64 gradient -> model cells, the adjoint of the edge padding
void launch_fold(const double* gp, int nxq, int nyq, int P, int nx, int ny, int nz, int dim, float* out,
                 cudaStream_t s);

// one interpolation tap of a source / receiver on field `field` at reference node (i, j, k)
struct TapPt {
    int field;
    int i, j, k;
    float w;
};

struct SsgBase : Engine {
    // grid
    int dim, nx, ny, nz, P, R, pr, NXp, NYp, NZp, NXs, NYs, NZs, pitch;
    long long plane, fs;  // floats per z-plane and per full field
    float dt;
    // layout sizes, set by the medium
    long long sst = 0;   // floats of forward state per shot
    long long sad = 0;   // floats of adjoint state per shot
    int nS = 0;          // full fields stored per step in the segment buffer
    int ngrad = 0;       // gradient accumulators (each with a Kahan compensation)
    int nparam = 0;      // model parameters
    int ncomp = 1;       // seismogram components
    std::vector<std::pair<long long, long long>> st_segments;  // (offset, length) of each state field in a shot

    // buffers
    DevBuf<float> st, ad, G, Sbuf, ckpt, ck_scale;
    DevBuf<unsigned short> ckpt16;
    DevBuf<int> ctr;
    DevBuf<float> rec, res, obs_t, src_adj, seis_tmp, amp;
    DevBuf<double> gpad, misfit_d, pt_val, trace_d;
    DevBuf<int> pt_idx;
    DevCSR inj, smp, sct;
    DevBuf<int> inj_shot_ptr, rec_shot_ptr, sct_shot_ptr;
    // each injection item's taps as a dense BOX_W^dim box: (field, x0, y0, z0)
    // storage coordinates of its lowest corner, weights [z][y][x] (0 off the taps)
    DevBuf<int4> inj_box;
    DevBuf<float> inj_bw;
    // per shot: bounding boxes (x0, x1, z0, z1; storage) of its taps on field 0,
    // then on every other field (2D media)
    DevBuf<int4> inj_bbox;
    bool fuse_on = false;  // this batch's point work runs inside the stencil kernels
    bool fuse_fwd = false; // ... in the forward steps too (else only the adjoint's residual scatter)
    int inj_fmask = 0;     // fields the batch's sources inject into (bit f: field f)
    bool want_src_now = false;  // the adjoint sweep records the source-side adjoint
    int fz_mode = 0;       // FZ_* work of the next stencil launches
    DevBuf<unsigned char> live;
    DevBuf<long long> segbuf;  // st_segments offsets then lengths, on the device
    GraphCache g_fwd, g_rec, g_adj, g_fst;

    long long launches = 0;
    int cur_k = 0, cur_S = 0, tile_x = 32;
    bool tune = false;
    int spt_f = 1, spt_a = 1, tz_f = 8, tz_a = 8;
    int ckpt_prec = OWL_CKPT_FP32;
    int rtot = 0;
    int nb_rec = 1, nb_sct = 1;  // CTAs per shot of the sampling / adjoint-injection point kernels
    std::vector<int> item_src, item_comp, item_shot;
    std::vector<long long> item_rho_cell;  // padded-grid index of the rho scaling a force component, -1 otherwise
    std::vector<float> item_rho;
    std::map<std::pair<int, int>, std::array<int, 4>> tune_cache;
    std::vector<float> h_rhop;  // padded rho, storage layout (force-source weights)
    std::vector<int> h_gather_ptr;  // trace ranges of the (shot, component) gathers of the batch
    AdjointSource adjsrc;
    DevBuf<float> syn_t, adj_t;     // trace-major synthetics / adjoint source (data-domain misfits)
    DevBuf<float> dat_a, dat_b;     // traces at the data sampling (resampled runs)
    // seismograms at a sampling other than the time axis (resample_su, src/lib/module_su.f90:426-470)
    bool resampled() const { return data_nt > 0 && (data_nt != desc.nt || data_dt != dt); }
    int dnt() const { return data_nt > 0 ? data_nt : desc.nt; }
    // synthetics of the batch (rec, (nt, rtot)) -> rows of dnt() samples at the data sampling
    void syn_to_data(float* out);
    // rows of dnt() samples at the data sampling -> adjoint source on the time axis in res ((nt, rtot))
    void data_to_res(const float* rows);
    // adjoint source of the batch from data at the data sampling (forward already run)
    void data_adjoint_source(const float* data, int adj_kind, int mem, int S, float* seis_out);

    SsgBase(const owl_ssg_desc& d, int dim_);
    ~SsgBase() override;

    // ---------------- medium hooks ----------------
    virtual int src_ncomp(const owl_source& q) const = 0;
    virtual void src_taps(const owl_source& q, int comp, std::vector<TapPt>& taps, long long& rho_cell,
                          float& rho_val) const = 0;
    virtual void rec_taps(const owl_receiver& q, int comp, std::vector<TapPt>& taps) const = 0;
    // adjoint of one sampling tap (free-surface images route through the mirrored node)
    virtual void scatter_map(const TapPt& t, std::vector<TapPt>& out) const { out.push_back(t); }
    virtual void launch_kernel(int id, int S, bool store) = 0;
    virtual double alg_bytes(int id, int S, int groups) const = 0;
    // stencil terms written per cell by the store variant of the p / stress kernel
    // (the velocity kernel writes the other nS - n_store_p)
    virtual int n_store_p() const { return 1; }
    virtual void chain_rule(int S, int groups) = 0;  // += into gpad
    virtual int rho_param() const = 0;
    virtual float* st_field(int f) const = 0;  // base pointer (shot 0) of forward field f
    virtual float* ad_field(int f) const = 0;  // base pointer (shot 0) of adjoint field f
    // autotuner candidates of pass 0 (forward kernels) / 1 (adjoint kernels): shots
    // per CTA and the kernel's second launch parameter (tile height, rows per
    // thread or rows per chunk, as the medium's kernels define it)
    virtual std::vector<int> tune_spt(int pass) const;
    virtual std::vector<int> tune_tz(int pass) const;
    // tile_x / tile_z of the run options (validated), spt_f / spt_a already set
    virtual void launch_params(const owl_run_opts& o);
    // point work inside the stencil kernels: whether the medium's kernels do it,
    // and whether an injection / sampling tap of `field` at storage (x, y, z)
    // lies in the nodes its kernel updates (else the batch keeps the point kernels)
    virtual bool fuse_supported() const { return false; }
    virtual bool fuse_tap_ok(int field, int x, int y, int z, bool sampling) const {
        (void)field; (void)x; (void)y; (void)z; (void)sampling;
        return false;
    }
    // launches of one time step of `kind` (launch_step)
    virtual int step_launches(int kind) const;
    // medium-specific tuning after the shared autotuner (S shots per launch)
    virtual void tune_extra(int S, int k, bool grad) { (void)S; (void)k; (void)grad; }

    // ---------------- helpers ----------------
    long long soff(int i, int j, int k) const {
        return (long long)(k + pr - 1) * plane + (dim == 3 ? (long long)(j + pr - 1) * pitch : 0LL) + (i + pr - 1);
    }
    // padded model grid [-P, n+P+1] per axis
    int nxq() const { return NXp + 2; }
    int nyq() const { return dim == 3 ? NYp + 2 : 1; }
    int nzq() const { return NZp + 2; }
    size_t npad() const { return (size_t)nxq() * nyq() * nzq(); }
    long long pad_index(int i, int j, int k) const {
        return ((long long)(k + P) * nyq() + (dim == 3 ? (j + P) : 0)) * nxq() + (i + P);
    }
    bool in_wavefield(int i, int j, int k) const {
        bool ok = i >= -P - R + 1 && i <= nx + P + R && k >= -P - R + 1 && k <= nz + P + R;
        if (dim == 3) ok = ok && j >= -P - R + 1 && j <= ny + P + R;
        return ok;
    }
    dim3 grid_for(int rows, int S, int spt, int tz) const {
        return dim3((NXp + tile_x - 1) / tile_x, (rows + tz - 1) / tz, (S + spt - 1) / spt);
    }

    DevBuf<long long>& seg_off();
    void set_step(int v);
    void build_tables(int S, const owl_shot* shots, bool need_sct);
    void ensure_state(int S, int k, bool grad);
    PointDev pdev(int S, bool adjoint, bool want_src_adj);
    virtual void launch_step(int kind, int S, const PointDev& q);
    // all n steps of a segment of kind `kind` as one persistent launch, where
    // the medium has one and it is selected; false: run_steps launches per step
    virtual bool run_steps_persistent(int kind, int n, int S) {
        (void)kind; (void)n; (void)S;
        return false;
    }
    void run_steps(int kind, int n, int S, const PointDev& q, bool graph);
    void resolve_opts(const owl_run_opts& o, int nshots, const owl_shot* shots, bool grad, int& B, int& k,
                      bool& graph);
    // device bytes one batch of S shots needs (k: checkpoint interval of a gradient)
    double batch_bytes(int S, int k, bool grad, int rec_per_shot) const;
    // bytes of the buffers a new batch would reuse or replace
    double held_bytes() const;
    int plan_k = 0, plan_B = 0;  // the last call's checkpoint interval and shots per batch
    void autotune(int S, int k, bool grad);
    void save_ckpt(int slot, int S);
    void restore_ckpt(int slot, int S);
    void forward_batch(int S, int k, bool graph, bool save, bool store_last = false);
    void check_nonfinite(const float* f, size_t n);
    void check_timeout();  // OWL_ERR_TIMEOUT if a kernel's bounded wait gave up
    void copy_out(void* dst, const void* src, size_t bytes, int mem);
    virtual void fold_out(float* grad, int mem);
    // FP64 planes of the padded gradient accumulator gpad (the model parameters;
    // a medium may keep other per-cell sums there that fold_out maps)
    virtual int grad_planes() const { return nparam; }
    void invalidate_graphs();
    void fill_info(owl_run_info& info, int nshots, int batches, bool grad);

    void forward(int nshots, const owl_shot* shots, const owl_run_opts& o, float* seis, int mem,
                 owl_run_info& info) override;
    void gradient(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                  double* misfit, float* grad, float* seis_out, int mem, owl_run_info& info) override;
    void source_gradient(int nshots, const owl_shot* shots, const float* adj, const owl_run_opts& o, float* stf_grad,
                         int mem, owl_run_info& info) override;
    void kernel_time(int id, int nlaunch, double* avg_ms, double* alg_bytes) override;
    void misfit(int nshots, const owl_shot* shots, const float* obs, const owl_run_opts& o, double* misfit,
                double* trace_misfit, float* seis_out, int mem, owl_run_info& info) override;
    void gradient_impl(int nshots, const owl_shot* shots, const float* data, int adj_kind, const owl_run_opts& o,
                       double* misfit, float* grad, float* seis_out, float* stf_grad, int mem, owl_run_info& info);
};

}  // namespace owl
