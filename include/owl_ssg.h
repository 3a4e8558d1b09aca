/*
 * owl_ssg.h -- C ABI of the B200 standard-staggered-grid (SSG) finite-difference
 * solver: forward modelling and adjoint-state FWI gradients for the media of
 * OWL's SSG solvers.
 *
 * The ABI replaces the type-bound procedures of OWL's solver objects:
 *   wave_solver_acoustic_iso_2d%forward / %adjoint
 *       src/solver/acoustic_iso_2d/interface.f90:30-60
 *   wave_solver_acoustic_iso_3d%forward / %adjoint
 *       src/solver/acoustic_iso_3d/interface.f90:30-60
 *   wave_solver_elastic_vhtiort_2d%forward / %adjoint
 *       src/solver/elastic_vhtiort_2d/interface.f90:29-77
 *   wave_solver_elastic_vhtiort_3d%forward / %adjoint
 *       src/solver/elastic_vhtiort_3d/interface.f90:30-79
 * One handle holds what the Fortran module variables hold there (padded model,
 * CFS-PML coefficients, wavefields), but per handle, so handles are re-entrant.
 *
 * Conventions shared with the reference:
 *   - model and gradient arrays are float32 (nz, nx) or (nz, ny, nx) with z
 *     fastest, i.e. the raw layout of OWL's model files
 *     (src/lib/module_model.f90:237-334) and of grad_<name>.bin outputs
 *     (src/inverse/2d/module_gradient.f90:454-468);
 *   - source / receiver node indices gx, gz, hx, hz and the 9-tap Kaiser
 *     windowed sinc vectors are exactly those of prepare_geometry
 *     (src/lib/module_source_receiver.f90:556-830), 1-based;
 *   - the source time function is the prepared STF (prepare_stf,
 *     src/lib/module_source_receiver.f90:1002-1130), injected from step nbeg.
 *
 * Every entry point returns OWL_OK (0) or a negative status; it never aborts
 * the process. owl_last_error() returns a thread-local message for the last
 * failure. Calls on one handle are not thread safe; distinct handles are.
 */
#ifndef OWL_SSG_H
#define OWL_SSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OWL_SSG_ABI_VERSION 10

/* status codes */
#define OWL_OK 0
#define OWL_ERR_INVALID (-1)     /* bad argument or descriptor */
#define OWL_ERR_CUDA (-2)        /* CUDA runtime error */
#define OWL_ERR_OOM (-3)         /* device allocation failed */
#define OWL_ERR_NONFINITE (-4)   /* NaN / Inf detected in a wavefield */
#define OWL_ERR_UNSTABLE (-5)    /* dt above the CFL bound and no adjustment allowed */
#define OWL_ERR_TIMEOUT (-6)     /* a bounded device wait gave up */
#define OWL_ERR_UNSUPPORTED (-7) /* medium / option not built */
#define OWL_ERR_NO_DEVICE (-8)   /* no usable CUDA device */

/* media (which_medium in OWL's parameter files, src/lib/module_parameters.f90:397) */
#define OWL_ACOUSTIC_ISO_2D 1
#define OWL_ACOUSTIC_ISO_3D 2
#define OWL_ELASTIC_VHTIORT_2D 3
#define OWL_ELASTIC_VHTIORT_3D 4

/* parameterisations of the elastic 2D medium (anisotropy_type,
 * src/solver/elastic_vhtiort_2d/module_vars.f90:235-296) */
#define OWL_ANISO_ISO 0     /* vp, vs, rho */
#define OWL_ANISO_THOMSEN 1 /* vp, vs, epsilon, delta, theta, rho */
#define OWL_ANISO_AT 2      /* vp, vs, epsilon, eta, theta, rho (Alkhalifah-Tsvankin) */
#define OWL_ANISO_CIJ 3     /* c11, c13, c33, c55, rho */

/* source mechanisms (src/lib/module_source_receiver.f90:66-83) */
#define OWL_SRC_EXPLOSION 0
#define OWL_SRC_FORCE 1
#define OWL_SRC_MT 2

/* memory kinds of the data buffers passed to forward / gradient. Device
 * buffers must hold their final contents, and no other work may still be
 * using them, when a call starts (synchronise the stream that produced them);
 * every call returns after its own GPU work has finished. */
#define OWL_MEM_HOST 0
#define OWL_MEM_DEVICE 1

/* checkpoint storage precision */
#define OWL_CKPT_FP32 0
#define OWL_CKPT_FP16 1
#define OWL_CKPT_BF16 2

/* adjoint-source kinds for owl_ssg_gradient */
#define OWL_ADJ_L2_RESIDUAL 0 /* adj = syn - obs, misfit = sum (obs - syn)^2 */
#define OWL_ADJ_GIVEN 1       /* adj given directly (the reference's adjoint SU) */

/* data-domain misfits (misfit_type, src/inverse/module_inversion_adjoint_source.f90:1099-1145) */
#define OWL_MISFIT_WAVEFORM 0 /* compute_adjsrc_waveform :371-383 */
#define OWL_MISFIT_CORR 1     /* compute_adjsrc_corr :391-412 (normalised zero-lag correlation) */
#define OWL_MISFIT_ENVELOPE 2 /* compute_adjsrc_envelope :424-451 */
#define OWL_MISFIT_PHASE 3    /* compute_adjsrc_phase :459-482 (instantaneous phase) */
#define OWL_MISFIT_ADAPTIVE 4 /* compute_adjsrc_adaptive :490-537 (adaptive waveform inversion) */
#define OWL_MISFIT_DTW 5      /* compute_adjsrc_dtw :715-980, solve_gdtw :73-234 (dynamic time warping) */
#define OWL_MISFIT_LOCAL_ADAPTIVE 6     /* compute_adjsrc_local_adaptive :545-625 (Gaussian-windowed AWI) */
#define OWL_MISFIT_ADAPTIVE_SPACETIME 7 /* compute_adjsrc_adaptive_spacetime :630-700 (AWI over neighbouring traces) */
#define OWL_MISFIT_DTW_VECTOR 8         /* compute_adjsrc_dtw on all components of a shot together (:1232-1236) */

/* form of the DTW misfit (dtw_form) */
#define OWL_DTW_PHASE 0     /* misfit sum q tau^2, adjoint q tau d/dt(warped obs) / dt */
#define OWL_DTW_AMP 1       /* misfit and adjoint of syn - warped obs */
#define OWL_DTW_PHASE_AMP 2 /* both, the amplitude term weighted by dtw_amp_weight */

/* penalty of the adaptive misfit (xcorr_penalty :321-363) */
#define OWL_PENALTY_LINEAR 0
#define OWL_PENALTY_POWER 1
#define OWL_PENALTY_GAUSSIAN 2
#define OWL_PENALTY_EXP 3

/* Misfit options: the reference's parameters of the same names
 * (src/lib/module_parameters.f90:550-570). Zero-initialised fields take
 * these defaults: tlag_max 0 -> 0.1 * (nt - 1) * dt, deconv_eps 0 -> 0.1,
 * penalty_power 0 -> 1, discard_threshold 0 -> 1e-6 (a negative value turns
 * the relative threshold off; traces of weight 0 or with a zero norm are
 * always dropped). DTW fields (:270-280, 559-569): dtw_niter 0 -> 5,
 * dtw_rinst 0 -> 0.1, dtw_rcuml 0 -> 1, dtw_epsabs 0 -> 1e-2, dtw_epsrel
 * 0 -> 1e-3 (a negative value of these four means 0), dtw_loss_power 0 -> 0.5
 * (the reference's 'l0.5'), dtw_amp_weight 0 -> 1, dtw_trc traces on each side
 * of a trace that enter its distance (0), dtw_form OWL_DTW_*. DTW takes the
 * traces at their own sampling; the shifts are not smoothed across traces.
 * lawi_sigma 0 -> 0.25 (s), adaptive_half_window 0 -> 3 (traces).
 * OWL_MISFIT_DTW_VECTOR: consecutive groups of ncomp gathers of equal length
 * are one shot's components; a receiver has one shift, one quality weight and
 * the norms over its kept components; its misfit is shared by its component
 * rows ('phase': equally; 'amp': each row its own; 'phase+amp': each row the
 * phase term and its own amplitude term). The gradient driver fills ncomp
 * (0) with the medium's component count. */
typedef struct {
    int misfit;              /* OWL_MISFIT_* */
    float dt;                /* sample interval of the traces (s) */
    float tlag_max;          /* adaptive: largest penalised lag; DTW: the candidate shifts are 2 tlag_max / dt + 1 (s) */
    int penalty;             /* OWL_PENALTY_* */
    float penalty_power;     /* exponent of the power / gaussian / exp penalties */
    float deconv_eps;        /* adaptive: water level, relative to max |D|^2 */
    float discard_threshold; /* trace_discard_threshold (relative to the gather's largest trace norm) */
    int dtw_form;            /* OWL_DTW_* */
    int dtw_niter;           /* refinements of the DTW search band */
    int dtw_trc;             /* neighbouring traces in the DTW distance */
    float dtw_rinst;         /* weight of the squared slope of the warping path */
    float dtw_rcuml;         /* weight of the squared shift */
    float dtw_epsabs;        /* absolute stop tolerance of the path cost */
    float dtw_epsrel;        /* relative stop tolerance of the path cost */
    float dtw_loss_power;    /* p of the distance sum |obs(t + tau) - syn(t)|^p */
    float dtw_amp_weight;    /* weight of the amplitude term of OWL_DTW_PHASE_AMP */
    float lawi_sigma;        /* local adaptive: standard deviation of the Gaussian time window (s) */
    int adaptive_half_window; /* space-time adaptive: neighbouring traces on each side */
    int ncomp;               /* dtw-vector: components (gathers) per shot */
    int adj_nt;              /* samples the traces are resampled to (cubic) before the misfit, the adjoint
                                resampled back (DTW: the shifts and quality weights are computed at adj_nt
                                samples and interpolated back, pchip); 0: owl_adjoint_source none, the
                                gradient driver the time axis' nt, as the reference */
} owl_misfit_opts;

typedef struct owl_ssg owl_ssg;

/* Solver descriptor: the scalar fields of wave_solver_* (interface.f90:32-40). */
typedef struct {
    int medium;          /* OWL_ACOUSTIC_ISO_2D, ... */
    int nx, ny, nz;      /* model cells; ny = 1 in 2D */
    float dx, dy, dz;    /* grid spacing (m) */
    float ox, oy, oz;    /* model origin (m) */
    int pml;             /* CFS-PML width in cells, outside the model */
    int fdhalf;          /* FD half-width: 4 (8th order) or 8 (16th order) */
    int free_surface;    /* 1: free surface on the top face */
    float dt;            /* time step (s) */
    int nt;              /* number of time steps */
    float f0_max;        /* max source f0 (Hz): PML alphamax = pi * f0_max */
    int max_shots;       /* capacity of one batched launch (>= 1) */
    int allow_dt_adjust; /* 0: dt above the CFL bound is OWL_ERR_UNSTABLE */
    int aniso;           /* OWL_ANISO_*: model parameterisation of elastic media */
    /* Depth-refined vertical mesh of the elastic solvers with a free surface
     * (free_surface_dz_refine and dz_max of wave_solver_elastic_vhtiort_2d / _3d,
     * elastic_vhtiort_2d/interface.f90:61-62; prepare_modeling,
     * module_vars.f90:313-376, 3D :424-490): rows dz / free_surface_dz_refine apart from the
     * surface down to (free_surface_refine_rows - 1) dz, then 2.5 % wider per
     * row up to dz_max. The model, the gradient and the geometry's x / z stay on
     * the regular (nz, nx) grid; owl_vertical_mesh gives the computational rows
     * that the geometry's gz / hz and taps refer to. All zero: the uniform grid. */
    float free_surface_dz_refine; /* >= 1; 0 = 1 */
    float dz_max;                 /* largest row spacing (m); 0 = dz */
    int free_surface_refine_rows; /* refine_nz (>= 1 when refined): owl_free_surface_refine_rows */
} owl_ssg_desc;

/* One source after prepare_geometry / prepare_stf. */
typedef struct {
    int mechanism;                  /* OWL_SRC_* */
    int gx, gy, gz;                 /* nearest integer node, 1-based */
    int hx, hy, hz;                 /* nearest half node, 1-based */
    float interp_ix[9], interp_iy[9], interp_iz[9];
    float interp_hx[9], interp_hy[9], interp_hz[9];
    float amp;                      /* amplitude */
    float polar, azimuth;           /* force direction, radians */
    float mt[6];                    /* moment tensor xx, yy, zz, xy, xz, yz */
    int nbeg;                       /* first step of injection (1-based) = nint(t0/dt)+1 */
    int nt_stf;                     /* samples in stf */
    const float *stf;               /* prepared source time function (host) */
} owl_source;

/* One receiver after prepare_geometry. weight == 0 disables the trace. */
typedef struct {
    int gx, gy, gz;
    int hx, hy, hz;
    float interp_ix[9], interp_iy[9], interp_iz[9];
    float interp_hx[9], interp_hy[9], interp_hz[9];
    float weight;
} owl_receiver;

/* One shot (one geometry file of OWL). */
typedef struct {
    int id;
    int nsrc;
    const owl_source *src;
    int nrec;
    const owl_receiver *rec;
} owl_shot;

/* Per-call execution options. Zero-initialised means defaults. */
typedef struct {
    int shots_per_launch;     /* shots per batched launch; 0 = the most up to max_shots whose buffers fit
                                 the free device memory; 1 = plain per-shot path */
    int checkpoint_interval;  /* k of every-k-step checkpoints; 0 = 50; < 0: the whole run when every
                                 buffer of the batch fits the free device memory with the stored stencil
                                 terms of every step, else the longest interval that fits. The forward
                                 stores the last segment's terms itself, so k >= nt recomputes nothing */
    int checkpoint_precision; /* OWL_CKPT_* */
    int use_graph;            /* 1: capture the time loop in CUDA graphs (default when 0 is -1) */
    int shots_per_cta;        /* shots handled per CTA; 0 = autotuned */
    int tile_x, tile_z;       /* CTA tile; 0 = autotuned */
    int check_every;          /* NaN/Inf check interval in steps; 0 = never */
} owl_run_opts;

/* Filled by forward / gradient. */
typedef struct {
    double elapsed_ms;        /* device time of the whole call (CUDA events) */
    double steps_cell_updates;/* padded cells x steps x shots x stencil passes */
    long long gpu_launches;   /* kernels launched by the library in the call */
    float dt_used;
    float dt_stable;
    int shots_per_cta;
    int tile_x, tile_z;
    int batches;
    int checkpoint_interval;  /* gradients: the interval used (opts, or chosen from free device memory) */
    int shots_per_launch;     /* shots per batched launch used (opts, or the most that fit the device) */
    int tile_z_forward;       /* the forward kernels' tile code (tile_z is the adjoint kernels' in a gradient) */
    int shots_per_cta_forward; /* the forward kernels' shots per CTA (shots_per_cta is the adjoint kernels' in a gradient) */
} owl_run_info;

/* ---- lifecycle ---------------------------------------------------------- */

/* Replaces prepare_modeling + compute_cfspml_damping_coef + alloc_*_wavefield
 * (src/solver/acoustic_iso_2d/module_vars.f90:90-208,
 *  src/solver/acoustic_iso_2d/module_cfspml.f90:61-133). */
int owl_ssg_create(const owl_ssg_desc *desc, owl_ssg **out);

/* Sets the model. Parameters (each a (nz[,ny],nx) z-fastest float32 host array):
 *   acoustic: vp, rho                                           (nparam = 2)
 *   elastic 2D, by desc.aniso (theta: tilt, radians):
 *     OWL_ANISO_ISO      vp, vs, rho                            (nparam = 3)
 *     OWL_ANISO_THOMSEN  vp, vs, epsilon, delta, theta, rho     (nparam = 6)
 *     OWL_ANISO_AT       vp, vs, epsilon, eta, theta, rho       (nparam = 6)
 *     OWL_ANISO_CIJ      c11, c13, c33, c55, rho                (nparam = 5)
 *   elastic 3D, by desc.aniso (theta, phi: tilt and azimuth, radians):
 *     OWL_ANISO_ISO      vp, vs, rho                            (nparam = 3)
 *     OWL_ANISO_THOMSEN  vp, vs, epsilon, delta, gamma, theta, phi, rho (nparam = 8)
 *     OWL_ANISO_CIJ      c11, c12, c13, c22, c23, c33, c44, c55, c66, rho (nparam = 10)
 * Replaces the transpose / pad_array / bk = rho*vp^2 part of prepare_modeling
 * (src/solver/acoustic_iso_2d/module_vars.f90:109-115) and, for elastic 2D, the
 * Cij set-up and M-PML coefficients (src/solver/elastic_vhtiort_2d/module_vars.f90:235-301,
 * src/lib/module_anisotropy.f90:310-402, src/solver/elastic_vhtiort_2d/module_cfspml.f90:229-577). */
int owl_ssg_set_model(owl_ssg *h, int nparam, const float *const *fields);

/* Seismogram sampling of the data: data_nt samples at data_dt (s) from t = 0
 * (the solver's data_dt / data_tmax, src/solver/acoustic_iso_2d/module_vars.f90:162-164;
 * data_nt = nint(data_tmax / data_dt + 1)). From this call on, forward and
 * misfit return, and gradient, gradient_misfit and source_gradient take, traces
 * of data_nt samples: the synthetics are resampled from the time axis (nt at
 * dt) as resample_su does after modelling (src/lib/module_su.f90:426-470,
 * submodule_forward_modeling.f90:124-125), the misfit and adjoint source are
 * computed at the data sampling, and the adjoint source is resampled back to
 * the time axis before injection (submodule_fwi_gradient.f90:46). The
 * resampling is cubic convolution (Keys, a = -1/2), zero outside the input
 * span. data_nt <= 0 returns to the time axis. */
int owl_ssg_set_data_sampling(owl_ssg *h, int data_nt, float data_dt);

/* Cubic-convolution resampling of ntr rows of nin samples at din from oin to
 * nout samples at dout from oout (resample_su's interp(..., 'cubic')), on the
 * GPU. in / out: host (OWL_MEM_HOST) or device (OWL_MEM_DEVICE) memory. */
int owl_resample_traces(int ntr, int nin, float din, float oin, const float *in, int nout, float dout, float oout,
                        float *out, int mem_kind);

/* SU files (the su type's output / load, src/lib/module_su.f90) assembled and
 * taken apart on the GPU. A record is the 240-byte trace header followed by
 * ns float32 samples in native byte order; the file is ntr records.
 * owl_su_encode: every record's header is the 240-byte host template `header`
 * (ns at byte 114, dt in microseconds at 116, d1 at 180), traces = ntr x ns
 * rows, out = ntr x (240 + 4 ns) bytes. owl_su_decode: the samples of every
 * record into traces. traces / out / in: host (OWL_MEM_HOST) or device
 * (OWL_MEM_DEVICE) memory; 1 <= ns <= 32767 (the header's int16 ns). */
int owl_su_encode(int ntr, int ns, const unsigned char *header, const float *traces, unsigned char *out,
                  int mem_kind);
int owl_su_decode(int ntr, int ns, const unsigned char *in, float *traces, int mem_kind);

/* ---- search directions and gradient processing ----------------------- */

/* search_method (src/inverse/module_inversion_search_direction.f90) */
#define OWL_SEARCH_SD 0    /* steepest descent: -g */
#define OWL_SEARCH_CG 1    /* Polak-Ribiere conjugate gradient (:38-86) */
#define OWL_SEARCH_LBFGS 2 /* two-loop L-BFGS (:91-246) */

/* Search direction of one parameter field of n floats. models / grads: nm
 * pointers each, oldest first, the last one the current iteration: the models
 * the gradients were computed at (the reference's updated_<name>.bin of
 * iterations k-nm+1 .. k, its <name>.bin at iteration 0) and those gradients.
 * L-BFGS uses the nm - 1 newest pairs (the reference keeps nstep_lbfgs = 10);
 * CG uses the last two gradients and prev_srch; nm = 1 (the first iteration)
 * gives -g for every method. Dot products are FP64 sums in a fixed order.
 * All arrays host (OWL_MEM_HOST) or device (OWL_MEM_DEVICE) memory. */
int owl_search_direction(int method, long long n, int nm, const float *const *models, const float *const *grads,
                         const float *prev_srch, float *srch, int mem_kind);

/* gradient processing operations (process_model_single_parameter,
 * src/inverse/2d/module_gradient.f90:733-892) on a field of n1 x n2 x n3
 * floats, n1 fastest (z, then x, then y as OWL's model files):
 *   OWL_GRAD_SMOOTH       Gaussian, param[0..2] = standard deviation in cells per axis (0: axis untouched)
 *   OWL_GRAD_TAPER        Blackman ramps, param[0..5] = ramp lengths in cells (axis 1 start, end, axis 2 ...)
 *   OWL_GRAD_MASK         multiply by mask (n1 x n2 x n3)
 *   OWL_GRAD_SCALE        multiply by param[0]
 *   OWL_GRAD_MAX_BALANCE  divide by the field's maximum when it is not 0
 *   OWL_GRAD_RMS_BALANCE  divide by the field's root-mean-square when it is not 0 (rms_balance)
 *   OWL_GRAD_RMS_BALANCE_AXIS  rms_balance_z / _x (/ _y): each slice j along axis param[0] (1, 2, 3)
 *                         divided by the L2 norm of the slices j - (w-1)/2 .. j + (w-1)/2, w =
 *                         param[1] cells rounded and made odd (zero slices beyond the ends); NaN / Inf -> 0
 *   OWL_GRAD_MEDIAN       median_filt: median of the window of half-widths param[0..2] cells per axis,
 *                         truncated at the ends (the mean of the two middle values of an even count);
 *                         the window holds at most 343 cells
 * param is host memory; field and mask host or device (mem_kind). */
#define OWL_GRAD_SMOOTH 0
#define OWL_GRAD_TAPER 1
#define OWL_GRAD_MASK 2
#define OWL_GRAD_SCALE 3
#define OWL_GRAD_MAX_BALANCE 4
#define OWL_GRAD_RMS_BALANCE 5
#define OWL_GRAD_RMS_BALANCE_AXIS 6
#define OWL_GRAD_MEDIAN 7
int owl_grad_process(int op, int n1, int n2, int n3, const float *param, const float *mask, float *field,
                     int mem_kind);

/* Forward modelling of nshots shots (batched by opts->shots_per_launch).
 * Replaces compute_forward (src/solver/acoustic_iso_2d/submodule_forward_modeling.f90:31-132).
 * seis: per shot, ncomp x nrec x nt float32 (trace-major, the SU trace order),
 * shots concatenated; ncomp = 1 (p) for acoustic, 2 (vx, vz) for elastic 2D,
 * 3 (vx, vy, vz) for elastic 3D. */
int owl_ssg_forward(owl_ssg *h, int nshots, const owl_shot *shots,
                    const owl_run_opts *opts, float *seis, int mem_kind,
                    owl_run_info *info);

/* Adjoint-state gradient. Replaces the per-shot pipeline of compute_gradient_shots
 * (src/inverse/2d/module_gradient.f90:114-135,323-358): forward, adjoint source
 * (compute_adjsrc_waveform, src/inverse/module_inversion_adjoint_source.f90:371-383),
 * adjoint propagation and imaging (src/solver/acoustic_iso_2d/submodule_fwi_gradient.f90:31-269),
 * stacked over the shots. The adjoint is the exact discrete transpose of the
 * forward with every-k-step checkpoints and segment recomputation.
 *   data: OWL_ADJ_L2_RESIDUAL -> observed seismograms; OWL_ADJ_GIVEN -> adjoint source;
 *         same layout as seis in owl_ssg_forward.
 *   misfit: nshots doubles (may be NULL), sum over traces of (obs - syn)^2.
 *   grad: nparam x (nz[,ny],nx) float32, z fastest, of J = 0.5 * misfit
 *         (the reference's adjoint source syn - obs), w.r.t. the model parameters
 *         in the order of owl_ssg_set_model.
 *   seis_out: optional synthetic seismograms (may be NULL). */
int owl_ssg_gradient(owl_ssg *h, int nshots, const owl_shot *shots,
                     const float *data, int adj_kind, const owl_run_opts *opts,
                     double *misfit, float *grad, float *seis_out, int mem_kind,
                     owl_run_info *info);

/* Gradient of the same J w.r.t. each source's STF samples (the adjoint of
 * add_source, src/solver/acoustic_iso_2d/module_wavefield.f90:192-263):
 * stf_grad holds, per shot and source, nt floats (step index 1..nt). Used for
 * source estimation and for the source-side dot-product test. */
int owl_ssg_source_gradient(owl_ssg *h, int nshots, const owl_shot *shots,
                            const float *adj, const owl_run_opts *opts,
                            float *stf_grad, int mem_kind, owl_run_info *info);

/* Misfit-only batched forward: the trial forwards of the step-length search
 * (compute_step_misfit / compute_step_coef, src/inverse/module_inversion_step_size.f90:263-592)
 * with the waveform misfit (compute_adjsrc_waveform,
 * src/inverse/module_inversion_adjoint_source.f90:371-383). No checkpoints.
 *   obs: observed (or reference) seismograms, the layout of owl_ssg_forward.
 *   misfit: nshots doubles, sum over traces of (obs - syn)^2 (may be NULL).
 *   trace_misfit: one double per trace, in seismogram trace order (may be NULL).
 *   seis_out: the synthetic seismograms (may be NULL). */
int owl_ssg_misfit(owl_ssg *h, int nshots, const owl_shot *shots, const float *obs,
                   const owl_run_opts *opts, double *misfit, double *trace_misfit,
                   float *seis_out, int mem_kind, owl_run_info *info);

/* owl_ssg_gradient with a data-domain misfit other than (or as well as) L2:
 * after the forward, the adjoint source and the per-trace misfits of every
 * gather are computed on the GPU exactly as owl_adjoint_source does (trace
 * discard rule included), and the gradient is that of 0.5 * the misfit.
 *   obs: observed seismograms, layout of owl_ssg_forward.
 *   misfit: nshots doubles (may be NULL), the sum of the shot's trace misfits. */
int owl_ssg_gradient_misfit(owl_ssg *h, int nshots, const owl_shot *shots, const float *obs,
                            const owl_misfit_opts *mopts, const owl_run_opts *opts, double *misfit,
                            float *grad, float *seis_out, int mem_kind, owl_run_info *info);

void owl_ssg_destroy(owl_ssg *h);

/* ---- adjoint sources (compute_adjoint_source,
 *      src/inverse/module_inversion_adjoint_source.f90:985-1277) ------------ */

/* Misfit and adjoint source of every trace of ngather gathers (one shot's one
 * component each), on the GPU. Traces are rows of nt samples, gathers are
 * contiguous: gather g holds traces gather_ptr[g] .. gather_ptr[g + 1] - 1 of
 * syn / obs / adj (host array of ngather + 1 ints, gather_ptr[0] = 0). A trace
 * is dropped (misfit 0, adjoint 0) when its weight is 0 or when its obs or syn
 * norm is below discard_threshold times the gather's largest obs or syn norm or
 * is 0 (:1047-1050). weight: one float per trace or NULL (all 1).
 *   adj: adjoint source, the layout of syn (may be NULL).
 *   trace_misfit: one double per trace (may be NULL).
 *   gather_misfit: one double per gather (may be NULL).
 * syn, obs, adj, weight, trace_misfit and gather_misfit are all host memory
 * (OWL_MEM_HOST) or all device memory of the current device (OWL_MEM_DEVICE).
 * Trace length: nt <= 8192 (envelope, phase), next_power_235(2 nt) <= 8192
 * (adaptive, local adaptive), next_power_235(4 nt) <= 8192 (space-time
 * adaptive), 3 <= nt <= 16384 with 3 <= 2 tlag_max / dt + 1 <= 4095 (DTW),
 * else OWL_ERR_INVALID. */
int owl_adjoint_source(const owl_misfit_opts *mopts, int ngather, const int *gather_ptr, int nt,
                       const float *syn, const float *obs, const float *weight, float *adj,
                       double *trace_misfit, double *gather_misfit, int mem_kind);

/* Time shifts tau(t) of the DTW misfit, obs(t + tau) ~ syn(t), in seconds, one
 * row per trace like syn (zero on dropped traces; dtw-vector: the receiver's
 * shift on each of its component rows): the reference's
 * shot_<id>_time_shift_<comp>.su output (compute_adjoint_source :1238-1246).
 * Same arguments and limits as owl_adjoint_source with mopts->misfit =
 * OWL_MISFIT_DTW or OWL_MISFIT_DTW_VECTOR. DTW limits: 3 <= nt <= 16384 and 3 <= 2 tlag_max / dt + 1
 * <= 4095. */
int owl_dtw_time_shifts(const owl_misfit_opts *mopts, int ngather, const int *gather_ptr, int nt,
                        const float *syn, const float *obs, const float *weight, float *tau, int mem_kind);

/* ---- diagnostics (no counterpart in the reference) ------------------------ */

/* Kernel ids for owl_ssg_kernel_time. */
#define OWL_K_FWD_P 0   /* pressure / stress update with fused CFS-PML */
#define OWL_K_FWD_V 1   /* velocity update with fused CFS-PML */
#define OWL_K_ADJ_P 2   /* adjoint of the velocity update (writes p^) */
#define OWL_K_ADJ_V 3   /* adjoint of the pressure update (writes v^) */
#define OWL_K_FWD_P_STORE 4 /* OWL_K_FWD_P also writing the step's stencil terms (recomputed and last
                               forward segments of a gradient) */
#define OWL_K_FWD_V_STORE 5 /* OWL_K_FWD_V also writing the step's stencil terms */

/* Times nlaunch back-to-back standalone launches of one kernel on the state of
 * the last batch of the last forward / gradient call (CUDA events on the
 * handle's stream). avg_ms: mean duration of one launch. alg_bytes: compulsory
 * HBM bytes of one launch (each state field read / written once per shot,
 * materials once per launch, PML memory only inside the PML, the stored
 * stencil terms of the _STORE variants once). The _STORE variants and the
 * adjoint kernels need a gradient call first. Leaves the wavefields in an
 * unspecified state. */
int owl_ssg_kernel_time(owl_ssg *h, int kernel_id, int nlaunch, double *avg_ms, double *alg_bytes);

/* ---- forward without device allocation (no counterpart in the reference) -- */

/* Size, in floats, of the one device array that owl_ssg_forward_noalloc works
 * in (64 MiB). Every GPU that loads the library holds this array until the
 * process exits. */
#define OWL_NOALLOC_MAX_FLOATS (16 * 1024 * 1024)

/* One 2D acoustic shot (explosion sources, no free surface) modelled without
 * any device allocation (no counterpart in the reference), for callers that
 * cannot call cudaMalloc where they model a shot: applications whose device
 * memory is owned by another allocator or reserved up front as a fixed budget,
 * where one more cudaMalloc fails or breaks the budget. Materials, PML
 * coefficients, wavefields and traces live in a static device array of
 * OWL_NOALLOC_MAX_FLOATS floats. Inputs and outputs are host memory: vp, rho as
 * for owl_ssg_set_model (nparam = 2), seis = nrec x nt floats in the layout of
 * owl_ssg_forward. The same seismograms as owl_ssg_forward. Returns
 * OWL_ERR_INVALID when the run needs more than OWL_NOALLOC_MAX_FLOATS floats.
 * The first call on a device looks up the array's device address and keeps it
 * for the process; make that first call before any stream capture starts. A
 * call after cudaDeviceReset on that device is not supported. All calls share
 * the array, which keeps the last call's contents (each call clears what must
 * start at zero); calls whose GPU work overlapped would race on it, so the
 * call holds a process-wide lock and returns only after its GPU work has
 * finished. */
int owl_ssg_forward_noalloc(const owl_ssg_desc *desc, int nparam, const float *const *fields,
                            const owl_shot *shot, float *seis);

/* ---- M-PML damping ratios of the 3D anisotropic elastic solver ---------- */

/* damp_ratio (src/solver/elastic_vhtiort_3d/module_cfspml.f90:193-248): the
 * M-PML ratio of one PML face cell, c = (c11, c12, c13, c22, c23, c33, c44,
 * c55, c66) of the cell, axis 0 / 1 / 2 the damped axis (x, y, z faces).
 * Host computation, no device needed; -1 on bad arguments. */
float owl_mpml_damp_ratio(const float *c, int axis);

/* The six face-ratio arrays an elastic 3D handle uses after set_model
 * (compute_damping_profile_ratio, module_cfspml.f90:253-421; all zero for the
 * iso parameterisation, as the reference's): faces = left, right (x low /
 * high: (nz + 2 pml) x (ny + 2 pml), y fastest), front, back (y: (nz + 2 pml) x
 * (nx + 2 pml), x fastest), top, bottom (z: (ny + 2 pml) x (nx + 2 pml), x
 * fastest), concatenated; index 0 of each axis is the reference's -pml + 1.
 * With a free surface the x / y faces hold zeros above row 1. On the
 * depth-refined free-surface mesh nz is the mesh's planes (owl_vertical_mesh). */
int owl_ssg_mpml_ratios(const owl_ssg *h, float *faces);

/* ---- queries ------------------------------------------------------------ */

/* Vertical mesh of a descriptor (host only, no device needed): the
 * computational rows of the elastic solvers with a free surface
 * (module_vars.f90:313-376). nz_mesh gets the number of rows (desc->nz for the
 * uniform grid); each non-null array gets nz_mesh + 2 pml + 2 values, rows
 * -pml .. nz_mesh + pml + 1 of the reference's zz_i, zz_h, dz_i, dz_h (depths
 * below the model origin, m). Geometry on this mesh (module_source_receiver.f90:
 * 596-616, 640-680): gz = the row of z_i nearest to z - oz (the first on a tie),
 * hz likewise on z_h (z = 0 counts as just below the surface), taps
 * kaiser_sinc((z - oz - z_i(gz)) / dz_i(gz)), the same with z_h, dz_h; with a
 * free surface, sources above dz_i(1) move to dz_i(1) with 1.2 x amplitude
 * (module_vars.f90:463-466). Call once with null arrays to size them. */
int owl_vertical_mesh(const owl_ssg_desc *desc, int *nz_mesh, float *z_i, float *z_h, float *dz_i, float *dz_h);
/* refine_nz of the refined mesh (module_vars.f90:315-317): ceil(0.5 lambda / dz)
 * with lambda = sqrt(mean over the padded surface row of c55 / rho) / f0_min,
 * c55 and rho of the model in desc->aniso's parameterisation (elastic 2D;
 * elastic 3D: the largest of the means of c44 / rho, c55 / rho, c66 / rho over
 * the padded surface plane, elastic_vhtiort_3d/module_vars.f90:424-428),
 * f0_min the lowest peak frequency of the sources. Host only. */
int owl_free_surface_refine_rows(const owl_ssg_desc *desc, int nparam, const float *const *fields, float f0_min,
                                 int *refine_rows);

const char *owl_last_error(void);
int owl_ssg_abi_version(void);
/* dt_stable of the current model (module_vars.f90:121-125); 0 before set_model. */
float owl_ssg_dt_stable(const owl_ssg *h);
/* number of parameters and seismogram components of a medium (elastic 2D:
 * the OWL_ANISO_ISO parameterisation) */
int owl_ssg_nparam(int medium);
/* number of model parameters of a descriptor (medium and parameterisation) */
int owl_ssg_desc_nparam(const owl_ssg_desc *desc);
int owl_ssg_ncomp(int medium);
/* 1 if the CUDA kernels for sm_100a are present and a device is usable */
int owl_ssg_device_ok(void);

#ifdef __cplusplus
}
#endif

#endif /* OWL_SSG_H */
