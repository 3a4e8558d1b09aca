!
! owl_ssg.f90 -- Fortran 2008 ISO_C_BINDING interface to the C ABI of
! include/owl_ssg.h, for OWL's own host code.
!
! A maintainer keeps OWL's solver types (e.g. wave_solver_acoustic_iso_2d,
! src/solver/acoustic_iso_2d/interface.f90:30-60) and drivers, and replaces the
! forward / adjoint submodules (submodule_forward_modeling.f90,
! submodule_fwi_gradient.f90) with ones that fill these structures from the
! solver's fields and from prepare_geometry / prepare_stf, and call the
! functions below. Every type mirrors the C struct of the same name field by
! field, in order; every constant is the C macro of the same name.
!
! Buffers that may live in host or device memory (model fields, seismograms,
! gradients, misfits) are passed as type(c_ptr), value: pass c_loc(array) for
! a host array or the device address for a device buffer, with mem_kind set
! to match. Optional pointers are c_null_ptr when absent.
!
module owl_ssg_c
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: OWL_SSG_ABI_VERSION = 10

    ! status codes
    integer(c_int), parameter :: OWL_OK = 0
    integer(c_int), parameter :: OWL_ERR_INVALID = -1
    integer(c_int), parameter :: OWL_ERR_CUDA = -2
    integer(c_int), parameter :: OWL_ERR_OOM = -3
    integer(c_int), parameter :: OWL_ERR_NONFINITE = -4
    integer(c_int), parameter :: OWL_ERR_UNSTABLE = -5
    integer(c_int), parameter :: OWL_ERR_TIMEOUT = -6
    integer(c_int), parameter :: OWL_ERR_UNSUPPORTED = -7
    integer(c_int), parameter :: OWL_ERR_NO_DEVICE = -8

    ! media (which_medium, src/lib/module_parameters.f90:397)
    integer(c_int), parameter :: OWL_ACOUSTIC_ISO_2D = 1
    integer(c_int), parameter :: OWL_ACOUSTIC_ISO_3D = 2
    integer(c_int), parameter :: OWL_ELASTIC_VHTIORT_2D = 3
    integer(c_int), parameter :: OWL_ELASTIC_VHTIORT_3D = 4

    ! elastic parameterisations (anisotropy_type)
    integer(c_int), parameter :: OWL_ANISO_ISO = 0
    integer(c_int), parameter :: OWL_ANISO_THOMSEN = 1
    integer(c_int), parameter :: OWL_ANISO_AT = 2
    integer(c_int), parameter :: OWL_ANISO_CIJ = 3

    ! source mechanisms
    integer(c_int), parameter :: OWL_SRC_EXPLOSION = 0
    integer(c_int), parameter :: OWL_SRC_FORCE = 1
    integer(c_int), parameter :: OWL_SRC_MT = 2

    ! memory kinds
    integer(c_int), parameter :: OWL_MEM_HOST = 0
    integer(c_int), parameter :: OWL_MEM_DEVICE = 1

    ! checkpoint precision
    integer(c_int), parameter :: OWL_CKPT_FP32 = 0
    integer(c_int), parameter :: OWL_CKPT_FP16 = 1
    integer(c_int), parameter :: OWL_CKPT_BF16 = 2

    ! adjoint-source kinds
    integer(c_int), parameter :: OWL_ADJ_L2_RESIDUAL = 0
    integer(c_int), parameter :: OWL_ADJ_GIVEN = 1

    ! misfit_type
    integer(c_int), parameter :: OWL_MISFIT_WAVEFORM = 0
    integer(c_int), parameter :: OWL_MISFIT_CORR = 1
    integer(c_int), parameter :: OWL_MISFIT_ENVELOPE = 2
    integer(c_int), parameter :: OWL_MISFIT_PHASE = 3
    integer(c_int), parameter :: OWL_MISFIT_ADAPTIVE = 4
    integer(c_int), parameter :: OWL_MISFIT_DTW = 5
    integer(c_int), parameter :: OWL_MISFIT_LOCAL_ADAPTIVE = 6
    integer(c_int), parameter :: OWL_MISFIT_ADAPTIVE_SPACETIME = 7
    integer(c_int), parameter :: OWL_MISFIT_DTW_VECTOR = 8

    ! dtw_form
    integer(c_int), parameter :: OWL_DTW_PHASE = 0
    integer(c_int), parameter :: OWL_DTW_AMP = 1
    integer(c_int), parameter :: OWL_DTW_PHASE_AMP = 2

    ! penalty_method of the adaptive misfit
    integer(c_int), parameter :: OWL_PENALTY_LINEAR = 0
    integer(c_int), parameter :: OWL_PENALTY_POWER = 1
    integer(c_int), parameter :: OWL_PENALTY_GAUSSIAN = 2
    integer(c_int), parameter :: OWL_PENALTY_EXP = 3

    ! search_method
    integer(c_int), parameter :: OWL_SEARCH_SD = 0
    integer(c_int), parameter :: OWL_SEARCH_CG = 1
    integer(c_int), parameter :: OWL_SEARCH_LBFGS = 2

    ! gradient processing operations
    integer(c_int), parameter :: OWL_GRAD_SMOOTH = 0
    integer(c_int), parameter :: OWL_GRAD_TAPER = 1
    integer(c_int), parameter :: OWL_GRAD_MASK = 2
    integer(c_int), parameter :: OWL_GRAD_SCALE = 3
    integer(c_int), parameter :: OWL_GRAD_MAX_BALANCE = 4
    integer(c_int), parameter :: OWL_GRAD_RMS_BALANCE = 5
    integer(c_int), parameter :: OWL_GRAD_RMS_BALANCE_AXIS = 6
    integer(c_int), parameter :: OWL_GRAD_MEDIAN = 7

    ! kernel ids of owl_ssg_kernel_time
    integer(c_int), parameter :: OWL_K_FWD_P = 0
    integer(c_int), parameter :: OWL_K_FWD_V = 1
    integer(c_int), parameter :: OWL_K_ADJ_P = 2
    integer(c_int), parameter :: OWL_K_ADJ_V = 3
    integer(c_int), parameter :: OWL_K_FWD_P_STORE = 4
    integer(c_int), parameter :: OWL_K_FWD_V_STORE = 5

    ! size of the no-alloc forward's static device array, in floats
    integer(c_int), parameter :: OWL_NOALLOC_MAX_FLOATS = 16*1024*1024

    ! misfit options (module_parameters.f90:550-570)
    type, bind(c) :: owl_misfit_opts
        integer(c_int) :: misfit
        real(c_float) :: dt
        real(c_float) :: tlag_max
        integer(c_int) :: penalty
        real(c_float) :: penalty_power
        real(c_float) :: deconv_eps
        real(c_float) :: discard_threshold
        integer(c_int) :: dtw_form
        integer(c_int) :: dtw_niter
        integer(c_int) :: dtw_trc
        real(c_float) :: dtw_rinst
        real(c_float) :: dtw_rcuml
        real(c_float) :: dtw_epsabs
        real(c_float) :: dtw_epsrel
        real(c_float) :: dtw_loss_power
        real(c_float) :: dtw_amp_weight
        real(c_float) :: lawi_sigma
        integer(c_int) :: adaptive_half_window
        integer(c_int) :: ncomp
        integer(c_int) :: adj_nt
    end type

    ! solver descriptor: the scalar fields of wave_solver_* (interface.f90:32-40)
    type, bind(c) :: owl_ssg_desc
        integer(c_int) :: medium
        integer(c_int) :: nx
        integer(c_int) :: ny
        integer(c_int) :: nz
        real(c_float) :: dx
        real(c_float) :: dy
        real(c_float) :: dz
        real(c_float) :: ox
        real(c_float) :: oy
        real(c_float) :: oz
        integer(c_int) :: pml
        integer(c_int) :: fdhalf
        integer(c_int) :: free_surface
        real(c_float) :: dt
        integer(c_int) :: nt
        real(c_float) :: f0_max
        integer(c_int) :: max_shots
        integer(c_int) :: allow_dt_adjust
        integer(c_int) :: aniso
        real(c_float) :: free_surface_dz_refine
        real(c_float) :: dz_max
        integer(c_int) :: free_surface_refine_rows
    end type

    ! one source after prepare_geometry / prepare_stf
    type, bind(c) :: owl_source
        integer(c_int) :: mechanism
        integer(c_int) :: gx
        integer(c_int) :: gy
        integer(c_int) :: gz
        integer(c_int) :: hx
        integer(c_int) :: hy
        integer(c_int) :: hz
        real(c_float) :: interp_ix(9)
        real(c_float) :: interp_iy(9)
        real(c_float) :: interp_iz(9)
        real(c_float) :: interp_hx(9)
        real(c_float) :: interp_hy(9)
        real(c_float) :: interp_hz(9)
        real(c_float) :: amp
        real(c_float) :: polar
        real(c_float) :: azimuth
        real(c_float) :: mt(6)
        integer(c_int) :: nbeg
        integer(c_int) :: nt_stf
        type(c_ptr) :: stf
    end type

    ! one receiver after prepare_geometry (weight 0 disables the trace)
    type, bind(c) :: owl_receiver
        integer(c_int) :: gx
        integer(c_int) :: gy
        integer(c_int) :: gz
        integer(c_int) :: hx
        integer(c_int) :: hy
        integer(c_int) :: hz
        real(c_float) :: interp_ix(9)
        real(c_float) :: interp_iy(9)
        real(c_float) :: interp_iz(9)
        real(c_float) :: interp_hx(9)
        real(c_float) :: interp_hy(9)
        real(c_float) :: interp_hz(9)
        real(c_float) :: weight
    end type

    ! one shot: src -> nsrc owl_source, rec -> nrec owl_receiver
    type, bind(c) :: owl_shot
        integer(c_int) :: id
        integer(c_int) :: nsrc
        type(c_ptr) :: src
        integer(c_int) :: nrec
        type(c_ptr) :: rec
    end type

    ! per-call execution options (zero means the default)
    type, bind(c) :: owl_run_opts
        integer(c_int) :: shots_per_launch
        integer(c_int) :: checkpoint_interval
        integer(c_int) :: checkpoint_precision
        integer(c_int) :: use_graph
        integer(c_int) :: shots_per_cta
        integer(c_int) :: tile_x
        integer(c_int) :: tile_z
        integer(c_int) :: check_every
    end type

    ! filled by forward / gradient
    type, bind(c) :: owl_run_info
        real(c_double) :: elapsed_ms
        real(c_double) :: steps_cell_updates
        integer(c_long_long) :: gpu_launches
        real(c_float) :: dt_used
        real(c_float) :: dt_stable
        integer(c_int) :: shots_per_cta
        integer(c_int) :: tile_x
        integer(c_int) :: tile_z
        integer(c_int) :: batches
        integer(c_int) :: checkpoint_interval
        integer(c_int) :: shots_per_launch
        integer(c_int) :: tile_z_forward
        integer(c_int) :: shots_per_cta_forward
    end type

    interface

        ! replaces prepare_modeling + compute_cfspml_damping_coef + alloc_*_wavefield
        integer(c_int) function owl_ssg_create(desc, out) bind(c, name='owl_ssg_create')
            import :: c_int, c_ptr, owl_ssg_desc
            type(owl_ssg_desc), intent(in) :: desc
            type(c_ptr), intent(out) :: out
        end function

        ! fields: nparam pointers to (nz[,ny],nx) z-fastest float32 host arrays
        integer(c_int) function owl_ssg_set_model(h, nparam, fields) bind(c, name='owl_ssg_set_model')
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: nparam
            type(c_ptr), intent(in) :: fields(*)
        end function

        integer(c_int) function owl_ssg_set_data_sampling(h, data_nt, data_dt) bind(c, name='owl_ssg_set_data_sampling')
            import :: c_int, c_ptr, c_float
            type(c_ptr), value :: h
            integer(c_int), value :: data_nt
            real(c_float), value :: data_dt
        end function

        integer(c_int) function owl_resample_traces(ntr, nin, din, oin, in, nout, dout, oout, out, mem_kind) &
                bind(c, name='owl_resample_traces')
            import :: c_int, c_ptr, c_float
            integer(c_int), value :: ntr, nin
            real(c_float), value :: din, oin
            type(c_ptr), value :: in
            integer(c_int), value :: nout
            real(c_float), value :: dout, oout
            type(c_ptr), value :: out
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_su_encode(ntr, ns, header, traces, out, mem_kind) bind(c, name='owl_su_encode')
            import :: c_int, c_ptr
            integer(c_int), value :: ntr, ns
            type(c_ptr), value :: header, traces, out
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_su_decode(ntr, ns, in, traces, mem_kind) bind(c, name='owl_su_decode')
            import :: c_int, c_ptr
            integer(c_int), value :: ntr, ns
            type(c_ptr), value :: in, traces
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_search_direction(method, n, nm, models, grads, prev_srch, srch, mem_kind) &
                bind(c, name='owl_search_direction')
            import :: c_int, c_ptr, c_long_long
            integer(c_int), value :: method
            integer(c_long_long), value :: n
            integer(c_int), value :: nm
            type(c_ptr), intent(in) :: models(*), grads(*)
            type(c_ptr), value :: prev_srch, srch
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_grad_process(op, n1, n2, n3, param, mask, field, mem_kind) &
                bind(c, name='owl_grad_process')
            import :: c_int, c_ptr
            integer(c_int), value :: op, n1, n2, n3
            type(c_ptr), value :: param, mask, field
            integer(c_int), value :: mem_kind
        end function

        ! replaces compute_forward (submodule_forward_modeling.f90:31-132)
        integer(c_int) function owl_ssg_forward(h, nshots, shots, opts, seis, mem_kind, info) &
                bind(c, name='owl_ssg_forward')
            import :: c_int, c_ptr, owl_shot, owl_run_opts, owl_run_info
            type(c_ptr), value :: h
            integer(c_int), value :: nshots
            type(owl_shot), intent(in) :: shots(*)
            type(owl_run_opts), intent(in) :: opts
            type(c_ptr), value :: seis
            integer(c_int), value :: mem_kind
            type(owl_run_info), intent(out) :: info
        end function

        ! replaces forward + compute_adjsrc_waveform + compute_adjoint per shot, stacked
        integer(c_int) function owl_ssg_gradient(h, nshots, shots, data, adj_kind, opts, misfit, grad, seis_out, &
                mem_kind, info) bind(c, name='owl_ssg_gradient')
            import :: c_int, c_ptr, owl_shot, owl_run_opts, owl_run_info
            type(c_ptr), value :: h
            integer(c_int), value :: nshots
            type(owl_shot), intent(in) :: shots(*)
            type(c_ptr), value :: data
            integer(c_int), value :: adj_kind
            type(owl_run_opts), intent(in) :: opts
            type(c_ptr), value :: misfit, grad, seis_out
            integer(c_int), value :: mem_kind
            type(owl_run_info), intent(out) :: info
        end function

        integer(c_int) function owl_ssg_source_gradient(h, nshots, shots, adj, opts, stf_grad, mem_kind, info) &
                bind(c, name='owl_ssg_source_gradient')
            import :: c_int, c_ptr, owl_shot, owl_run_opts, owl_run_info
            type(c_ptr), value :: h
            integer(c_int), value :: nshots
            type(owl_shot), intent(in) :: shots(*)
            type(c_ptr), value :: adj
            type(owl_run_opts), intent(in) :: opts
            type(c_ptr), value :: stf_grad
            integer(c_int), value :: mem_kind
            type(owl_run_info), intent(out) :: info
        end function

        ! the trial forwards of the step-length search (module_inversion_step_size.f90:263-592)
        integer(c_int) function owl_ssg_misfit(h, nshots, shots, obs, opts, misfit, trace_misfit, seis_out, &
                mem_kind, info) bind(c, name='owl_ssg_misfit')
            import :: c_int, c_ptr, owl_shot, owl_run_opts, owl_run_info
            type(c_ptr), value :: h
            integer(c_int), value :: nshots
            type(owl_shot), intent(in) :: shots(*)
            type(c_ptr), value :: obs
            type(owl_run_opts), intent(in) :: opts
            type(c_ptr), value :: misfit, trace_misfit, seis_out
            integer(c_int), value :: mem_kind
            type(owl_run_info), intent(out) :: info
        end function

        integer(c_int) function owl_ssg_gradient_misfit(h, nshots, shots, obs, mopts, opts, misfit, grad, seis_out, &
                mem_kind, info) bind(c, name='owl_ssg_gradient_misfit')
            import :: c_int, c_ptr, owl_shot, owl_misfit_opts, owl_run_opts, owl_run_info
            type(c_ptr), value :: h
            integer(c_int), value :: nshots
            type(owl_shot), intent(in) :: shots(*)
            type(c_ptr), value :: obs
            type(owl_misfit_opts), intent(in) :: mopts
            type(owl_run_opts), intent(in) :: opts
            type(c_ptr), value :: misfit, grad, seis_out
            integer(c_int), value :: mem_kind
            type(owl_run_info), intent(out) :: info
        end function

        subroutine owl_ssg_destroy(h) bind(c, name='owl_ssg_destroy')
            import :: c_ptr
            type(c_ptr), value :: h
        end subroutine

        ! compute_adjoint_source (module_inversion_adjoint_source.f90:985-1277)
        integer(c_int) function owl_adjoint_source(mopts, ngather, gather_ptr, nt, syn, obs, weight, adj, &
                trace_misfit, gather_misfit, mem_kind) bind(c, name='owl_adjoint_source')
            import :: c_int, c_ptr, owl_misfit_opts
            type(owl_misfit_opts), intent(in) :: mopts
            integer(c_int), value :: ngather
            integer(c_int), intent(in) :: gather_ptr(*)
            integer(c_int), value :: nt
            type(c_ptr), value :: syn, obs, weight, adj, trace_misfit, gather_misfit
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_dtw_time_shifts(mopts, ngather, gather_ptr, nt, syn, obs, weight, tau, mem_kind) &
                bind(c, name='owl_dtw_time_shifts')
            import :: c_int, c_ptr, owl_misfit_opts
            type(owl_misfit_opts), intent(in) :: mopts
            integer(c_int), value :: ngather
            integer(c_int), intent(in) :: gather_ptr(*)
            integer(c_int), value :: nt
            type(c_ptr), value :: syn, obs, weight, tau
            integer(c_int), value :: mem_kind
        end function

        integer(c_int) function owl_ssg_kernel_time(h, kernel_id, nlaunch, avg_ms, alg_bytes) &
                bind(c, name='owl_ssg_kernel_time')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: kernel_id, nlaunch
            real(c_double), intent(out) :: avg_ms, alg_bytes
        end function

        ! one 2D acoustic shot without device allocation (no counterpart in the reference)
        integer(c_int) function owl_ssg_forward_noalloc(desc, nparam, fields, shot, seis) &
                bind(c, name='owl_ssg_forward_noalloc')
            import :: c_int, c_ptr, owl_ssg_desc, owl_shot
            type(owl_ssg_desc), intent(in) :: desc
            integer(c_int), value :: nparam
            type(c_ptr), intent(in) :: fields(*)
            type(owl_shot), intent(in) :: shot
            type(c_ptr), value :: seis
        end function

        ! damp_ratio (module_cfspml.f90:193-248) of one face cell, host computation
        real(c_float) function owl_mpml_damp_ratio(c, axis) bind(c, name='owl_mpml_damp_ratio')
            import :: c_float, c_int
            real(c_float), intent(in) :: c(*)
            integer(c_int), value :: axis
        end function

        ! the six M-PML face-ratio arrays of an elastic 3D handle
        integer(c_int) function owl_ssg_mpml_ratios(h, faces) bind(c, name='owl_ssg_mpml_ratios')
            import :: c_int, c_ptr
            type(c_ptr), value :: h, faces
        end function

        ! returns a NUL-terminated C string (c_f_pointer it to a character array)
        type(c_ptr) function owl_last_error() bind(c, name='owl_last_error')
            import :: c_ptr
        end function

        integer(c_int) function owl_ssg_abi_version() bind(c, name='owl_ssg_abi_version')
            import :: c_int
        end function

        real(c_float) function owl_ssg_dt_stable(h) bind(c, name='owl_ssg_dt_stable')
            import :: c_float, c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function owl_ssg_nparam(medium) bind(c, name='owl_ssg_nparam')
            import :: c_int
            integer(c_int), value :: medium
        end function

        integer(c_int) function owl_ssg_desc_nparam(desc) bind(c, name='owl_ssg_desc_nparam')
            import :: c_int, owl_ssg_desc
            type(owl_ssg_desc), intent(in) :: desc
        end function

        ! computational rows of the depth-refined free-surface mesh (host only);
        ! null arrays (c_null_ptr) size them: nz_mesh + 2 pml + 2 values each
        integer(c_int) function owl_vertical_mesh(desc, nz_mesh, z_i, z_h, dz_i, dz_h) &
                bind(c, name='owl_vertical_mesh')
            import :: c_int, c_ptr, owl_ssg_desc
            type(owl_ssg_desc), intent(in) :: desc
            integer(c_int), intent(out) :: nz_mesh
            type(c_ptr), value :: z_i, z_h, dz_i, dz_h
        end function

        ! refine_nz from the model's surface row and the lowest source f0 (host only)
        integer(c_int) function owl_free_surface_refine_rows(desc, nparam, fields, f0_min, refine_rows) &
                bind(c, name='owl_free_surface_refine_rows')
            import :: c_int, c_ptr, c_float, owl_ssg_desc
            type(owl_ssg_desc), intent(in) :: desc
            integer(c_int), value :: nparam
            type(c_ptr), intent(in) :: fields(*)
            real(c_float), value :: f0_min
            integer(c_int), intent(out) :: refine_rows
        end function

        integer(c_int) function owl_ssg_ncomp(medium) bind(c, name='owl_ssg_ncomp')
            import :: c_int
            integer(c_int), value :: medium
        end function

        integer(c_int) function owl_ssg_device_ok() bind(c, name='owl_ssg_device_ok')
            import :: c_int
        end function

    end interface

end module owl_ssg_c
