!> m_calypso_b200.f90 -- Fortran 2003 interfaces (iso_c_binding) to the C
!! ABI of libcalypso_b200 declared in calypso_b200.h.
!!
!! A Fortran host of the time step (the reference's own language) uses this
!! module in place of the module procedures the library replaces; the
!! comments of calypso_b200.h give the reference routine of every entry
!! point and the layouts of its arrays.  Conventions of these interfaces:
!!   * contexts, ensembles and networks are type(c_ptr) handles, passed by
!!     value; a constructor returns its handle through a type(c_ptr) dummy;
!!   * host arrays are assumed-size real(c_double) / real(c_float) arrays
!!     (Fortran passes their address); arguments the C side takes as device
!!     addresses (the *_device / dev_* dummies) are type(c_ptr) by value;
!!   * C `unsigned` seeds are integer(c_int); strings are NUL-terminated
!!     character(kind=c_char) arrays (trim(s)//c_null_char);
!!   * every function returns 0 or a negative CB2_ERR_* code, and
!!     cb2_last_error returns a C string with the message.
!! The derived types cb2_params and cb2_sph_tables are bind(C) copies of
!! the C structs, field for field.
module m_calypso_b200
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: CB2_OK = 0
  integer(c_int), parameter :: CB2_ERR_ARG = -1
  integer(c_int), parameter :: CB2_ERR_CUDA = -2
  integer(c_int), parameter :: CB2_ERR_SINGULAR = -3
  integer(c_int), parameter :: CB2_ERR_NAN = -4
  integer(c_int), parameter :: CB2_ERR_STATE = -5
  integer(c_int), parameter :: CB2_ERR_TIMEOUT = -6
  integer(c_int), parameter :: CB2_PREC_FP64 = 0
  integer(c_int), parameter :: CB2_PREC_MIXED = 1

  !> control_sph_shell / control_MHD values of the shell (struct cb2_params)
  type, bind(C) :: cb2_params
    integer(c_int) :: ltr, nth, nph, nr, radial_grid_type
    real(c_double) :: r_icb, r_cmb
    real(c_double) :: dt
    real(c_double) :: coef_imp_v, coef_imp_t, coef_imp_b
    real(c_double) :: coef_velo, coef_d_velo, coef_buo, coef_cor, coef_lor
    real(c_double) :: coef_temp, coef_d_temp
    real(c_double) :: coef_magne, coef_d_magne, coef_induct
    integer(c_int) :: use_ref_temp
    real(c_double) :: depth_high_t, depth_low_t, high_temp, low_temp
    real(c_double) :: temp_icb, temp_cmb
    integer(c_int) :: nthreads
  end type cb2_params

  !> index tables of a single-domain grid, as m_spheric_parameter holds
  !! them (struct cb2_sph_tables): c_loc of the integer(c_int) arrays
  !! idx_gl_1d_rlm_j(nidx_rlm(2), 3) and idx_gl_1d_rtm_m(nidx_rtm(3), 2)
  type, bind(C) :: cb2_sph_tables
    integer(c_int) :: nidx_rlm(2), istep_rlm(2)
    type(c_ptr) :: idx_gl_1d_rlm_j
    integer(c_int) :: nidx_rtm(3), istep_rtm(3)
    type(c_ptr) :: idx_gl_1d_rtm_m
    integer(c_int) :: nidx_rtp(3), istep_rtp(3)
  end type cb2_sph_tables

  interface

    function cb2_last_error() bind(C, name='cb2_last_error') result(rc)
      import
      type(c_ptr) :: rc
    end function cb2_last_error

    function cb2_create(p, precision, device, out) bind(C, name='cb2_create') result(rc)
      import
      type(cb2_params), intent(in) :: p
      integer(c_int), value :: precision
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: out
      integer(c_int) :: rc
    end function cb2_create

    function cb2_destroy(ctx) bind(C, name='cb2_destroy') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function cb2_destroy

    function cb2_init_fields(ctx, kind, seed) bind(C, name='cb2_init_fields') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: kind
      integer(c_int), value :: seed
      integer(c_int) :: rc
    end function cb2_init_fields

    function cb2_start(ctx) bind(C, name='cb2_start') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function cb2_start

    function cb2_step(ctx, nsteps) bind(C, name='cb2_step') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      integer(c_int) :: rc
    end function cb2_step

    function cb2_step_graph(ctx, nsteps) bind(C, name='cb2_step_graph') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      integer(c_int) :: rc
    end function cb2_step_graph

    function cb2_sync(ctx) bind(C, name='cb2_sync') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function cb2_sync

    function cb2_time_steps(ctx, nsteps, use_graph, ms) bind(C, name='cb2_time_steps') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      integer(c_int), value :: use_graph
      real(c_double), intent(out) :: ms
      integer(c_int) :: rc
    end function cb2_time_steps

    function cb2_istep(ctx) bind(C, name='cb2_istep') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function cb2_istep

    function cb2_energies(ctx, out) bind(C, name='cb2_energies') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(7)
      integer(c_int) :: rc
    end function cb2_energies

    function cb2_energy_spectra(ctx, out_l, out_m, out_lm) &
        bind(C, name='cb2_energy_spectra') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: out_l(*)
      real(c_double), intent(inout) :: out_m(*)
      real(c_double), intent(inout) :: out_lm(*)
      integer(c_int) :: rc
    end function cb2_energy_spectra

    function cb2_energies_static(ctx, out) bind(C, name='cb2_energies_static') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(7)
      integer(c_int) :: rc
    end function cb2_energies_static

    function cb2_get_field(ctx, slot, host) bind(C, name='cb2_get_field') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: slot
      real(c_double), intent(inout) :: host(*)
      integer(c_int) :: rc
    end function cb2_get_field

    function cb2_set_field(ctx, slot, host) bind(C, name='cb2_set_field') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: slot
      real(c_double), intent(in) :: host(*)
      integer(c_int) :: rc
    end function cb2_set_field

    function cb2_get_field_device(ctx, slot, dev) bind(C, name='cb2_get_field_device') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: slot
      type(c_ptr), value :: dev
      integer(c_int) :: rc
    end function cb2_get_field_device

    function cb2_set_field_device(ctx, slot, dev) bind(C, name='cb2_set_field_device') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: slot
      type(c_ptr), value :: dev
      integer(c_int) :: rc
    end function cb2_set_field_device

    function cb2_step_host_state(ctx, state, out_energies) &
        bind(C, name='cb2_step_host_state') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: state(*)
      real(c_double), intent(out) :: out_energies(7)
      integer(c_int) :: rc
    end function cb2_step_host_state

    function cb2_get_restart_state(ctx, state) bind(C, name='cb2_get_restart_state') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: state(*)
      integer(c_int) :: rc
    end function cb2_get_restart_state

    function cb2_set_restart_state(ctx, state, istep) bind(C, name='cb2_set_restart_state') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: state(*)
      integer(c_int), value :: istep
      integer(c_int) :: rc
    end function cb2_set_restart_state

    function cb2_step_restart_state(ctx, state, out_energies) &
        bind(C, name='cb2_step_restart_state') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: state(*)
      real(c_double), intent(out) :: out_energies(7)
      integer(c_int) :: rc
    end function cb2_step_restart_state

    function cb2_sht_backward(ctx, nvec, nscal, spec, grid) &
        bind(C, name='cb2_sht_backward') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nvec
      integer(c_int), value :: nscal
      real(c_double), intent(in) :: spec(*)
      real(c_double), intent(inout) :: grid(*)
      integer(c_int) :: rc
    end function cb2_sht_backward

    function cb2_sht_forward(ctx, nvec, nscal, grid, spec) &
        bind(C, name='cb2_sht_forward') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: nvec
      integer(c_int), value :: nscal
      real(c_double), intent(in) :: grid(*)
      real(c_double), intent(inout) :: spec(*)
      integer(c_int) :: rc
    end function cb2_sht_forward

    function cb2_leg_bwd(ctx, t, ncomp, nvector, nscalar, n_WR, n_WS, WR, WS) &
        bind(C, name='cb2_leg_bwd') result(rc)
      import
      type(c_ptr), value :: ctx
      type(cb2_sph_tables), intent(in) :: t
      integer(c_int), value :: ncomp
      integer(c_int), value :: nvector
      integer(c_int), value :: nscalar
      integer(c_size_t), value :: n_WR
      integer(c_size_t), value :: n_WS
      real(c_double), intent(in) :: WR(*)
      real(c_double), intent(inout) :: WS(*)
      integer(c_int) :: rc
    end function cb2_leg_bwd

    function cb2_leg_fwd(ctx, t, ncomp, nvector, nscalar, n_WR, n_WS, WR, WS) &
        bind(C, name='cb2_leg_fwd') result(rc)
      import
      type(c_ptr), value :: ctx
      type(cb2_sph_tables), intent(in) :: t
      integer(c_int), value :: ncomp
      integer(c_int), value :: nvector
      integer(c_int), value :: nscalar
      integer(c_size_t), value :: n_WR
      integer(c_size_t), value :: n_WS
      real(c_double), intent(in) :: WR(*)
      real(c_double), intent(inout) :: WS(*)
      integer(c_int) :: rc
    end function cb2_leg_fwd

    function cb2_fft_bwd(ctx, t, ncomp, n_WR, WR, fld_rtp) bind(C, name='cb2_fft_bwd') result(rc)
      import
      type(c_ptr), value :: ctx
      type(cb2_sph_tables), intent(in) :: t
      integer(c_int), value :: ncomp
      integer(c_size_t), value :: n_WR
      real(c_double), intent(in) :: WR(*)
      real(c_double), intent(inout) :: fld_rtp(*)
      integer(c_int) :: rc
    end function cb2_fft_bwd

    function cb2_fft_fwd(ctx, t, ncomp, frc_rtp, n_WS, WS) bind(C, name='cb2_fft_fwd') result(rc)
      import
      type(c_ptr), value :: ctx
      type(cb2_sph_tables), intent(in) :: t
      integer(c_int), value :: ncomp
      real(c_double), intent(in) :: frc_rtp(*)
      integer(c_size_t), value :: n_WS
      real(c_double), intent(inout) :: WS(*)
      integer(c_int) :: rc
    end function cb2_fft_fwd

    function cb2_fft_products(ctx, t, n_WR, WR, n_WS, WS) &
        bind(C, name='cb2_fft_products') result(rc)
      import
      type(c_ptr), value :: ctx
      type(cb2_sph_tables), intent(in) :: t
      integer(c_size_t), value :: n_WR
      real(c_double), intent(in) :: WR(*)
      integer(c_size_t), value :: n_WS
      real(c_double), intent(inout) :: WS(*)
      integer(c_int) :: rc
    end function cb2_fft_products

    function cb2_legendre_trans_mode(legendre_trans_loop_ctl) &
        bind(C, name='cb2_legendre_trans_mode') result(rc)
      import
      character(kind=c_char), intent(in) :: legendre_trans_loop_ctl(*)
      integer(c_int) :: rc
    end function cb2_legendre_trans_mode

    function cb2_fft_library_known(fft_library_ctl) bind(C, name='cb2_fft_library_known') result(rc)
      import
      character(kind=c_char), intent(in) :: fft_library_ctl(*)
      integer(c_int) :: rc
    end function cb2_fft_library_known

    function cb2_get_gauss(ctx, colat, weight) bind(C, name='cb2_get_gauss') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(inout) :: colat(*)
      real(c_double), intent(inout) :: weight(*)
      integer(c_int) :: rc
    end function cb2_get_gauss

    function cb2_get_plm(ctx, l, m, p, dp) bind(C, name='cb2_get_plm') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), value :: l
      integer(c_int), value :: m
      real(c_double), intent(inout) :: p(*)
      real(c_double), intent(inout) :: dp(*)
      integer(c_int) :: rc
    end function cb2_get_plm

    function cb2_alloc_pinned(bytes, out) bind(C, name='cb2_alloc_pinned') result(rc)
      import
      integer(c_size_t), value :: bytes
      type(c_ptr), intent(out) :: out
      integer(c_int) :: rc
    end function cb2_alloc_pinned

    function cb2_free_pinned(p) bind(C, name='cb2_free_pinned') result(rc)
      import
      type(c_ptr), value :: p
      integer(c_int) :: rc
    end function cb2_free_pinned

    function cb2_autotune(ctx) bind(C, name='cb2_autotune') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function cb2_autotune

    function cb2_get_tuning(ctx, tuning) bind(C, name='cb2_get_tuning') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), intent(inout) :: tuning(5)
      integer(c_int) :: rc
    end function cb2_get_tuning

    function cb2_tuning_note(ctx) bind(C, name='cb2_tuning_note') result(rc)
      import
      type(c_ptr), value :: ctx
      type(c_ptr) :: rc
    end function cb2_tuning_note

    function cb2_set_tuning(ctx, tuning) bind(C, name='cb2_set_tuning') result(rc)
      import
      type(c_ptr), value :: ctx
      integer(c_int), intent(in) :: tuning(5)
      integer(c_int) :: rc
    end function cb2_set_tuning

    function cb2_ensemble_create(params, n, precision, device, autotune_shapes, out) &
        bind(C, name='cb2_ensemble_create') result(rc)
      import
      type(cb2_params), intent(in) :: params(*)
      integer(c_int), value :: n
      integer(c_int), value :: precision
      integer(c_int), value :: device
      integer(c_int), value :: autotune_shapes
      type(c_ptr), intent(out) :: out
      integer(c_int) :: rc
    end function cb2_ensemble_create

    function cb2_ensemble_destroy(e) bind(C, name='cb2_ensemble_destroy') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int) :: rc
    end function cb2_ensemble_destroy

    function cb2_ensemble_size(e) bind(C, name='cb2_ensemble_size') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int) :: rc
    end function cb2_ensemble_size

    function cb2_ensemble_shell(e, i) bind(C, name='cb2_ensemble_shell') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int), value :: i
      type(c_ptr) :: rc
    end function cb2_ensemble_shell

    function cb2_ensemble_init_fields(e, kind, seed0) &
        bind(C, name='cb2_ensemble_init_fields') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int), value :: kind
      integer(c_int), value :: seed0
      integer(c_int) :: rc
    end function cb2_ensemble_init_fields

    function cb2_ensemble_step(e, nsteps) bind(C, name='cb2_ensemble_step') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int), value :: nsteps
      integer(c_int) :: rc
    end function cb2_ensemble_step

    function cb2_ensemble_set_batched(e, on) bind(C, name='cb2_ensemble_set_batched') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int), value :: on
      integer(c_int) :: rc
    end function cb2_ensemble_set_batched

    function cb2_ensemble_sync(e) bind(C, name='cb2_ensemble_sync') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int) :: rc
    end function cb2_ensemble_sync

    function cb2_ensemble_time_steps(e, nsteps, ms) &
        bind(C, name='cb2_ensemble_time_steps') result(rc)
      import
      type(c_ptr), value :: e
      integer(c_int), value :: nsteps
      real(c_double), intent(out) :: ms
      integer(c_int) :: rc
    end function cb2_ensemble_time_steps

    function cb2_ensemble_energies(e, out) bind(C, name='cb2_ensemble_energies') result(rc)
      import
      type(c_ptr), value :: e
      real(c_double), intent(inout) :: out(*)
      integer(c_int) :: rc
    end function cb2_ensemble_energies

    function cb2_mlp_create(nin, nhid, nout, seed, out) bind(C, name='cb2_mlp_create') result(rc)
      import
      integer(c_int), value :: nin
      integer(c_int), value :: nhid
      integer(c_int), value :: nout
      integer(c_int), value :: seed
      type(c_ptr), intent(out) :: out
      integer(c_int) :: rc
    end function cb2_mlp_create

    function cb2_mlp_destroy(net) bind(C, name='cb2_mlp_destroy') result(rc)
      import
      type(c_ptr), value :: net
      integer(c_int) :: rc
    end function cb2_mlp_destroy

    function cb2_mlp_num_params(net) bind(C, name='cb2_mlp_num_params') result(rc)
      import
      type(c_ptr), value :: net
      integer(c_int) :: rc
    end function cb2_mlp_num_params

    function cb2_mlp_get_params(net, host) bind(C, name='cb2_mlp_get_params') result(rc)
      import
      type(c_ptr), value :: net
      real(c_float), intent(inout) :: host(*)
      integer(c_int) :: rc
    end function cb2_mlp_get_params

    function cb2_mlp_set_params(net, host) bind(C, name='cb2_mlp_set_params') result(rc)
      import
      type(c_ptr), value :: net
      real(c_float), intent(in) :: host(*)
      integer(c_int) :: rc
    end function cb2_mlp_set_params

    function cb2_mlp_forward(net, dev_x, rows, dev_y) bind(C, name='cb2_mlp_forward') result(rc)
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: dev_x
      integer(c_long_long), value :: rows
      type(c_ptr), value :: dev_y
      integer(c_int) :: rc
    end function cb2_mlp_forward

    function cb2_mlp_loss_grad(net, dev_x, dev_t, rows, loss, host_grad) &
        bind(C, name='cb2_mlp_loss_grad') result(rc)
      import
      type(c_ptr), value :: net
      type(c_ptr), value :: dev_x
      real(c_float), intent(in) :: dev_t(*)
      integer(c_long_long), value :: rows
      real(c_double), intent(out) :: loss
      real(c_float), intent(inout) :: host_grad(*)
      integer(c_int) :: rc
    end function cb2_mlp_loss_grad

    function cb2_mlp_adam_step(net, lr, beta1, beta2, eps) &
        bind(C, name='cb2_mlp_adam_step') result(rc)
      import
      type(c_ptr), value :: net
      real(c_float), value :: lr
      real(c_float), value :: beta1
      real(c_float), value :: beta2
      real(c_float), value :: eps
      integer(c_int) :: rc
    end function cb2_mlp_adam_step

    function cb2_mlp_sync(net) bind(C, name='cb2_mlp_sync') result(rc)
      import
      type(c_ptr), value :: net
      integer(c_int) :: rc
    end function cb2_mlp_sync

    function cb2_filter_fields(src, dst) bind(C, name='cb2_filter_fields') result(rc)
      import
      type(c_ptr), value :: src
      type(c_ptr), value :: dst
      integer(c_int) :: rc
    end function cb2_filter_fields

    function cb2_filter_terms(src, dst, dev_out) bind(C, name='cb2_filter_terms') result(rc)
      import
      type(c_ptr), value :: src
      type(c_ptr), value :: dst
      type(c_ptr), value :: dev_out
      integer(c_int) :: rc
    end function cb2_filter_terms

    function cb2_closure_features(ctx, dev_x) bind(C, name='cb2_closure_features') result(rc)
      import
      type(c_ptr), value :: ctx
      type(c_ptr), value :: dev_x
      integer(c_int) :: rc
    end function cb2_closure_features

    function cb2_closure_targets(ctx, dev_hi, dev_y) bind(C, name='cb2_closure_targets') result(rc)
      import
      type(c_ptr), value :: ctx
      type(c_ptr), value :: dev_hi
      type(c_ptr), value :: dev_y
      integer(c_int) :: rc
    end function cb2_closure_targets

    function cb2_closure_attach(ctx, net, norm) bind(C, name='cb2_closure_attach') result(rc)
      import
      type(c_ptr), value :: ctx
      type(c_ptr), value :: net
      real(c_float), intent(in) :: norm(*)
      integer(c_int) :: rc
    end function cb2_closure_attach

    function cb2_stage_times(ctx, ms) bind(C, name='cb2_stage_times') result(rc)
      import
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: ms(32)
      integer(c_int) :: rc
    end function cb2_stage_times


  end interface

end module m_calypso_b200
