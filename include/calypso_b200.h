/*
 * calypso_b200.h -- C ABI of the B200 (sm_100a) time-step hot path of the
 * Calypso spherical-shell MHD dynamo code.
 *
 * The reference (hlokavarapu/calypso) is Fortran 90; its hot path is reached
 * through module procedures with module-global state.  Each entry point
 * below names the reference routine it replaces (paths relative to the
 * reference's src/Fortran_libraries).  A Fortran host binds these with the
 * bind(C) interfaces of include/m_calypso_b200.f90; the Python host
 * (calypso_b200/) binds them with ctypes.
 *
 * Conventions
 *   - every call returns 0 on success or a negative CB2_ERR_* code;
 *     cb2_last_error() gives a message.  Nothing aborts the process.
 *   - spectral (rj) arrays are float64 [nr][jmax] with j = l*(l+1)+m,
 *     m < 0 holding the sin(|m| phi) part (the reference's d_rj(inod, field)
 *     with inod = j + (k-1)*jmax when its j table is ordered by l*(l+1)+m).
 *   - vector fields are three slots (poloidal S, dS/dr, toroidal T).
 *   - grid arrays are float64 [comp][nr][nth][nph], theta index 0 nearest
 *     the south pole (reference Gauss ordering), phi_p = 2 pi p / nph.
 *   - host pointers are plain host memory; the library copies through its
 *     own pinned staging buffers.  Calls on one context are not thread safe.
 */
#ifndef CALYPSO_B200_H
#define CALYPSO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CB2_OK 0
#define CB2_ERR_ARG -1        /* bad argument / unsupported configuration   */
#define CB2_ERR_CUDA -2       /* a CUDA call failed (message has the name)  */
#define CB2_ERR_SINGULAR -3   /* zero pivot in a radial LU factorisation    */
#define CB2_ERR_NAN -4        /* NaN/Inf found in the energy diagnostics    */
#define CB2_ERR_STATE -5      /* call out of order (e.g. step before start) */
#define CB2_ERR_TIMEOUT -6    /* a bounded wait inside a tensor-core kernel
                                 ran out; the results of that step are void
                                 and later launches on the context do
                                 nothing: destroy it.  Each wait's budget is
                                 200 ms, or CB2_PIPE_WAIT_NS (nanoseconds)
                                 from the environment at cb2_create */

#define CB2_PREC_FP64 0       /* plain path: every stage in float64          */
#define CB2_PREC_MIXED 1      /* Legendre split-fp16 tcgen05, fp32 FFT and
                                 products, fp64 radial solves / diagnostics */

/* Shell and equation parameters: the values the reference reads from
 * control_sph_shell (num_grid_sph) and control_MHD (model, control) and
 * turns into coefficients in F/MHD_src/sph_MHD/material_property.f90. */
typedef struct cb2_params {
  int ltr;              /* truncation_level_ctl                          */
  int nth;              /* ngrid_meridonal_ctl                           */
  int nph;              /* ngrid_zonal_ctl                               */
  int nr;               /* radial points = num_fluid_grid_ctl + 1        */
  int radial_grid_type; /* 0 equidistance, 1 Chebyshev                   */
  double r_icb, r_cmb;
  double dt;
  double coef_imp_v, coef_imp_t, coef_imp_b;
  double coef_velo, coef_d_velo, coef_buo, coef_cor, coef_lor;
  double coef_temp, coef_d_temp;
  double coef_magne, coef_d_magne, coef_induct;
  int use_ref_temp;     /* ref_temp_ctl spherical_shell                  */
  double depth_high_t, depth_low_t, high_temp, low_temp;
  double temp_icb, temp_cmb;   /* fixed total temperature at the walls   */
  int nthreads;         /* unused by the GPU library (layout compatible) */
} cb2_params;

typedef struct cb2_ctx cb2_ctx;

const char *cb2_last_error(void);

/* SPH_initialize_MHD set-up part (programs/SPH_MHD/SPH_analyzer_MHD.f90:21-110):
 * radial grid and FDM weights (set_radius_func.f90), boundary weights
 * (MHD_src/sph_MHD/set_bc_sph_mhd.f90), Gauss nodes and Schmidt P_l^m on the
 * GPU (PARALLEL_src/SPH_SHELL_src/init_sph_trans.f90:64-92), Coriolis
 * couplings (MHD_src/sph_MHD/const_coriolis_sph_rlm.f90:34-67) and the
 * banded LU factors of the implicit operators on the GPU
 * (MHD_src/sph_MHD/const_radial_mat_4_sph.f90:33-114).  device < 0 keeps
 * the current device. */
int cb2_create(const cb2_params *p, int precision, int device, cb2_ctx **out);
/* sel_finalize_legendre_trans + deallocation of the module globals */
int cb2_destroy(cb2_ctx *ctx);

/* Initial state on the device: kind 1 = dynamo benchmark case 1
 * (MHD_src/sph_MHD/set_initial_sph_dynamo.f90 sph_initial_data_control with
 * rst_ctl dynamo_benchmark_1); kind 2 = seeded thermal perturbation on
 * random l <= 8 modes plus a weak dipole-dominated seed field.  Ends with
 * cb2_start(). */
int cb2_init_fields(cb2_ctx *ctx, int kind, unsigned seed);
/* set_sph_field_to_start + first nonlinear (SPH_analyzer_MHD.f90:92-101):
 * recompute gradients, vorticity, current, diffusion terms and the
 * nonlinear terms of the state loaded with cb2_set_field. */
int cb2_start(cb2_ctx *ctx);
/* SPH_analyze_MHD (SPH_analyzer_MHD.f90:115-202) repeated nsteps times on
 * the context's stream (asynchronous): Euler first step, Adams-Bashforth 2
 * after, Crank-Nicolson radial solves, nonlinear terms through the SHT. */
int cb2_step(cb2_ctx *ctx, int nsteps);
/* the same nsteps, captured once as a CUDA graph and replayed */
int cb2_step_graph(cb2_ctx *ctx, int nsteps);
int cb2_sync(cb2_ctx *ctx);
/* nsteps of cb2_step (use_graph = 0) or cb2_step_graph (1) bracketed by CUDA
 * events on the context's stream; ms = device time.  Synchronises. */
int cb2_time_steps(cb2_ctx *ctx, int nsteps, int use_graph, double *ms);
int cb2_istep(const cb2_ctx *ctx);
/* volume mean squares of sph_pwr_volume_s.dat after the last step
 * (PARALLEL_src/SPH_SHELL_src/cal_rms_fields_by_sph.f90 cal_rms_sph_outer_core):
 * out = K_pol, K_tor, K, <T^2> (total temperature), M_pol, M_tor, M.
 * Synchronises.  Returns CB2_ERR_NAN if any value is not finite
 * (MHD_src/sph_MHD/cal_sol_sph_fluid_crank.f90 check_NaN_temperature). */
int cb2_energies(cb2_ctx *ctx, double out[7]);
/* The seven energies of cb2_energies as volume spectra (the reference's
 * sph_pwr_volume_l.dat, _m.dat and _lm.dat columns:
 * PARALLEL_src/SPH_SHELL_src/sum_sph_rms_data.f90:135-192 grouping,
 * cal_rms_by_sph_spectr.f90:74-172 per mode): out_l[q (L+1) + l] over the
 * modes of degree l, out_m[q (L+1) + m] over order |m|, out_lm[q (L+1) + d]
 * over l - |m| = d; q in the order of cb2_energies.  Synchronises;
 * CB2_ERR_NAN on a non-finite value. */
int cb2_energy_spectra(cb2_ctx *ctx, double *out_l, double *out_m, double *out_lm);
/* The same seven values as cb2_energies, computed without allocating any
 * device memory: the partial sums go to a static array in the library (one
 * per device, 3.5 MiB) instead of a buffer of the context.  This entry point
 * has no counterpart in the reference; it is for hosts that must not call
 * the CUDA allocator during a run (device memory owned and budgeted by
 * another component, or a monitoring loop that must not add allocations).
 * Limits: jmax = (L+1)^2 <= 65536 (L <= 255), else CB2_ERR_ARG.  Every call
 * on a device shares the array (it keeps the last call's contents; nothing
 * in it needs to start at zero), so calls that overlap on one device race:
 * serialise them.  cb2_create looks the array up on its device, so the
 * array's memory is reserved while a context is set up, never by a call of
 * this function.  Synchronises. */
int cb2_energies_static(cb2_ctx *ctx, double out[7]);

/* d_rj field slot access (host buffers of nr*jmax float64).  Slot numbers:
 * 0 velocity, 3 vorticity, 6 magnetic field, 9 current density,
 * 12 (perturbation) temperature; other slots are work fields. */
int cb2_get_field(cb2_ctx *ctx, int slot, double *host);
int cb2_set_field(cb2_ctx *ctx, int slot, const double *host);
/* the same with device buffers on the context's device (no copy to host) */
int cb2_get_field_device(cb2_ctx *ctx, int slot, double *dev);
int cb2_set_field_device(cb2_ctx *ctx, int slot, const double *dev);

/* Drop-in for a host that keeps d_rj in its own memory (the reference's
 * Fortran host): copies in the 20 fields one step reads, advances one
 * Adams-Bashforth step (call cb2_step for the first, Euler step) and copies
 * the same 20 fields back.  state = 20 x nr*jmax float64 in this order:
 * vorticity S,T; vorticity diffusion S,T; curl of forces S,T; its previous
 * value S,T; magnetic field S,T; magnetic diffusion S,T; induction S,T; its
 * previous value S,T; temperature; thermal diffusion; heat advection; its
 * previous value (negated).  out_energies may be NULL. */
int cb2_step_host_state(cb2_ctx *ctx, double *state, double out_energies[7]);

/* The reference's restart state (MHD_src/IO/sph_mhd_rst_IO_control.f90:89-145,
 * MHD_src/sph_MHD/set_sph_restart_IO.f90:62-142: the fields of a restart
 * file): 14 x nr*jmax float64 host array, in this order: velocity S, dS/dr,
 * T; temperature (the total temperature, reference profile included, as
 * the reference writes it after trans_per_temp_to_temp_sph); magnetic field
 * S, dS/dr, T; previous_momentum (3); previous_induction (3);
 * previous_heat (the negated heat advection of the last step).
 * cb2_get_restart_state reads it after any step.  cb2_set_restart_state
 * loads it and restarts the loop as the reference's start from a restart
 * file does (set_sph_field_to_start and the first nonlinear terms); the
 * next step is an Adams-Bashforth step numbered istep + 1. */
int cb2_get_restart_state(cb2_ctx *ctx, double *state);
int cb2_set_restart_state(cb2_ctx *ctx, const double *state, int istep);
/* One Adams-Bashforth step of a host that keeps the restart state in its
 * own memory (14 fields in and out instead of the 20 of
 * cb2_step_host_state): loads the state, computes its derived fields and
 * nonlinear terms, advances one step and returns the new state.  The
 * nonlinear terms of the new state are left to the next call (or to the
 * next cb2_step, which computes them first).  out_energies may be NULL.
 * A step does not write the dS/dr entries of previous_momentum and
 * previous_induction (entries 8 and 11), so the call leaves them as they are
 * in `state` and copies 12 entries back instead of 14. */
int cb2_step_restart_state(cb2_ctx *ctx, double *state, double out_energies[7]);

/* Spherical transform of nvec vectors + nscal scalars at every radius
 * (PARALLEL_src/SPH_SHELL_src/legendre_transform_select.f90:309-439
 *  sel_backward_legendre_trans / sel_forward_legendre_trans, plus
 *  MHD_src/sph_MHD/MHD_FFT_selector.F90:185-249 back/fwd_MHD_FFT_sel_from_recv).
 * spec: (3*nvec+nscal) x nr x jmax float64; grid: (3*nvec+nscal) x nr x nth x
 * nph float64, vector components (r, theta, phi).  Host buffers.  The
 * context's precision selects the Legendre / FFT arithmetic. */
int cb2_sht_backward(cb2_ctx *ctx, int nvec, int nscal, const double *spec, double *grid);
int cb2_sht_forward(cb2_ctx *ctx, int nvec, int nscal, const double *grid, double *spec);

/* Index tables of a single-domain spherical grid, as the reference's
 * module SERIAL_src/SPH_SPECTR_src/m_spheric_parameter.f90 holds them for
 * its Legendre and FFT routines (Fortran order, 1-based values):
 *   rlm spectra   sp_rlm(comp + ncomp*((k-1)*istep_rlm(1) + (j-1)*istep_rlm(2)))
 *                 idx_gl_1d_rlm_j(j, 1:3) = global j, degree l, order m
 *   rtm Fourier   vr_rtm(comp + ncomp*((k-1)*istep_rtm(1) + (l-1)*istep_rtm(2)
 *                                      + (mp-1)*istep_rtm(3)))
 *                 idx_gl_1d_rtm_m(mp, 1:2) = global index, order m (m < 0:
 *                 the sin(|m| phi) coefficient; colatitude l is the Gauss
 *                 node l counted from the south pole)
 *   rtp grid      fld_rtp(inod, comp), inod = (k-1)*istep_rtp(1)
 *                 + (l-1)*istep_rtp(2) + (p-1)*istep_rtp(3) + 1
 * The arrays are column-major (nidx x 3 and nidx x 2) int32. */
typedef struct cb2_sph_tables {
  int nidx_rlm[2];              /* radial points, harmonics of the rlm layout  */
  int istep_rlm[2];
  const int *idx_gl_1d_rlm_j;   /* nidx_rlm(2) x 3                            */
  int nidx_rtm[3];              /* radial points, colatitudes, orders          */
  int istep_rtm[3];
  const int *idx_gl_1d_rtm_m;   /* nidx_rtm(3) x 2                            */
  int nidx_rtp[3];              /* radial points, colatitudes, longitudes      */
  int istep_rtp[3];
} cb2_sph_tables;

/* Legendre transform alone, in the context's precision, on the reference's
 * transposed buffers (PARALLEL_src/SPH_SHELL_src/legendre_transform_select.f90:
 * 309-317 sel_backward_legendre_trans and 375-383 sel_forward_legendre_trans,
 * same arguments).  Backward: WR = sp_rlm (per vector S, dS/dr, T; then the
 * scalars) -> WS = vr_rtm (per vector v_r, v_theta, v_phi; then the
 * scalars), WS cleared first as the reference's transforms do.  Forward:
 * WR = vr_rtm -> WS = sp_rlm.  ncomp is the component stride (>= 3 nvector
 * + nscalar); components beyond 3 nvector + nscalar are left alone.  WR and
 * WS may be host or device memory (device buffers are used in place). */
int cb2_leg_bwd(cb2_ctx *ctx, const cb2_sph_tables *t, int ncomp, int nvector, int nscalar, size_t n_WR,
                size_t n_WS, const double *WR, double *WS);
int cb2_leg_fwd(cb2_ctx *ctx, const cb2_sph_tables *t, int ncomp, int nvector, int nscalar, size_t n_WR,
                size_t n_WS, const double *WR, double *WS);
/* Longitudinal transform alone (MHD_src/sph_MHD/MHD_FFT_selector.F90:219-249
 * back_MHD_FFT_sel_from_recv and 185-215 fwd_MHD_FFT_sel_from_recv, plus
 * the rtm <-> rtp transposes around them): Fourier coefficients in the rtm
 * layout (a_m, b_m with f = a_0 + sum a_m cos m phi + b_m sin m phi) <->
 * grid fld_rtp(nnod_rtp, ncomp), nnod_rtp = nr nth nph.  Host or device
 * buffers. */
int cb2_fft_bwd(cb2_ctx *ctx, const cb2_sph_tables *t, int ncomp, size_t n_WR, const double *WR,
                double *fld_rtp);
int cb2_fft_fwd(cb2_ctx *ctx, const cb2_sph_tables *t, int ncomp, const double *frc_rtp, size_t n_WS,
                double *WS);

/* The grid-space products alone, with the FFTs around them: the kernel the
 * time step runs for MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:35-84
 * (s_cal_nonlinear_sph_MHD) between back_MHD_FFT_sel_from_recv and
 * fwd_MHD_FFT_sel_from_recv.  WR: 13 Fourier components in the rtm layout
 * (ncomp = 13: u, w, B, J as r, theta, phi, then T); WS: 12 (ncomp = 12:
 * c_v w x u, c_L J x B, c_i u x B, c_T u T), the coefficients of the
 * context's parameters.  Host or device buffers. */
int cb2_fft_products(cb2_ctx *ctx, const cb2_sph_tables *t, size_t n_WR, const double *WR, size_t n_WS,
                     double *WS);

/* Precision selected by a Legendre_trans_loop_ctl value of control_MHD
 * (set_legendre_trans_mode_ctl, legendre_transform_select.f90:181-224):
 * "B200_mixed" or "B200_tcgen05" (any case) -> CB2_PREC_MIXED; "B200_fp64",
 * every loop name of the reference and an unknown value (the reference then
 * falls back to original_loop) -> CB2_PREC_FP64.  NULL -> CB2_PREC_FP64. */
int cb2_legendre_trans_mode(const char *legendre_trans_loop_ctl);
/* FFT_library_ctl (set_fft_library_ctl, SERIAL_src/FFT_wrapper/
 * m_FFT_selector.f90:60-80): 1 for the names the reference knows (fftpack,
 * ispack, fftw, fftw3 and their _single / _field forms) and "B200", 0 for
 * others (the reference keeps its default then).  Every name selects the
 * library's own FFT, in the precision of the Legendre mode. */
int cb2_fft_library_known(const char *fft_library_ctl);

/* Tables computed on the device, for checking: Gauss colatitudes/weights
 * (nth), Schmidt P_l^m and dP/dtheta at the nth nodes for one (l, m>=0). */
int cb2_get_gauss(cb2_ctx *ctx, double *colat, double *weight);
int cb2_get_plm(cb2_ctx *ctx, int l, int m, double *p, double *dp);

/* pinned host memory for cb2_step_host_state callers without an allocator
 * of their own (the library copies pinned buffers without staging) */
int cb2_alloc_pinned(size_t bytes, void **out);
int cb2_free_pinned(void *p);

/* Kernel-variant autotuner (the counterpart of the reference's
 * select_legendre_transform, MHD_src/sph_MHD/sph_transforms_4_MHD.f90:309-426,
 * which times its Legendre loop variants at start-up): times every
 * candidate tile / launch shape of the transform kernels on this context
 * and keeps the fastest.  Only before cb2_init_fields / cb2_start (it
 * overwrites the work fields).  tuning[5]: float64 backward kernel (1: on
 * the float64 tensor cores; 2, 4: on the CUDA cores with that radial tile),
 * float64 forward kernel (1, 2: on the CUDA cores with that radial tile; 3:
 * on the float64 tensor cores), mixed pack radial tile, FFT kernel of either
 * precision (384: the four-step kernel, used where nphi = 3 (ltr + 1);
 * 128, 256, 512: the Stockham kernel, float64 always with 512 threads), and
 * 1 to run the explicit update, the radial solves and the derived fields
 * of the step as one kernel, 0 (the default) as separate kernels; -1
 * (fixed) where the one kernel cannot take the context (cb2_tuning_note
 * says why). */
int cb2_autotune(cb2_ctx *ctx);
int cb2_get_tuning(const cb2_ctx *ctx, int tuning[5]);
int cb2_set_tuning(cb2_ctx *ctx, const int tuning[5]);
/* Why the one-kernel Crank-Nicolson step is unavailable on this context
 * (tuning entry 4 = -1), e.g. a radial LU factor with a row interchange
 * more than two rows away; "" when it is available.  Owned by the context. */
const char *cb2_tuning_note(const cb2_ctx *ctx);

/* Ensemble of independent shells (any mix of truncations and parameters),
 * advanced together: one CUDA graph holds a time step of every shell, so one
 * graph launch advances all of them.  By default each shell's whole step is
 * one branch of the graph.  Batched (cb2_ensemble_set_batched(e, 1),
 * mixed-precision shells): each of the two tensor-core Legendre GEMMs is one
 * persistent launch over the tiles of every shell, and the other kernels of
 * the step run as parallel per-shell branches between them.
 * No counterpart in the reference (it runs one shell per job).  Shells of
 * one shape (ltr, nr, nth, nph) share one autotuning when
 * autotune_shapes != 0.  Shell i is an ordinary context
 * (cb2_ensemble_shell); call cb2_ensemble_sync before using it directly
 * after cb2_ensemble_step. */
typedef struct cb2_ensemble cb2_ensemble;
int cb2_ensemble_create(const cb2_params *params, int n, int precision, int device, int autotune_shapes,
                        cb2_ensemble **out);
int cb2_ensemble_destroy(cb2_ensemble *e);
int cb2_ensemble_size(const cb2_ensemble *e);
cb2_ctx *cb2_ensemble_shell(cb2_ensemble *e, int i);
/* shell i gets cb2_init_fields(kind, seed0 + i) */
int cb2_ensemble_init_fields(cb2_ensemble *e, int kind, unsigned seed0);
int cb2_ensemble_step(cb2_ensemble *e, int nsteps);
/* on != 0: batched Legendre GEMM launches (default off); takes effect at the
 * next cb2_ensemble_step, with identical results either way */
int cb2_ensemble_set_batched(cb2_ensemble *e, int on);
int cb2_ensemble_sync(cb2_ensemble *e);
/* nsteps of cb2_ensemble_step bracketed by CUDA events; ms = device time */
int cb2_ensemble_time_steps(cb2_ensemble *e, int nsteps, double *ms);
/* out = n x 7 energies (cb2_energies of each shell) */
int cb2_ensemble_energies(cb2_ensemble *e, double *out);

/* Learned spectral subgrid closure.  No counterpart in the reference (its
 * SGS hooks, MHD_src/sph_MHD/cal_explicit_terms.f90:70-95, are unused on
 * the spherical-shell path).  A low-resolution shell misses the part of its
 * nonlinear terms carried by modes it does not resolve; a small MLP
 * predicts it per radial level and (l, m) from 16 local spectral features
 * (the 13 coefficients of velocity, vorticity, magnetic field, current and
 * temperature, l/L, m/L, r) for the 5 explicit nonlinear terms (curl of
 * the forces S, T; induction S, T; heat advection).  Weights bfloat16,
 * float32 accumulation; trained on the GPU by these kernels. */
typedef struct cb2_mlp cb2_mlp;
/* MLP nin -> nhid -> nhid -> nout, SiLU, seeded initial weights */
int cb2_mlp_create(int nin, int nhid, int nout, unsigned seed, cb2_mlp **out);
int cb2_mlp_destroy(cb2_mlp *net);
int cb2_mlp_num_params(const cb2_mlp *net);
/* float32 master parameters W1[nhid][nin], b1, W2[nhid][nhid], b2, W3[nout][nhid], b3 */
int cb2_mlp_get_params(cb2_mlp *net, float *host);
int cb2_mlp_set_params(cb2_mlp *net, const float *host);
/* device buffers: x = rows x nin, y = rows x nout (float32) */
int cb2_mlp_forward(cb2_mlp *net, const float *dev_x, long long rows, float *dev_y);
/* mean squared error against dev_t and its gradient (kept for
 * cb2_mlp_adam_step; also copied to host_grad when it is not NULL) */
int cb2_mlp_loss_grad(cb2_mlp *net, const float *dev_x, const float *dev_t, long long rows, double *loss,
                      float *host_grad);
int cb2_mlp_adam_step(cb2_mlp *net, float lr, float beta1, float beta2, float eps);
int cb2_mlp_sync(cb2_mlp *net);
/* dst state := src state truncated to dst's L and restricted to dst's
 * radial points (a subset of src's Chebyshev points), then cb2_start(dst) */
int cb2_filter_fields(cb2_ctx *src, cb2_ctx *dst);
/* src's 5 nonlinear terms filtered onto dst's shape: dev_out = 5 x nr x jmax float64 */
int cb2_filter_terms(cb2_ctx *src, cb2_ctx *dst, double *dev_out);
/* features (nr*jmax x 16) and targets (nr*jmax x 5: dev_hi minus ctx's own
 * terms) of ctx's current state, float32 device buffers */
int cb2_closure_features(cb2_ctx *ctx, float *dev_x);
int cb2_closure_targets(cb2_ctx *ctx, const double *dev_hi, float *dev_y);
/* attach (net != NULL) or detach the closure: each step then adds
 * net((features - mean[k]) / std[k]) * scale[k] to the 5 nonlinear terms at
 * the interior radial levels k (the walls are left to the boundary
 * conditions).  norm = nr x 16 means, nr x 16 standard deviations, nr x 5
 * output scales.  Attach before the step graph is captured; one context
 * per network at a time. */
int cb2_closure_attach(cb2_ctx *ctx, cb2_mlp *net, const float *norm);

/* CUDA-event time of the last cb2_step/cb2_step_graph call, per stage
 * (stage ids follow the reference's elapsed-time labels of
 * MHD_src/IO/init_sph_MHD_elapsed_label.f90: 6 explicit, 7 implicit,
 * 22 Legendre backward, 23 Legendre forward, 24 FFT+products, 17 rj
 * operators with the Coriolis term; 13, the reference's Coriolis label,
 * stays zero since the term is computed inside 17).  ms[0..31]; only
 * filled when CB2_TIMERS=1 in the env. */
int cb2_stage_times(cb2_ctx *ctx, double ms[32]);

#ifdef __cplusplus
}
#endif
#endif
