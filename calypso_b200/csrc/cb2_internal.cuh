// cb2_internal.cuh -- private state and helpers of libcalypso_b200.
//
// Device layouts (HBM):
//   spectral field  f[slot][k][jj]   float64, jj = "m-major" index: for
//                   m = 0..L the block of l = m..L of order +m, then (m>0)
//                   the block of l = m..L of order -m.  All rj operators
//                   are elementwise in jj and 3-point stencils in k.
//   Fourier data    F[theta][k][c][s] with s = 2m (cos, order +m) and
//                   s = 2m+1 (sin, order -m), NS = 2(L+1) slots per row:
//                   one (theta, k) row of all components is contiguous for
//                   the fused FFT + product kernel.
//   Legendre tables per order m:  P_lt[m][l-m][i], i over the nh = nth/2
//                   Gauss nodes nearest the south pole (the other half
//                   follows from the parity of P_l^m), and P_tl[m][i][l-m].
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/calypso_b200.h"

namespace cb2 {

// field slots: the same numbering as the reference-side diagnostics use
enum Slot {
  VELO = 0, VORT = 3, MAGNE = 6, CURRENT = 9, TEMP = 12, WDIFF = 13,
  BDIFF = 16, TDIFF = 19, MADV = 20, LOR = 23, VPIND = 26, HFLUX = 29,
  ROTINERT = 32, ROTLOR = 35, INDUCT = 38, HADV = 41, ROTCOR = 42,
  ROTBUO = 45, FORCES = 48, PREMOM = 51, PREUXB = 54, PREHEAT = 57,
  NSLOT = 58
};

// one-sided boundary weights (see host set-up in cb2_tables.cu)
struct BCW {
  double fix_fld_icb[3][4], fix_fld_cmb[3][4];
  double fix_dr_icb[3][4], fix_dr_cmb[3][4];
  double r_icb[3], r_cmb[3];
};

// everything the rj kernels read by value
struct RJArgs {
  int nr, jmax, L, kin, kout;
  double dt, cev, cet, ceb;           // explicit (1 - implicit) fractions
  double coef_d_velo, coef_d_magne, coef_d_temp, coef_buo, coef_cor;
  double coef_temp;
  int use_ref_temp;
  double temp_icb_fld, temp_cmb_fld;  // l = 0 perturbation wall values
  BCW bc;
  // per-jj tables
  const int *jl, *jm;
  const double *g3, *g3rlm, *gl;
  // radial tables
  const double *r, *ar1, *ar2, *d1, *d2, *reft0, *reft1, *om;  // d1/d2: [3][nr]
};

struct Ctx {
  cb2_params p;
  int prec = 0;
  int device = 0;
  int L = 0, nth = 0, nph = 0, nr = 0, jmax = 0, nh = 0, NS = 0, kin = 0, kout = 0;
  cudaStream_t stream = nullptr;
  // host tables
  std::vector<int> h_jl, h_jm;          // per jj
  std::vector<int> h_perm;              // jj -> j = l(l+1)+m
  std::vector<int> h_moff;              // offset of block (m, +) for m = 0..L
  std::vector<size_t> h_poff;           // offset of order m in the P tables
  std::vector<double> h_r, h_colat, h_wgt;
  BCW bc{};
  double cev = 0, cet = 0, ceb = 0, temp_icb_fld = 0, temp_cmb_fld = 0;
  // device tables
  int *d_jl = nullptr, *d_jm = nullptr, *d_perm = nullptr, *d_moff = nullptr;
  double *d_g3 = nullptr, *d_g3rlm = nullptr, *d_gl = nullptr, *d_g6 = nullptr;
  double *d_g7 = nullptr, *d_g11 = nullptr, *d_g12 = nullptr;
  double *d_r = nullptr, *d_ar1 = nullptr, *d_ar2 = nullptr, *d_d1 = nullptr, *d_d2 = nullptr;
  double *d_reft0 = nullptr, *d_reft1 = nullptr, *d_om = nullptr;
  double *d_colat = nullptr, *d_wgt = nullptr, *d_asin = nullptr;
  size_t *d_poff = nullptr;
  double *d_Plt = nullptr, *d_dPlt = nullptr, *d_Ptl = nullptr, *d_dPtl = nullptr;
  int *d_jgi1 = nullptr, *d_jgi2 = nullptr, *d_jei1 = nullptr;
  double *d_sw = nullptr, *d_tw = nullptr;       // [6][jmax], [8][jmax]
  double *d_lu_vp = nullptr, *d_lu_vt = nullptr, *d_lu_bs = nullptr, *d_lu_bt = nullptr, *d_lu_t = nullptr;
  int *d_pv_vp = nullptr, *d_pv_vt = nullptr, *d_pv_bs = nullptr, *d_pv_bt = nullptr, *d_pv_t = nullptr;
  // implicit-solve blocks: int4 (sign, m0, l0, -) tiles of consecutive
  // degrees x orders, imp_slots of them
  int *d_imp_map = nullptr;
  int imp_slots = 0;
  // fused Crank-Nicolson step (cb2_cn.cu): the factors in its forms (one
  // allocation), int4 (field, m0, l0, -) block tiles, the kernel's view of
  // the factors (CnPack), its shared memory; cn_ready when usable
  double *d_cn_lu = nullptr;
  int4 *d_cn_tiles = nullptr;
  int cn_tiles = 0;
  void *cn_pack = nullptr;
  size_t cn_smem = 0;
  bool cn_ready = false;
  const char *cn_off_reason = "";   // why the fused kernel is unavailable ("" when it is)
  int *d_status = nullptr;               // device error word
  // budget of each wait inside the tensor-core pipelines (ns): 200 ms, or
  // CB2_PIPE_WAIT_NS from the environment at cb2_create (0: one try, so the
  // first wait that is not already complete runs out)
  unsigned long long pipe_wait_ns = 200ull * 1000 * 1000;
  double *d_tw_fft = nullptr;            // exp(-2 pi i e / nph), e = 0..nph-1
  float *d_tw_fft32 = nullptr;
  void *d_twp32 = nullptr;               // per-stage float2 twiddles of the compile-time FFT plans
  void *d_twf4 = nullptr;                // tables of the four-step products kernel (nphi = 3 (L + 1))
  void *d_twf4_64 = nullptr;             // the same in float64 (float64 four-step kernel)
  // state
  double *d_f = nullptr;                 // NSLOT * nr * jmax
  void *d_four = nullptr;                // F: nth*nr*13*NS (double or float)
  void *d_four2 = nullptr;               // G: nth*nr*12*NS
  double *d_ene = nullptr;               // energy partial sums
  double *h_stage = nullptr;             // pinned staging buffer
  size_t h_stage_bytes = 0;
  double *d_tmp = nullptr;               // nr*jmax scratch for host transfers
  double *d_host_state = nullptr;        // 20 slots for cb2_step_host_state
  // copy stream of cb2_step_restart_state (the restart history uploads
  // while the nonlinear terms of the state are computed) and its events:
  // state staged, history read by the step staged, all history staged
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ev[3] = {nullptr, nullptr, nullptr};
  // mixed-precision Legendre operands (split fp16) -- owned by cb2_legendre_mixed.cu
  void *mixed = nullptr;
  // learned subgrid closure attached to the step (cb2_closure.cu), or null
  void *closure = nullptr;
  // routine-level entry points (cb2_boundary.cu): device staging of the
  // caller's host buffers, a grid buffer and the index tables, grown on demand
  double *d_bnd_a = nullptr, *d_bnd_b = nullptr, *d_bnd_grid = nullptr;
  size_t bnd_a_bytes = 0, bnd_b_bytes = 0, bnd_grid_bytes = 0;
  int *d_bnd_tab = nullptr;
  size_t bnd_tab_bytes = 0;
  int istep = 0;
  bool started = false;
  // the nonlinear terms of the current state are not computed yet
  // (cb2_step_restart_state leaves them to the next call)
  bool terms_stale = false;
  bool timers = false;
  cudaEvent_t ev[64];
  double stage_ms[32] = {0};
  cudaGraphExec_t graph_exec = nullptr;
  int graph_nsteps = 0;
  // kernel variants chosen by the autotuner (cb2_autotune); defaults until tuned
  int tune[8] = {4, 2, 2, 384, 0, 0, 0, 0};
  // persistent Legendre kernels launch min(SMs, tiles / ws_tiles_per_cta)
  // CTAs: 1 = every SM; an ensemble raises it so small shells take a few
  // SMs each and run side by side
  int ws_tiles_per_cta = 1;

  size_t fsize() const { return (size_t)nr * jmax; }
  double *fld(int slot) { return d_f + (size_t)slot * fsize(); }
  RJArgs rj_args() const;
};

void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define CB2_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);  \
  } while (0)

// Raise (never lower) a kernel's dynamic shared-memory limit.  The limit is
// a property of the kernel in the whole process, shared by every context:
// lowering it for a small shell would make the launches of a larger shell
// created earlier fail.
template <typename K>
inline cudaError_t raise_smem_limit(K *kernel, size_t bytes) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// set-up (cb2_tables.cu)
int setup_tables(Ctx &c);
void free_tables(Ctx &c);
// Legendre fp64 (cb2_legendre_f64.cu)
void leg_bwd_f64(Ctx &c, int nvec, int nscal, const int *slots, double *four);
void leg_fwd_f64(Ctx &c, int nvec, int nscal, const double *four, const int *slots);
// FFT and grid products (cb2_fft.cu)
int fft_setup(Ctx &c);
template <typename T> void fft_products(Ctx &c, const T *four, T *four2);
template <typename T> void fft_backward_grid(Ctx &c, int ncomp, const T *four, double *grid);
template <typename T> void fft_forward_grid(Ctx &c, int ncomp, const double *grid, T *four);
// rj operators and solves (cb2_rj.cu)
void rj_explicit(Ctx &c, bool euler);
void rj_implicit(Ctx &c);
void rj_after_transform(Ctx &c);
void rj_start_derived(Ctx &c);
void rj_temp_total(Ctx &c, double sign);
int rj_energies(Ctx &c, double out[7]);
int rj_energies_scratch(Ctx &c, double *scratch, double out[7]);
int rj_energy_spectra(Ctx &c, double *out_l, double *out_m, double *out_lm);
// look up the static scratch of cb2_energies_static on a device (cb2_static_scratch.cu)
int static_scratch_setup(int device);
int rj_lu_factorise(Ctx &c);
// fused Crank-Nicolson step (cb2_cn.cu): set-up after rj_lu_factorise, and
// the step (explicit update, solves, derived fields) when c.cn_ready
int cn_setup(Ctx &c);
void cn_step(Ctx &c, bool euler);
void cn_free(Ctx &c);
// the Crank-Nicolson stage as the tuning selects it: cn_step, or
// rj_explicit + rj_implicit
void cn_stage(Ctx &c, bool euler);
// Fourier coefficients of the mixed-precision path, order-major so that one
// Legendre GEMM row is one contiguous element.  For nvec vectors + nscal
// scalars, at each (m, theta):
//   P block: nr * 2 (nvec + nscal) floats ordered (k, field, s): the r
//            component of each vector, then each scalar;
//   D block: nr * 4 nvec floats ordered (k, vector, {theta s=0, theta s=1,
//            phi s=0, phi s=1});
// s = 0 is the cos (order +m) coefficient, s = 1 the sin (order -m) one.
// P[m][theta][...] sits at `P`, D[m][theta][...] at `D`.
struct MLayout {
  float *P = nullptr, *D = nullptr;
  int nvec = 0, nscal = 0, nr = 0, nth = 0;
  __host__ __device__ int rpP() const { return 2 * (nvec + nscal); }
  __host__ __device__ int rpD() const { return 4 * nvec; }
  // per-(m, theta) block strides, rounded up to 4 floats (16 bytes) so TMA
  // boxes can start on any block
  __host__ __device__ size_t sP() const { return (((size_t)nr * rpP() + 3) / 4) * 4; }
  __host__ __device__ size_t sD() const { return (((size_t)nr * rpD() + 3) / 4) * 4; }
  // element of component c (vector v: 3v r, 3v+1 theta, 3v+2 phi; scalars
  // after the vectors) at (m, theta, k), order sign s
  __host__ __device__ float *at(int m, int th, int k, int c, int s) const {
    if (c < 3 * nvec) {
      const int v = c / 3, cc = c - 3 * v;
      if (cc == 0) return P + ((size_t)m * nth + th) * sP() + (size_t)k * rpP() + 2 * v + s;
      return D + ((size_t)m * nth + th) * sD() + (size_t)k * rpD() + 4 * v + 2 * (cc - 1) + s;
    }
    return P + ((size_t)m * nth + th) * sP() + (size_t)k * rpP() + 2 * (nvec + (c - 3 * nvec)) + s;
  }
};
// layout over a float buffer of at least mlayout_floats(c) floats (any
// nvec, nscal with 3 nvec + nscal <= 13)
MLayout mlayout(const Ctx &c, void *buf, int nvec, int nscal);
size_t mlayout_floats(const Ctx &c);

// mixed-precision Legendre (cb2_legendre_mixed.cu)
int mixed_setup(Ctx &c);
void mixed_free(Ctx &c);
// slots: first rj slot of each vector, then of each scalar (out.nvec + out.nscal)
int leg_bwd_mixed(Ctx &c, const int *slots, const MLayout &out);
// rowmax_ready: the FFT kernel that wrote `in` also wrote the partial row
// maxima of mixed_fwd_pmax (fft_products_m returned true)
int leg_fwd_mixed(Ctx &c, const MLayout &in, const int *slots, bool rowmax_ready = false);
// the two halves of each: the kernels before the GEMM (spectra packing; row
// scales) and the tensor-core GEMM itself
int leg_bwd_pack(Ctx &c, const int *slots, const MLayout &out);
int leg_bwd_gemm(Ctx &c, const MLayout &out);
void leg_fwd_rowmax(Ctx &c, const MLayout &in, bool rowmax_ready);
int leg_fwd_gemm(Ctx &c, const MLayout &in, const int *slots);
// one persistent GEMM launch per transform over the tiles of several
// mixed-precision shells (an ensemble): the backward transform of each
// shell's d_four (bnvec vectors, bnscal scalars) and the forward transform
// of its d_four2 into fslots; the buffers and slots are fixed at set-up
struct MultiLeg;
int multi_leg_setup(const std::vector<Ctx *> &shells, int bnvec, int bnscal, const int *fslots, int fnvec, int fnscal,
                    MultiLeg **out);
void multi_leg_bwd(const MultiLeg *m, cudaStream_t st);
void multi_leg_fwd(const MultiLeg *m, cudaStream_t st);
void multi_leg_free(MultiLeg *m);
// buffer for the partial forward row maxima of a four-step FFT kernel
// ([theta][(L+1)/16][elements], nullptr when the shape has none) and the
// Gauss weights in float32
float *mixed_fwd_pmax(Ctx &c);
const float *mixed_weights32(Ctx &c);
// FFT and products of the mixed path (cb2_fft.cu), float32, order-major layouts
// returns true when it wrote the partial row maxima into pmax (the
// four-step kernel; pmax may be nullptr)
bool fft_products_m(Ctx &c, const MLayout &in, const MLayout &out, float *pmax = nullptr);
void fft_backward_grid_m(Ctx &c, const MLayout &in, double *grid);
void fft_forward_grid_m(Ctx &c, const double *grid, const MLayout &out);

// autotuned kernel variants (Ctx::tune)
enum Tune {
  TUNE_BWD_KT = 0,       // float64 backward Legendre: 1 tensor cores (mma f64); CUDA cores with 2 or 4 radial levels per block
  TUNE_FWD_KT = 1,       // float64 forward Legendre: CUDA cores with 1 or 2 radial levels per block; 3 tensor cores (mma f64)
  TUNE_PACK_KC = 2,      // mixed backward pack: radial levels per block (1, 2, 4)
  TUNE_FFT_THREADS = 3,  // mixed FFT + products: threads per row block; 384 = the four-step kernel
                         // (nphi = 3 (L + 1)), 128 / 256 / 512 = the Stockham kernel
  TUNE_CN = 4,           // 1: explicit update, solves and derived fields in one kernel
                         // (k_cn_step); 0: the separate kernels; -1: the one kernel
                         // cannot take this context's factors (fixed)
  TUNE_N = 5
};
// one time step (explicit, implicit, nonlinear); advances istep (cb2_api.cu)
int step_once(Ctx &c);
// the same step of a mixed-precision context without its two Legendre
// GEMMs, in three phases: 0 (solves, Coriolis, backward packing), then the
// backward GEMM, 1 (FFT + products, forward row scales), then the forward
// GEMM, 2 (after the transform); phase 0 advances istep
int step_phase(Ctx &c, int phase);
// the multi-shell Legendre GEMM launches of step_phase's shells
int step_gemms_setup(const std::vector<Ctx *> &shells, MultiLeg **out);
// learned closure (cb2_closure.cu): adds its tendency to the nonlinear terms
int closure_apply(Ctx &c);
void closure_free(Ctx &c);

// bits of the device status word d_status
constexpr int CB2_STATUS_SINGULAR = 1;        // zero pivot in an LU factorisation
constexpr int CB2_STATUS_PIPE_TIMEOUT = 2;    // a tensor-core pipeline wait ran out
// reads d_status (synchronises the stream); CB2_ERR_TIMEOUT after a pipeline timeout
int check_status(Ctx &c);

constexpr int kThreads = 256;
inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace cb2

struct cb2_ctx : public cb2::Ctx {};
