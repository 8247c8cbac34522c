// cb2_rj.cu -- (r, l, m) space of the time step on the GPU, float64:
// Adams-Bashforth / Euler explicit update, pivoted banded LU factorisation
// and Crank-Nicolson radial solves per (l, m), radial derivatives, curl /
// divergence of the transformed forces, Coriolis term by Gaunt couplings,
// and the volume mean square energies.
//
// Reference routines restated here (MHD_src/sph_MHD unless noted):
//   cal_momentum_eq_explicit.f90, cal_vorticity_terms_adams.f90,
//   cal_explicit_terms.f90, cal_diff_adv_src_explicit.f90 (explicit terms);
//   cal_sol_sph_fluid_crank.f90 (solves), const_r_mat_4_vector_sph.f90,
//   const_r_mat_4_scalar_sph.f90, set_radial_mat_sph.f90,
//   set_sph_scalar_mat_bc.f90, set_sph_magne_mat_bc.f90 (operators),
//   SOLVER_src/direct_solver/m_ludcmp_3band.f90, m_ludcmp_band.f90,
//   lubksb_357band_mul.f90, mat_product_3band_mul.f90 (LU);
//   cal_sph_exp_rotation.f90, cal_sph_exp_diffusion.f90, set_sph_exp_rigid_*.f90,
//   cal_sph_exp_nod_*_ins.f90, cal_sph_exp_fixed_scalar.f90 (rj operators);
//   sum_coriolis_terms_rlm.f90 (Coriolis); PARALLEL_src/SPH_SHELL_src/
//   cal_rms_by_sph_spectr.f90 + sum_sph_rms_data.f90 (energies).
#include <cmath>
#include <cstdio>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

RJArgs Ctx::rj_args() const {
  RJArgs a;
  a.nr = nr; a.jmax = jmax; a.L = L; a.kin = kin; a.kout = kout;
  a.dt = p.dt; a.cev = cev; a.cet = cet; a.ceb = ceb;
  a.coef_d_velo = p.coef_d_velo; a.coef_d_magne = p.coef_d_magne; a.coef_d_temp = p.coef_d_temp;
  a.coef_buo = p.coef_buo; a.coef_cor = p.coef_cor; a.coef_temp = p.coef_temp;
  a.use_ref_temp = p.use_ref_temp;
  a.temp_icb_fld = temp_icb_fld; a.temp_cmb_fld = temp_cmb_fld;
  a.bc = bc;
  a.jl = d_jl; a.jm = d_jm; a.g3 = d_g3; a.g3rlm = d_g3rlm; a.gl = d_gl;
  a.r = d_r; a.ar1 = d_ar1; a.ar2 = d_ar2; a.d1 = d_d1; a.d2 = d_d2;
  a.reft0 = d_reft0; a.reft1 = d_reft1; a.om = d_om;
  return a;
}

// ---------------------------------------------------------------------------
// banded LU (column-major band storage lu[(col-1)*nb + band-1], 1-based)
#define M3(a, b, c) (a)[((c) - 1) * 3 + ((b) - 1)]
#define M5(a, b, c) (a)[((c) - 1) * 5 + ((b) - 1)]
#define M9(a, b, c) (a)[((c) - 1) * 9 + ((b) - 1)]

__device__ static int d_ludcmp_3band(int n, const double *A, double *lu, int *piv, double *vwk,
                                     int *idx) {
  const double TINY = 1.0e-30;
  for (int i = 0; i < 5 * n; i++) lu[i] = 0.0;
  M5(lu, 3, 1) = M3(A, 2, 1);
  M5(lu, 4, 1) = M3(A, 3, 1);
  for (int j = 2; j <= n - 1; j++) {
    M5(lu, 2, j) = M3(A, 1, j); M5(lu, 3, j) = M3(A, 2, j); M5(lu, 4, j) = M3(A, 3, j);
  }
  M5(lu, 2, n) = M3(A, 1, n);
  M5(lu, 3, n) = M3(A, 2, n);
  for (int i = 1; i <= n; i++) {
    double am = fabs(M5(lu, 3, i));
    if (i < n) am = fmax(am, fabs(M5(lu, 2, i + 1)));
    if (i > 1) am = fmax(am, fabs(M5(lu, 4, i - 1)));
    if (!(am > 0.0) || !isfinite(am)) return 1;   // zero row, or an entry that is not finite
    vwk[i] = 1.0 / am;
    idx[i] = i;
  }
  for (int j = 1; j <= n; j++) {
    if (j == 2) {
      M5(lu, 3, j) = M5(lu, 3, j) - M5(lu, 4, j - 1) * M5(lu, 2, j);
    } else if (j > 2) {
      M5(lu, 2, j) = M5(lu, 2, j) - M5(lu, 4, j - 2) * M5(lu, 1, j);
      M5(lu, 3, j) = M5(lu, 3, j) - M5(lu, 5, j - 2) * M5(lu, 1, j) - M5(lu, 4, j - 1) * M5(lu, 2, j);
    }
    piv[j - 1] = j;
    if (j < n) {
      double am = vwk[j] * fabs(M5(lu, 3, j));
      if (j > 1) M5(lu, 4, j) = M5(lu, 4, j) - M5(lu, 5, j - 1) * M5(lu, 2, j);
      double dum = vwk[j + 1] * fabs(M5(lu, 4, j));
      if (dum >= am && j <= idx[j]) {
        int k = idx[j + 1]; idx[j + 1] = idx[j]; idx[j] = k;
        piv[j - 1] = j + 1;
        int kst = max(j - 1, 1), ked = min(j + 2, n);
        for (k = kst; k <= ked; k++) {
          double t = M5(lu, j + 4 - k, k);
          M5(lu, j + 4 - k, k) = M5(lu, j + 3 - k, k);
          M5(lu, j + 3 - k, k) = t;
        }
        vwk[j + 1] = vwk[j];
      }
    }
    if (M5(lu, 3, n) == 0.0) M5(lu, 3, n) = TINY;
    double dum = 1.0 / M5(lu, 3, j);
    if (j < n) M5(lu, 4, j) = M5(lu, 4, j) * dum;
  }
  return 0;
}

// general band LU, 5 bands; swaps that would reach outside the 9 stored
// bands only exchange zeros and are skipped
__device__ static int d_ludcmp_band5(int n, const double *A, double *lu, int *piv, double *vv,
                                     int *idx) {
  const double TINY = 1.0e-30;
  const int nb1 = 2, nb2 = 4;
  for (int i = 1; i <= n; i++) {
    int jst = max(i - nb1, 1), jed = min(i + nb1, n);
    double am = fabs(M5(A, i - jst + nb1 + 1, jst));
    for (int j = jst + 1; j <= jed; j++) am = fmax(am, fabs(M5(A, i - j + nb1 + 1, j)));
    if (!(am > 0.0) || !isfinite(am)) return 1;   // zero row, or an entry that is not finite
    vv[i] = 1.0 / am;
    idx[i] = i;
  }
  for (int i = 0; i < 9 * n; i++) lu[i] = 0.0;
  for (int i = 1; i <= n; i++) {
    int jst = max(i - nb1, 1), jed = min(i + nb1, n);
    for (int j = jst; j <= jed; j++) M9(lu, i - j + nb2 + 1, j) = M5(A, i - j + nb1 + 1, j);
  }
  for (int j = 1; j <= n; j++) {
    int ist = max(j - nb2, 1), ied = min(j + nb1, n);
    for (int i = ist; i <= j - 1; i++) {
      int l = i - j + nb2 + 1;
      for (int k = ist; k <= i - 1; k++)
        M9(lu, l, j) = M9(lu, l, j) - M9(lu, i - k + nb2 + 1, k) * M9(lu, k - j + nb2 + 1, j);
    }
    double am = 0.0;
    int imax = j;
    for (int i = j; i <= ied; i++) {
      int l = i - j + nb2 + 1, kst = max(i - nb2, 1);
      for (int k = kst; k <= j - 1; k++)
        M9(lu, l, j) = M9(lu, l, j) - M9(lu, i - k + nb2 + 1, k) * M9(lu, k - j + nb2 + 1, j);
      double dum = vv[i] * fabs(M9(lu, l, j));
      if (dum >= am && i <= idx[j] + nb1) { imax = i; am = dum; }
    }
    if (j != imax) {
      int k = idx[imax]; idx[imax] = idx[j]; idx[j] = k;
      int kst = max(j - nb2, 1), ked = min(imax + nb2, n);
      for (k = kst; k <= ked; k++) {
        int m1 = j - k + nb2 + 1, m2 = imax - k + nb2 + 1;
        if (m1 < 1 || m2 < 1 || m1 > 9 || m2 > 9) continue;
        double t = M9(lu, m2, k);
        M9(lu, m2, k) = M9(lu, m1, k);
        M9(lu, m1, k) = t;
      }
      vv[imax] = vv[j];
    }
    piv[j - 1] = imax;
    if (M9(lu, nb2 + 1, j) == 0.0) M9(lu, nb2 + 1, j) = TINY;
    if (j != n) {
      double dum = 1.0 / M9(lu, nb2 + 1, j);
      int ie = min(j + nb2, n);
      for (int i = j + 1; i <= ie; i++) M9(lu, i - j + nb2 + 1, j) = M9(lu, i - j + nb2 + 1, j) * dum;
    }
  }
  return 0;
}

__device__ static void add_vector_poisson(const RJArgs &a, int kin, int kout, double g3, double c,
                                          double *m3) {
  for (int k = kin + 1; k <= kout - 1; k++) {
    int kk = k - 1;
    M3(m3, 3, k - 1) = M3(m3, 3, k - 1) - c * a.d2[0 * a.nr + kk];
    M3(m3, 2, k) = M3(m3, 2, k) - c * (a.d2[1 * a.nr + kk] - g3 * a.ar2[kk]);
    M3(m3, 1, k + 1) = M3(m3, 1, k + 1) - c * a.d2[2 * a.nr + kk];
  }
}

__device__ static void add_scalar_poisson(const RJArgs &a, int kin, int kout, double g3, double c,
                                          double *m3) {
  for (int k = kin + 1; k <= kout - 1; k++) {
    int kk = k - 1;
    M3(m3, 3, k - 1) = M3(m3, 3, k - 1) - c * (a.d2[kk] + 2.0 * a.ar1[kk] * a.d1[kk]);
    M3(m3, 2, k) = M3(m3, 2, k)
        - c * (a.d2[a.nr + kk] + 2.0 * a.ar1[kk] * a.d1[a.nr + kk] - g3 * a.ar2[kk]);
    M3(m3, 1, k + 1) = M3(m3, 1, k + 1)
        - c * (a.d2[2 * a.nr + kk] + 2.0 * a.ar1[kk] * a.d1[2 * a.nr + kk]);
  }
}

__device__ static void unit_evo(int n, double *m3) {
  for (int i = 0; i < 3 * n; i++) m3[i] = 0.0;
  for (int k = 1; k <= n; k++) M3(m3, 2, k) = 1.0;
}

// one thread per degree l: build and factorise the five radial operators
__global__ void k_lu_factorise(RJArgs a, double cv, double cb, double ct, double *work,
                               double *lu_vp, int *pv_vp, double *lu_vt, int *pv_vt,
                               double *lu_bs, int *pv_bs, double *lu_bt, int *pv_bt,
                               double *lu_t, int *pv_t, int *status) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > a.L) return;
  int n = a.nr, kin = a.kin + 1, kout = a.kout + 1;
  double g3 = (double)(l * (l + 1)), gl = (double)l;
  const BCW &b = a.bc;
  double *vt = work + (size_t)l * (18 * n + 2 * (n + 1));
  double *wt = vt + 3 * n, *vs = wt + 3 * n, *vp = vs + 3 * n, *m3 = vp + 5 * n;
  double *vv = m3 + 3 * n;
  int *idx = (int *)(vv + (n + 1));
  int err = 0;
  // velocity (const_radial_mat_vort_2step), non-slip walls
  unit_evo(n, vt);
  unit_evo(n, wt);
  for (int i = 0; i < 3 * n; i++) vs[i] = 0.0;
  for (int k = 1; k <= n; k++) M3(vs, 2, k) = (k < kin || k > kout) ? 1.0 : 0.0;
  add_vector_poisson(a, kin, kout, g3, cv, vt);
  add_vector_poisson(a, kin, kout, g3, cv, wt);
  add_vector_poisson(a, kin, kout, g3, 1.0, vs);
  M3(wt, 2, kin) = M3(wt, 2, kin) - cv * (b.fix_dr_icb[1][3] - g3 * b.r_icb[2]);
  M3(wt, 1, kin + 1) = M3(wt, 1, kin + 1) - cv * b.fix_dr_icb[2][3];
  M3(vt, 2, kin) = 1.0;
  M3(vt, 1, kin + 1) = 0.0;
  M3(vs, 2, kin) = M3(vs, 2, kin) - 1.0 * (b.fix_dr_icb[1][3] - g3 * b.r_icb[2]);
  M3(vs, 1, kin + 1) = M3(vs, 1, kin + 1) - 1.0 * b.fix_dr_icb[2][3];
  M3(wt, 3, kout - 1) = M3(wt, 3, kout - 1) - cv * b.fix_dr_cmb[0][3];
  M3(wt, 2, kout) = M3(wt, 2, kout) - cv * (b.fix_dr_cmb[1][3] - g3 * b.r_cmb[2]);
  M3(vt, 3, kout - 1) = 0.0;
  M3(vt, 2, kout) = 1.0;
  M3(vs, 3, kout - 1) = M3(vs, 3, kout - 1) - 1.0 * b.fix_dr_cmb[0][3];
  M3(vs, 2, kout) = M3(vs, 2, kout) - 1.0 * (b.fix_dr_cmb[1][3] - g3 * b.r_cmb[2]);
  // product wt * vs (mat_product_3band_mul.f90)
  for (int i = 0; i < 5 * n; i++) vp[i] = 0.0;
  for (int k = 1; k < kin; k++) M5(vp, 3, k) = 1.0;
  for (int k = kout + 1; k <= n; k++) M5(vp, 3, k) = 1.0;
  for (int k = kin + 1; k <= kout - 1; k++) {
    if (k >= kin + 2) M5(vp, 5, k - 2) = M3(wt, 3, k - 1) * M3(vs, 3, k - 2);
    M5(vp, 4, k - 1) = M3(wt, 3, k - 1) * M3(vs, 2, k - 1) + M3(wt, 2, k) * M3(vs, 3, k - 1);
    M5(vp, 3, k) = M3(wt, 3, k - 1) * M3(vs, 1, k) + M3(wt, 2, k) * M3(vs, 2, k)
                 + M3(wt, 1, k + 1) * M3(vs, 3, k);
    M5(vp, 2, k + 1) = M3(wt, 2, k) * M3(vs, 1, k + 1) + M3(wt, 1, k + 1) * M3(vs, 2, k + 1);
    if (k <= kout - 2) M5(vp, 1, k + 2) = M3(wt, 1, k + 1) * M3(vs, 1, k + 2);
  }
  M5(vp, 3, kin) = 1.0;
  M5(vp, 2, kin + 1) = 0.0;
  M5(vp, 1, kin + 2) = 0.0;
  M5(vp, 5, kout - 2) = 0.0;
  M5(vp, 4, kout - 1) = 0.0;
  M5(vp, 3, kout) = 1.0;
  err |= d_ludcmp_band5(n, vp, lu_vp + (size_t)l * 9 * n, pv_vp + (size_t)l * n, vv, idx);
  err |= d_ludcmp_3band(n, vt, lu_vt + (size_t)l * 5 * n, pv_vt + (size_t)l * n, vv, idx);
  // magnetic field (const_radial_mat_4_magne_sph), insulating walls
  unit_evo(n, m3);
  add_vector_poisson(a, kin, kout, g3, cb, m3);
  M3(m3, 2, kin) = M3(m3, 2, kin)
      - cb * (b.fix_dr_icb[1][3] - g3 * b.r_icb[2] + (gl + 1.0) * b.r_icb[1] * b.fix_dr_icb[0][3]);
  M3(m3, 1, kin + 1) = M3(m3, 1, kin + 1) - cb * b.fix_dr_icb[2][3];
  M3(m3, 3, kout - 1) = M3(m3, 3, kout - 1) - cb * b.fix_dr_cmb[0][3];
  M3(m3, 2, kout) = M3(m3, 2, kout)
      - cb * (b.fix_dr_cmb[1][3] - g3 * b.r_cmb[2] - gl * b.r_cmb[1] * b.fix_dr_cmb[2][3]);
  err |= d_ludcmp_3band(n, m3, lu_bs + (size_t)l * 5 * n, pv_bs + (size_t)l * n, vv, idx);
  unit_evo(n, m3);
  add_vector_poisson(a, kin, kout, g3, cb, m3);
  M3(m3, 2, kin) = 1.0; M3(m3, 1, kin + 1) = 0.0;
  M3(m3, 3, kout - 1) = 0.0; M3(m3, 2, kout) = 1.0;
  err |= d_ludcmp_3band(n, m3, lu_bt + (size_t)l * 5 * n, pv_bt + (size_t)l * n, vv, idx);
  // temperature (const_radial_mat_4_scalar_sph), fixed values
  unit_evo(n, m3);
  add_scalar_poisson(a, kin, kout, g3, ct, m3);
  M3(m3, 2, kin) = 1.0; M3(m3, 1, kin + 1) = 0.0;
  M3(m3, 3, kout - 1) = 0.0; M3(m3, 2, kout) = 1.0;
  err |= d_ludcmp_3band(n, m3, lu_t + (size_t)l * 5 * n, pv_t + (size_t)l * n, vv, idx);
  if (err) atomicOr(status, 1);
}

// [l][row][entry] -> [row][entry][l]: the degrees side by side, so a warp of
// consecutive (l, m) columns of one order reads each band factor as one run
template <typename T>
__global__ void k_interleave_l(const T *src, T *dst, int nl, int w, int n) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x, tot = (size_t)nl * w * n;
  if (e >= tot) return;
  const int l = (int)(e % nl);
  const size_t re = e / nl;   // row * w + entry
  dst[e] = src[(size_t)l * w * n + re];
}

// implicit solve: blocks of IMP_LD degrees x IMP_MD orders; band factors of
// the block's degrees in shared memory
constexpr int IMP_LD = 8, IMP_MD = 16;
struct ImpLU {
  const double *lu[5];   // fields 0 (5-band), 1-4 (3-band), degree-interleaved
  const int *pv[5];
};
static size_t imp_smem(int n, int w) { return (size_t)n * w * IMP_LD * sizeof(double) + (size_t)n * IMP_LD * sizeof(int); }
struct Fields;
template <int W>
__global__ void k_implicit(RJArgs a, Fields F, ImpLU lup, const int *moff, const int4 *tiles);

int rj_lu_factorise(Ctx &c) {
  int n = c.nr, L = c.L;
  size_t per = (size_t)(18 * n + 2 * (n + 1));
  double *work = nullptr;
  CB2_CUDA(cudaMalloc(&work, per * (L + 1) * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_lu_vp, (size_t)(L + 1) * 9 * n * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_lu_vt, (size_t)(L + 1) * 5 * n * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_lu_bs, (size_t)(L + 1) * 5 * n * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_lu_bt, (size_t)(L + 1) * 5 * n * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_lu_t, (size_t)(L + 1) * 5 * n * sizeof(double)));
  for (int **pv : {&c.d_pv_vp, &c.d_pv_vt, &c.d_pv_bs, &c.d_pv_bt, &c.d_pv_t})
    CB2_CUDA(cudaMalloc(pv, (size_t)(L + 1) * n * sizeof(int)));
  CB2_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(int), c.stream));
  double dt = c.p.dt;
  k_lu_factorise<<<cdiv(L + 1, 64), 64, 0, c.stream>>>(
      c.rj_args(), c.p.coef_imp_v * c.p.coef_d_velo * dt, c.p.coef_imp_b * c.p.coef_d_magne * dt,
      c.p.coef_imp_t * c.p.coef_d_temp * dt, work, c.d_lu_vp, c.d_pv_vp, c.d_lu_vt, c.d_pv_vt,
      c.d_lu_bs, c.d_pv_bs, c.d_lu_bt, c.d_pv_bt, c.d_lu_t, c.d_pv_t, c.d_status);
  CB2_CUDA(cudaGetLastError());
  // degree-interleaved copies (through the work buffer, which is larger)
  {
    const int nl = L + 1;
    double *lus[5] = {c.d_lu_vp, c.d_lu_vt, c.d_lu_bs, c.d_lu_bt, c.d_lu_t};
    const int ws[5] = {9, 5, 5, 5, 5};
    for (int q = 0; q < 5; q++) {
      const size_t tot = (size_t)nl * ws[q] * n;
      k_interleave_l<double><<<cdiv((long)tot, 256), 256, 0, c.stream>>>(lus[q], work, nl, ws[q], n);
      CB2_CUDA(cudaMemcpyAsync(lus[q], work, tot * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    }
    int *pvs[5] = {c.d_pv_vp, c.d_pv_vt, c.d_pv_bs, c.d_pv_bt, c.d_pv_t};
    for (int q = 0; q < 5; q++) {
      const size_t tot = (size_t)nl * n;
      k_interleave_l<int><<<cdiv((long)tot, 256), 256, 0, c.stream>>>(pvs[q], (int *)work, nl, 1, n);
      CB2_CUDA(cudaMemcpyAsync(pvs[q], work, tot * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
    }
    CB2_CUDA(cudaGetLastError());
  }
  // implicit-solve blocks: (sign, m0, l0) tiles of IMP_LD degrees x IMP_MD
  // orders that hold at least one (l, m) of the sign
  {
    std::vector<int4> tl;
    for (int s = 0; s < 2; s++)
      for (int m0 = 0; m0 <= L; m0 += IMP_MD)
        for (int l0 = 0; l0 <= L; l0 += IMP_LD) {
          bool any = false;
          for (int q = 0; q < IMP_LD * IMP_MD && !any; q++) {
            const int l = l0 + q % IMP_LD, m = m0 + q / IMP_LD;
            any = l <= L && m <= l && !(s == 1 && m == 0);
          }
          if (any) tl.push_back(int4{s, m0, l0, 0});
        }
    c.imp_slots = (int)tl.size();
    CB2_CUDA(cudaMalloc(&c.d_imp_map, tl.size() * sizeof(int4)));
    CB2_CUDA(cudaMemcpyAsync(c.d_imp_map, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice, c.stream));
    if (imp_smem(n, 9) > 227 * 1024) {
      cudaStreamSynchronize(c.stream);
      cudaFree(work);
      set_error("too many radial levels for the implicit solve's shared-memory band factors");
      return CB2_ERR_ARG;
    }
    CB2_CUDA(raise_smem_limit(k_implicit<9>, imp_smem(n, 9)));
    CB2_CUDA(raise_smem_limit(k_implicit<5>, imp_smem(n, 5)));
  }
  int st = 0;
  CB2_CUDA(cudaMemcpyAsync(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  CB2_CUDA(cudaFree(work));
  if (st) {
    set_error("singular radial operator in the LU factorisation");
    return CB2_ERR_SINGULAR;
  }
  return 0;
}

// column access x(k) = base[(k-1)*stride], 1-based k
#define XC(i) x[(size_t)((i) - 1) * stride]

// Banded back substitutions of one column (lubksb_3band / lubksb_5band,
// SOLVER_src/direct_solver/lubksb_357band.f90:69-148, over the pivoted LU of
// m_ludcmp_3band.f90 / m_ludcmp_band.f90): row interchanges, L y = P b, then
// U x = y.  The recurrence is carried in registers and the column streamed
// in chunks of PF rows, the loads of the next chunk issued before the stores
// of this one, so a sweep waits on memory once per chunk rather than once
// per row; the band factors come from the block's shared-memory copy
// (k_implicit stages them) and the divisions by the diagonal of U become
// multiplications by its reciprocal (off the dependency chain).
// band factors in the degree-interleaved layout: lu = base + l, entry b of
// row c at lu[((c - 1) * width + b - 1) * nl]
#define M5I(a, b, c) (a)[(size_t)(((c) - 1) * 5 + ((b) - 1)) * nl]
#define M9I(a, b, c) (a)[(size_t)(((c) - 1) * 9 + ((b) - 1)) * nl]

constexpr int PF = 8;

__device__ static void d_pivots(int n, const int *piv, int nl, double *x, size_t stride) {
  for (int i = 1; i <= n; i++) {
    const int ll = piv[(size_t)(i - 1) * nl];
    if (ll != i) { const double s = XC(ll); XC(ll) = XC(i); XC(i) = s; }
  }
}

// rows i0 .. i0 + PF - 1 (ascending, dir = +1) or i0 .. i0 - PF + 1
// (descending, dir = -1) that lie in 1 .. n; others read as zero
template <int DIR>
__device__ __forceinline__ void d_chunk(const double *x, size_t stride, int n, int i0, double (&v)[PF]) {
#pragma unroll
  for (int u = 0; u < PF; u++) {
    const int q = i0 + DIR * u;
    v[u] = (q >= 1 && q <= n) ? XC(q) : 0.0;
  }
}

__device__ static void d_solve_3band(int n, const double *lu, const int *piv, int nl, double *x, size_t stride) {
  d_pivots(n, piv, nl, x, stride);
  // forward: L y = P b
  double ym2 = XC(1), ym1 = XC(2) - (M5I(lu, 4, 1)) * ym2;
  XC(2) = ym1;
  double buf[PF], nb[PF];
  d_chunk<1>(x, stride, n, 3, buf);
  for (int i0 = 3; i0 <= n; i0 += PF) {
    d_chunk<1>(x, stride, n, i0 + PF, nb);
#pragma unroll
    for (int u = 0; u < PF; u++) {
      const int i = i0 + u;
      if (i <= n) {
        const double y = buf[u] - (M5I(lu, 5, i - 2)) * ym2 - (M5I(lu, 4, i - 1)) * ym1;
        XC(i) = y;
        ym2 = ym1; ym1 = y;
      }
    }
#pragma unroll
    for (int u = 0; u < PF; u++) buf[u] = nb[u];
  }
  // backward: U x = y
  double xp2 = ym1 * (1.0 / (M5I(lu, 3, n)));
  const double yn1 = XC(n - 1);
  double xp1 = (yn1 - (M5I(lu, 2, n)) * xp2) * (1.0 / (M5I(lu, 3, n - 1)));
  d_chunk<-1>(x, stride, n, n - 2, buf);
  XC(n) = xp2;
  XC(n - 1) = xp1;
  for (int i0 = n - 2; i0 >= 1; i0 -= PF) {
    d_chunk<-1>(x, stride, n, i0 - PF, nb);
#pragma unroll
    for (int u = 0; u < PF; u++) {
      const int i = i0 - u;
      if (i >= 1) {
        const double v = (buf[u] - (M5I(lu, 2, i + 1)) * xp1 - (M5I(lu, 1, i + 2)) * xp2) *
                         (1.0 / (M5I(lu, 3, i)));
        XC(i) = v;
        xp2 = xp1; xp1 = v;
      }
    }
#pragma unroll
    for (int u = 0; u < PF; u++) buf[u] = nb[u];
  }
}

__device__ static void d_solve_5band(int n, const double *lu, const int *piv, int nl, double *x, size_t stride) {
  d_pivots(n, piv, nl, x, stride);
  // forward: L y = P b
  double y1 = XC(1);
  double y2 = XC(2) - (M9I(lu, 6, 1)) * y1;
  double y3 = XC(3) - (M9I(lu, 7, 1)) * y1 - (M9I(lu, 6, 2)) * y2;
  double y4 = XC(4) - (M9I(lu, 8, 1)) * y1 - (M9I(lu, 7, 2)) * y2 - (M9I(lu, 6, 3)) * y3;
  double buf[PF], nb[PF];
  d_chunk<1>(x, stride, n, 5, buf);
  XC(2) = y2; XC(3) = y3; XC(4) = y4;
  for (int i0 = 5; i0 <= n; i0 += PF) {
    d_chunk<1>(x, stride, n, i0 + PF, nb);
#pragma unroll
    for (int u = 0; u < PF; u++) {
      const int i = i0 + u;
      if (i <= n) {
        const double y = buf[u] - (M9I(lu, 9, i - 4)) * y1 - (M9I(lu, 8, i - 3)) * y2
                       - (M9I(lu, 7, i - 2)) * y3 - (M9I(lu, 6, i - 1)) * y4;
        XC(i) = y;
        y1 = y2; y2 = y3; y3 = y4; y4 = y;
      }
    }
#pragma unroll
    for (int u = 0; u < PF; u++) buf[u] = nb[u];
  }
  // backward: U x = y (y4 = y(n))
  const double b1 = XC(n - 1), b2 = XC(n - 2), b3 = XC(n - 3);
  const double x0 = y4 * (1.0 / (M9I(lu, 5, n)));
  const double xm1 = (b1 - (M9I(lu, 4, n)) * x0) * (1.0 / (M9I(lu, 5, n - 1)));
  const double xm2 = (b2 - (M9I(lu, 4, n - 1)) * xm1 - (M9I(lu, 3, n)) * x0) *
                     (1.0 / (M9I(lu, 5, n - 2)));
  const double xm3 = (b3 - (M9I(lu, 4, n - 2)) * xm2 - (M9I(lu, 3, n - 1)) * xm1
                      - (M9I(lu, 2, n)) * x0) * (1.0 / (M9I(lu, 5, n - 3)));
  d_chunk<-1>(x, stride, n, n - 4, buf);
  XC(n) = x0; XC(n - 1) = xm1; XC(n - 2) = xm2; XC(n - 3) = xm3;
  double p1 = xm3, p2 = xm2, p3 = xm1, p4 = x0;   // x(i+1) .. x(i+4)
  for (int i0 = n - 4; i0 >= 1; i0 -= PF) {
    d_chunk<-1>(x, stride, n, i0 - PF, nb);
#pragma unroll
    for (int u = 0; u < PF; u++) {
      const int i = i0 - u;
      if (i >= 1) {
        const double v = (buf[u] - (M9I(lu, 4, i + 1)) * p1 - (M9I(lu, 3, i + 2)) * p2
                          - (M9I(lu, 2, i + 3)) * p3 - (M9I(lu, 1, i + 4)) * p4) *
                         (1.0 / (M9I(lu, 5, i)));
        XC(i) = v;
        p4 = p3; p3 = p2; p2 = p1; p1 = v;
      }
    }
#pragma unroll
    for (int u = 0; u < PF; u++) buf[u] = nb[u];
  }
}

// ---------------------------------------------------------------------------
struct Fields {
  double *f;
  size_t fs;
  __device__ double *operator()(int slot) const { return f + (size_t)slot * fs; }
};

// explicit update (Euler on the first step, Adams-Bashforth 2 after)
__global__ void k_explicit(RJArgs a, Fields F, int euler) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (jj >= a.jmax) return;
  const size_t idx = (size_t)k * a.jmax + jj;
  bool in_shell = (k >= a.kin && k <= a.kout);
  const double adam_0 = 3.0 / 2.0, adam_1 = -1.0 / 2.0, dt = a.dt;
  double *wS = F(VORT), *wT = F(VORT + 2), *dwS = F(WDIFF), *dwT = F(WDIFF + 2);
  double *fS = F(FORCES), *fT = F(FORCES + 2), *pS = F(PREMOM), *pT = F(PREMOM + 2);
  double *bS = F(MAGNE), *bT = F(MAGNE + 2), *dbS = F(BDIFF), *dbT = F(BDIFF + 2);
  double *iS = F(INDUCT), *iT = F(INDUCT + 2), *qS = F(PREUXB), *qT = F(PREUXB + 2);
  double *T = F(TEMP), *dT = F(TDIFF), *H = F(HADV), *pH = F(PREHEAT);
  if (euler) {
    if (in_shell) {
      wS[idx] = wS[idx] + dt * (a.cev * dwS[idx] + fS[idx]);
      wT[idx] = wT[idx] + dt * (a.cev * dwT[idx] + fT[idx]);
      T[idx] = T[idx] + dt * (a.cet * dT[idx] - H[idx]);
      pH[idx] = -H[idx];
    }
    bS[idx] = bS[idx] + dt * (a.ceb * dbS[idx] + iS[idx]);
    bT[idx] = bT[idx] + dt * (a.ceb * dbT[idx] + iT[idx]);
    pS[idx] = fS[idx]; pT[idx] = fT[idx];
    qS[idx] = iS[idx]; qT[idx] = iT[idx];
  } else {
    if (in_shell) {
      wS[idx] = wS[idx] + dt * (a.cev * dwS[idx] + adam_0 * fS[idx] + adam_1 * pS[idx]);
      wT[idx] = wT[idx] + dt * (a.cev * dwT[idx] + adam_0 * fT[idx] + adam_1 * pT[idx]);
      pS[idx] = fS[idx]; pT[idx] = fT[idx];
      T[idx] = T[idx] + dt * (a.cet * dT[idx] - adam_0 * H[idx] + adam_1 * pH[idx]);
      pH[idx] = -H[idx];
    }
    bS[idx] = bS[idx] + dt * (a.ceb * dbS[idx] + adam_0 * iS[idx] + adam_1 * qS[idx]);
    bT[idx] = bT[idx] + dt * (a.ceb * dbT[idx] + adam_0 * iT[idx] + adam_1 * qT[idx]);
    qS[idx] = iS[idx]; qT[idx] = iT[idx];
  }
}

__device__ inline double icb_fld(const RJArgs &a, int jj) { return jj == 0 ? a.temp_icb_fld : 0.0; }
__device__ inline double cmb_fld(const RJArgs &a, int jj) { return jj == 0 ? a.temp_cmb_fld : 0.0; }

// Crank-Nicolson solves: one thread per (field, (l, m) column).  A block
// holds IMP_LD consecutive degrees x IMP_MD orders of one sign; it first
// stages the band factors and pivots of its IMP_LD degrees in shared memory
// (interleaved by degree, loaded together), so every factor a thread needs in
// its sweeps is a shared-memory read.  W = 9: the 5-band poloidal velocity
// (field 0); W = 5: the 3-band systems (fields 1-4, blockIdx.y + 1).
template <int W>
__global__ void __launch_bounds__(IMP_LD * IMP_MD)
k_implicit(RJArgs a, Fields F, ImpLU lup, const int *moff, const int4 *tiles) {
  extern __shared__ double lus[];                                   // [n * W][IMP_LD]
  const int n = a.nr, nl = a.L + 1, tid = threadIdx.x;
  int *pvs = reinterpret_cast<int *>(lus + (size_t)n * W * IMP_LD);  // [n][IMP_LD]
  const int4 tl = tiles[blockIdx.x];                                // (sign, m0, l0, -)
  const int fld = (W == 9) ? 0 : 1 + blockIdx.y;
  const double *lug = lup.lu[fld];
  const int *pvg = lup.pv[fld];
  for (int e = tid; e < n * W * IMP_LD; e += IMP_LD * IMP_MD) {
    const int lo = e % IMP_LD, l = tl.z + lo;
    lus[e] = (l < nl) ? __ldg(lug + (size_t)(e / IMP_LD) * nl + l) : 1.0;
  }
  for (int e = tid; e < n * IMP_LD; e += IMP_LD * IMP_MD) {
    const int lo = e % IMP_LD, l = tl.z + lo, row = e / IMP_LD;
    pvs[e] = (l < nl) ? __ldg(pvg + (size_t)row * nl + l) : row + 1;
  }
  __syncthreads();
  const int lo = tid % IMP_LD, l = tl.z + lo, m = tl.y + tid / IMP_LD, sgn = tl.x;
  if (l >= nl || m > l || (sgn == 1 && m == 0)) return;
  const int jj = moff[m] + sgn * (nl - m) + (l - m);
  const double *lu = lus + lo;
  const int *pv = pvs + lo;
  const size_t st = a.jmax;
  if (fld < 2) {
    // velocity from vorticity: S <- tor(w), T <- pol(w); l = 0 removed; walls zero
    double *u = F(VELO + 2 * fld) + jj, *udS = F(VELO + 1) + jj;
    const double *w = F(VORT + 2 - 2 * fld) + jj;
    // PF levels per pass, loads before stores (w is only read here)
    for (int k0 = 0; k0 < n; k0 += PF) {
      double v[PF];
#pragma unroll
      for (int q = 0; q < PF; q++) {
        const int k = k0 + q;
        const bool wall = (k <= a.kin || k == a.kout);
        v[q] = (k < n && jj != 0 && !wall) ? __ldg(w + (size_t)k * st) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < PF; q++) {
        const int k = k0 + q;
        if (k < n) {
          u[(size_t)k * st] = v[q];
          if (fld == 0 && (k <= a.kin || k == a.kout)) udS[(size_t)k * st] = 0.0;
        }
      }
    }
    if constexpr (W == 9) d_solve_5band(n, lu, pv, IMP_LD, u, st);
    else d_solve_3band(n, lu, pv, IMP_LD, u, st);
  } else if constexpr (W == 5) {
    if (fld == 2) {
      // temperature with fixed wall values
      double *T = F(TEMP) + jj;
      for (int k = a.kout; k < n; k++) T[k * st] = cmb_fld(a, jj);
      for (int k = 0; k <= a.kin; k++) T[k * st] = icb_fld(a, jj);
      d_solve_3band(n, lu, pv, IMP_LD, T, st);
    } else if (fld == 3) {
      // poloidal magnetic field, insulating walls, l = 0 removed
      double *bS = F(MAGNE) + jj, *bdS = F(MAGNE + 1) + jj;
      if (jj == 0)
        for (int k = 0; k < n; k++) bS[k * st] = 0.0;
      bdS[a.kin * st] = (a.gl[jj] + 1.0) * a.bc.r_icb[1] * bS[a.kin * st];
      bdS[a.kout * st] = -a.gl[jj] * a.bc.r_cmb[1] * bS[a.kout * st];
      d_solve_3band(n, lu, pv, IMP_LD, bS, st);
    } else {
      // toroidal magnetic field, zero at the walls
      double *bT = F(MAGNE + 2) + jj;
      if (jj == 0)
        for (int k = 0; k < n; k++) bT[k * st] = 0.0;
      bT[a.kin * st] = 0.0;
      bT[a.kout * st] = 0.0;
      d_solve_3band(n, lu, pv, IMP_LD, bT, st);
    }
  }
}

__device__ inline double D1(const RJArgs &a, const double *f, int k, int jj) {
  size_t s = a.jmax;
  return a.d1[k] * f[(k - 1) * s + jj] + a.d1[a.nr + k] * f[k * s + jj]
       + a.d1[2 * a.nr + k] * f[(k + 1) * s + jj];
}
__device__ inline double D2(const RJArgs &a, const double *f, int k, int jj) {
  size_t s = a.jmax;
  return a.d2[k] * f[(k - 1) * s + jj] + a.d2[a.nr + k] * f[k * s + jj]
       + a.d2[2 * a.nr + k] * f[(k + 1) * s + jj];
}

// gradients, vorticity, current density and buoyancy of the new state
// (const_grad_vp_and_vorticity with non-slip walls, const_grad_bp_and_current
//  with insulating walls, cal_rot_buoyancy_sph_MHD).  Wall values of u and
// of the toroidal field are zero by the boundary conditions.
__global__ void k_derived_a(RJArgs a, Fields F) {
  // grid (jj blocks, radial level k): no division to find k and jj
  const int jj = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (jj >= a.jmax) return;
  const size_t idx = (size_t)k * a.jmax + jj;
  size_t s = a.jmax;
  const BCW &b = a.bc;
  double g3 = a.g3[jj], gl = a.gl[jj];
  int ki = a.kin, ko = a.kout;
  double *uS = F(VELO), *udS = F(VELO + 1), *uT = F(VELO + 2);
  double *wS = F(VORT), *wdS = F(VORT + 1), *wT = F(VORT + 2);
  double *bS = F(MAGNE), *bdS = F(MAGNE + 1), *bT = F(MAGNE + 2);
  double *cS = F(CURRENT), *cdS = F(CURRENT + 1), *cT = F(CURRENT + 2);
  auto US = [&](int q) { return (q <= ki || q >= ko) ? 0.0 : uS[q * s + jj]; };
  auto UT = [&](int q) { return (q <= ki || q >= ko) ? 0.0 : uT[q * s + jj]; };
  auto BT = [&](int q) { return (q == ki || q == ko) ? 0.0 : bT[q * s + jj]; };
  if (k <= ki) {
    uS[idx] = 0.0; udS[idx] = 0.0; uT[idx] = 0.0;
  }
  if (k == ki) {
    double d2s = b.fix_dr_icb[1][3] * US(ki) + b.fix_dr_icb[2][3] * US(ki + 1);
    double d1t = b.fix_fld_icb[0][2] * UT(ki) + b.fix_fld_icb[1][2] * UT(ki + 1)
               + b.fix_fld_icb[2][2] * UT(ki + 2);
    wS[idx] = UT(ki);
    wdS[idx] = d1t;
    wT[idx] = -(d2s - g3 * b.r_icb[2] * US(ki));
    double B0 = bS[idx], B1 = bS[idx + s];
    double d1s = (gl + 1.0) * b.r_icb[1] * B0;
    double d2b = ((gl + 1.0) * b.r_icb[1] * b.fix_dr_icb[0][3] + b.fix_dr_icb[1][3]) * B0
               + b.fix_dr_icb[2][3] * B1;
    double d1bt = b.fix_fld_icb[1][2] * BT(ki + 1) + b.fix_fld_icb[2][2] * BT(ki + 2);
    bdS[idx] = d1s; bT[idx] = 0.0;
    cS[idx] = 0.0; cdS[idx] = d1bt;
    cT[idx] = -(d2b - g3 * b.r_icb[2] * B0);
  } else if (k == ko) {
    uS[idx] = 0.0; udS[idx] = 0.0; uT[idx] = 0.0;
    double d2s = b.fix_dr_cmb[0][3] * US(ko - 1);
    double d1t = b.fix_fld_cmb[2][2] * UT(ko - 2) + b.fix_fld_cmb[1][2] * UT(ko - 1)
               + b.fix_fld_cmb[0][2] * UT(ko);
    wS[idx] = UT(ko);
    wdS[idx] = d1t;
    wT[idx] = -d2s;
    double B0 = bS[idx], Bm = bS[idx - s];
    double d1s = -gl * b.r_cmb[1] * B0;
    double d2b = b.fix_dr_cmb[0][3] * Bm + (b.fix_dr_cmb[1][3] - gl * b.r_cmb[1] * b.fix_dr_cmb[2][3]) * B0;
    double d1bt = b.fix_fld_cmb[2][2] * BT(ko - 2) + b.fix_fld_cmb[1][2] * BT(ko - 1);
    bdS[idx] = d1s; bT[idx] = 0.0;
    cS[idx] = 0.0; cdS[idx] = d1bt;
    cT[idx] = -(d2b - g3 * b.r_cmb[2] * B0);
  } else if (k > ki && k < ko) {
    double ar2 = a.ar2[k];
    double c0 = a.d1[k], c1 = a.d1[a.nr + k], c2 = a.d1[2 * a.nr + k];
    double e0 = a.d2[k], e1 = a.d2[a.nr + k], e2 = a.d2[2 * a.nr + k];
    double s0 = US(k - 1), s1 = US(k), s2 = US(k + 1);
    double t0 = UT(k - 1), t1 = UT(k), t2 = UT(k + 1);
    udS[idx] = c0 * s0 + c1 * s1 + c2 * s2;
    wS[idx] = t1;
    wdS[idx] = c0 * t0 + c1 * t1 + c2 * t2;
    wT[idx] = -(e0 * s0 + e1 * s1 + e2 * s2) + g3 * ar2 * s1;
    double B0 = bS[idx - s], B1 = bS[idx], B2 = bS[idx + s];
    double T0 = BT(k - 1), T1 = BT(k), T2 = BT(k + 1);
    bdS[idx] = c0 * B0 + c1 * B1 + c2 * B2;
    cS[idx] = T1;
    cdS[idx] = c0 * T0 + c1 * T1 + c2 * T2;
    cT[idx] = -(e0 * B0 + e1 * B1 + e2 * B2) + g3 * ar2 * B1;
  }
  if (k >= ki && k <= ko) F(ROTBUO + 2)[idx] = a.coef_buo * F(TEMP)[idx] * a.r[k];
}

// diffusion terms (const_sph_vorticirty_diffusion, const_sph_scalar_diffusion,
// const_sph_mag_diffuse_by_j); the wall values of T are the fixed values
__global__ void k_derived_b(RJArgs a, Fields F) {
  // grid (jj blocks, radial level k): no division to find k and jj
  const int jj = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (jj >= a.jmax) return;
  const size_t idx = (size_t)k * a.jmax + jj;
  size_t s = a.jmax;
  const BCW &b = a.bc;
  double g3 = a.g3[jj], gl = a.gl[jj];
  int ki = a.kin, ko = a.kout;
  const double cv = a.coef_d_velo, cb = a.coef_d_magne, ct = a.coef_d_temp;
  const double *wS = F(VORT), *wT = F(VORT + 2);
  double *dwS = F(WDIFF), *dwT = F(WDIFF + 2);
  const double *bS = F(MAGNE), *bT = F(MAGNE + 2), *cS = F(CURRENT), *cT = F(CURRENT + 2);
  double *dbS = F(BDIFF), *dbT = F(BDIFF + 2);
  double *T = F(TEMP), *dT = F(TDIFF);
  auto TT = [&](int q) {
    return (q == ki) ? icb_fld(a, jj) : (q == ko) ? cmb_fld(a, jj) : T[q * s + jj];
  };
  if (k == ki) {
    size_t i1 = idx + s, i2 = idx + 2 * s;
    double d2s = b.fix_fld_icb[0][3] * wS[idx] + b.fix_fld_icb[1][3] * wS[i1] + b.fix_fld_icb[2][3] * wS[i2];
    double d2t = b.fix_fld_icb[0][3] * wT[idx] + b.fix_fld_icb[1][3] * wT[i1] + b.fix_fld_icb[2][3] * wT[i2];
    dwS[idx] = cv * (d2s - g3 * b.r_icb[2] * wS[idx]);
    dwT[idx] = cv * (d2t - g3 * b.r_icb[2] * wT[idx]);
    double fb = icb_fld(a, jj);
    double d1t = b.fix_fld_icb[0][2] * fb + b.fix_fld_icb[1][2] * TT(ki + 1) + b.fix_fld_icb[2][2] * TT(ki + 2);
    double d2T = b.fix_fld_icb[0][3] * fb + b.fix_fld_icb[1][3] * TT(ki + 1) + b.fix_fld_icb[2][3] * TT(ki + 2);
    T[idx] = fb;
    dT[idx] = ct * (d2T + 2.0 * b.r_icb[1] * d1t - g3 * b.r_icb[2] * fb);
    double d2b = ((gl + 1.0) * b.r_icb[1] * b.fix_dr_icb[0][3] + b.fix_dr_icb[1][3]) * bS[idx]
               + b.fix_dr_icb[2][3] * bS[i1];
    double d2bt = b.fix_fld_icb[0][3] * bT[idx] + b.fix_fld_icb[1][3] * bT[i1] + b.fix_fld_icb[2][3] * bT[i2];
    dbS[idx] = cb * (d2b - g3 * b.r_icb[2] * bS[idx]);
    dbT[idx] = cb * (d2bt - g3 * b.r_icb[2] * bT[idx]);
  } else if (k == ko) {
    size_t i1 = idx - s, i2 = idx - 2 * s;
    double d2s = b.fix_fld_cmb[2][3] * wS[i2] + b.fix_fld_cmb[1][3] * wS[i1] + b.fix_fld_cmb[0][3] * wS[idx];
    double d2t = b.fix_fld_cmb[2][3] * wT[i2] + b.fix_fld_cmb[1][3] * wT[i1] + b.fix_fld_cmb[0][3] * wT[idx];
    dwS[idx] = cv * (d2s - g3 * b.r_cmb[2] * wS[idx]);
    dwT[idx] = cv * (d2t - g3 * b.r_cmb[2] * wT[idx]);
    double fb = cmb_fld(a, jj);
    double d1t = b.fix_fld_cmb[2][2] * TT(ko - 2) + b.fix_fld_cmb[1][2] * TT(ko - 1) + b.fix_fld_cmb[0][2] * fb;
    double d2T = b.fix_fld_cmb[2][3] * TT(ko - 2) + b.fix_fld_cmb[1][3] * TT(ko - 1) + b.fix_fld_cmb[0][3] * fb;
    T[idx] = fb;
    dT[idx] = ct * (d2T + 2.0 * b.r_cmb[1] * d1t - g3 * b.r_cmb[2] * fb);
    double d2b = b.fix_dr_cmb[0][3] * bS[i1]
               + (b.fix_dr_cmb[1][3] - gl * b.r_cmb[1] * b.fix_dr_cmb[2][3]) * bS[idx];
    double d2bt = b.fix_fld_cmb[2][3] * bT[i2] + b.fix_fld_cmb[1][3] * bT[i1] + b.fix_fld_cmb[0][3] * bT[idx];
    dbS[idx] = cb * (d2b - g3 * b.r_cmb[2] * bS[idx]);
    dbT[idx] = cb * (d2bt - g3 * b.r_cmb[2] * bT[idx]);
  } else if (k > ki && k < ko) {
    double ar1 = a.ar1[k], ar2 = a.ar2[k];
    dwS[idx] = cv * (D2(a, wS, k, jj) - g3 * ar2 * wS[idx]);
    dwT[idx] = cv * (D2(a, wT, k, jj) - g3 * ar2 * wT[idx]);
    double c0 = a.d1[k], c1 = a.d1[a.nr + k], c2 = a.d1[2 * a.nr + k];
    double e0 = a.d2[k], e1 = a.d2[a.nr + k], e2 = a.d2[2 * a.nr + k];
    double t0 = TT(k - 1), t1 = TT(k), t2 = TT(k + 1);
    dT[idx] = ct * ((e0 * t0 + e1 * t1 + e2 * t2) + 2.0 * ar1 * (c0 * t0 + c1 * t1 + c2 * t2)
                    - g3 * ar2 * t1);
    dbS[idx] = -cb * cT[idx];
    dbT[idx] = cb * (D2(a, cS, k, jj) - g3 * ar2 * cS[idx]);
  }
}

// Coriolis term (sum_rot_coriolis_rlm_10): one thread per (k, jj)
// The Coriolis term at (k, jj) in spectral space, rotation form
// (sum_rot_coriolis_rlm_10): Gaunt / Elsasser couplings of the velocity and
// vorticity at l +- 1; the poloidal (rc0) and toroidal (rc2) parts.  It is
// evaluated where the force sum consumes it (k_after_transform); nothing
// changes the state between the solve and that kernel.
struct CorTables {
  const int *jgi1, *jgi2, *jei1;
  const double *sw, *tw;   // [6][jmax], [8][jmax]
};

__device__ inline void coriolis_terms(const RJArgs &a, const Fields &F, const CorTables &ct, int jj, int k,
                                      double &rc0, double &rc2) {
  size_t base = (size_t)k * a.jmax, J = a.jmax;
  const double *vS = F(VELO), *vdS = F(VELO + 1), *wS = F(VORT), *wdS = F(VORT + 1), *wT = F(VORT + 2);
  const double *sw = ct.sw, *tw = ct.tw;
  size_t i11 = base + ct.jgi1[jj], i21 = base + ct.jgi2[jj], i12 = base + ct.jei1[jj];
  double a1 = a.ar1[k], o0 = a.om[k], o1 = a.om[a.nr + k], o2 = a.om[2 * a.nr + k];
  double d2vp_l1 = a1 * a1 * a.g3rlm[jj] * vS[i12] - wT[i12];
  double dwp1 = wdS[i11] - 2.0 * a1 * wS[i11];
  double dwp2 = wdS[i21] - 2.0 * a1 * wS[i21];
  double p = sw[0 * J + jj] * o0 * vdS[i11] + sw[1 * J + jj] * o0 * vdS[i21]
           + sw[4 * J + jj] * o0 * wS[i12] + sw[2 * J + jj] * o1 * vS[i11]
           + sw[3 * J + jj] * o1 * vS[i21];
  double t = tw[0 * J + jj] * o0 * d2vp_l1 - tw[2 * J + jj] * o2 * vS[i12]
           + tw[4 * J + jj] * o1 * wS[i11] + tw[5 * J + jj] * o1 * wS[i21]
           + tw[6 * J + jj] * o0 * dwp1 + tw[7 * J + jj] * o0 * dwp2;
  rc0 = -a.coef_cor * p * a1 * a1;
  rc2 = -a.coef_cor * t * a1 * a1;
}

// curl / divergence of the transformed forces and the force sum
// (const_sph_force_rot2, const_sph_rotation_uxb, const_sph_scalar_advect,
//  add_reftemp_advect_sph_MHD, set_MHD_terms_to_force)
__global__ void k_after_transform(RJArgs a, Fields F, CorTables ct) {
  // grid (jj blocks, radial level k): no division to find k and jj
  const int jj = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (jj >= a.jmax) return;
  const size_t idx = (size_t)k * a.jmax + jj;
  size_t s = a.jmax;
  const BCW &b = a.bc;
  double g3 = a.g3[jj], gl = a.gl[jj];
  int ki = a.kin, ko = a.kout;
  double rot[2][3];
  const int src[2] = {MADV, LOR};
  for (int q = 0; q < 2; q++) {
    const double *fS = F(src[q]), *fdS = F(src[q] + 1), *fT = F(src[q] + 2);
    if (k == ki) {
      double d2s = b.fix_dr_icb[1][3] * fS[idx] + b.fix_dr_icb[2][3] * fS[idx + s];
      double d1t = b.fix_fld_icb[0][2] * fT[idx] + b.fix_fld_icb[1][2] * fT[idx + s]
                 + b.fix_fld_icb[2][2] * fT[idx + 2 * s];
      rot[q][0] = fT[idx]; rot[q][1] = d1t; rot[q][2] = -(d2s - g3 * b.r_icb[2] * fS[idx]);
    } else if (k == ko) {
      double d2s = b.fix_dr_cmb[0][3] * fS[idx - s] + b.fix_dr_cmb[1][3] * fS[idx];
      double d1t = b.fix_fld_cmb[2][2] * fT[idx - 2 * s] + b.fix_fld_cmb[1][2] * fT[idx - s]
                 + b.fix_fld_cmb[0][2] * fT[idx];
      rot[q][0] = fT[idx]; rot[q][1] = d1t; rot[q][2] = -(d2s - g3 * b.r_cmb[2] * fS[idx]);
    } else if (k > ki && k < ko) {
      rot[q][0] = fT[idx];
      rot[q][1] = D1(a, fT, k, jj);
      rot[q][2] = -D1(a, fdS, k, jj) + g3 * a.ar2[k] * fS[idx];
    } else {
      rot[q][0] = rot[q][1] = rot[q][2] = 0.0;
    }
  }
  for (int c = 0; c < 3; c++) {
    F(ROTINERT + c)[idx] = rot[0][c];
    F(ROTLOR + c)[idx] = rot[1][c];
  }
  // induction
  {
    const double *fS = F(VPIND), *fdS = F(VPIND + 1), *fT = F(VPIND + 2);
    double r0, r1, r2;
    if (k == ki) { r0 = fT[idx]; r1 = (gl + 1.0) * b.r_icb[1] * fT[idx]; r2 = 0.0; }
    else if (k == ko) { r0 = fT[idx]; r1 = -gl * b.r_cmb[1] * fT[idx]; r2 = 0.0; }
    else if (k > ki && k < ko) {
      r0 = fT[idx]; r1 = D1(a, fT, k, jj); r2 = -D1(a, fdS, k, jj) + g3 * a.ar2[k] * fS[idx];
    } else { r0 = r1 = r2 = 0.0; }
    F(INDUCT)[idx] = r0; F(INDUCT + 1)[idx] = r1; F(INDUCT + 2)[idx] = r2;
  }
  // heat advection
  {
    const double *fS = F(HFLUX), *fdS = F(HFLUX + 1);
    double gm = fmax(g3, 0.5), h = 0.0;
    if (k == ki) {
      double d1s = b.fix_fld_icb[0][2] * icb_fld(a, jj) + b.fix_fld_icb[1][2] * fS[idx + s]
                 + b.fix_fld_icb[2][2] * fS[idx + 2 * s];
      h = (d1s - fdS[idx]) * gm * b.r_icb[2];
    } else if (k == ko) {
      double d1s = b.fix_fld_cmb[2][2] * fS[idx - 2 * s] + b.fix_fld_cmb[1][2] * fS[idx - s]
                 + b.fix_fld_cmb[0][2] * cmb_fld(a, jj);
      h = (d1s - fdS[idx]) * gm * b.r_cmb[2];
    } else if (k > ki && k < ko) {
      h = (D1(a, fS, k, jj) - fdS[idx]) * gm * a.ar2[k];
    }
    if (a.use_ref_temp && k >= ki && k <= ko)
      h = h + a.coef_temp * g3 * a.ar2[k] * a.reft1[k] * F(VELO)[idx];
    F(HADV)[idx] = h;
  }
  double rc0, rc2;
  coriolis_terms(a, F, ct, jj, k, rc0, rc2);
  F(FORCES)[idx] = -rot[0][0] + rc0 + rot[1][0];
  F(FORCES + 2)[idx] = -rot[0][2] + rc2 + rot[1][2] + F(ROTBUO + 2)[idx];
}

__global__ void k_temp_total(RJArgs a, Fields F, double sign) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nr) return;
  F(TEMP)[(size_t)k * a.jmax] += sign * a.reft0[k];
}

// energies: per (l, m) radial trapezoid of the mean-square spectra, then a
// deterministic reduction (cal_rms_each_vector_sph_spec, radial_int_by_trapezoid)
__global__ void k_energy_j(RJArgs a, Fields F, const double *g11, const double *g12, double *ej) {
  int jj = blockIdx.x * blockDim.x + threadIdx.x;
  if (jj >= a.jmax) return;
  size_t s = a.jmax;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  double prev[7];
  for (int k = a.kin; k <= a.kout; k++) {
    double cur[7];
    double a1 = a.ar1[k];
    for (int v = 0; v < 2; v++) {
      int sl = v ? MAGNE : VELO;
      double S = F(sl)[k * s + jj], dS = F(sl + 1)[k * s + jj], T = F(sl + 2)[k * s + jj];
      double p, t;
      if (jj == 0) { p = (0.5 * S) * (0.5 * S) * a1 * a1; t = 0.0; }
      else { p = g12[jj] * (a.g3[jj] * a1 * a1 * S * S + dS * dS); t = g12[jj] * T * T; }
      int o = v ? 4 : 0;
      cur[o + 0] = 0.5 * p; cur[o + 1] = 0.5 * t; cur[o + 2] = 0.5 * (p + t);
    }
    // total temperature: the l = 0 part carries the reference profile
    double tv = F(TEMP)[k * s + jj];
    if (jj == 0 && a.use_ref_temp) tv = tv + a.reft0[k];
    cur[3] = tv * tv * g11[jj] * a.r[k] * a.r[k];
    if (k > a.kin) {
      double h = 0.5 * (a.r[k] - a.r[k - 1]);
      for (int q = 0; q < 7; q++) acc[q] = acc[q] + h * (prev[q] + cur[q]);
    }
    for (int q = 0; q < 7; q++) prev[q] = cur[q];
  }
  for (int q = 0; q < 7; q++) ej[(size_t)q * a.jmax + jj] = acc[q];
}

__global__ void k_energy_reduce(int jmax, const double *ej, double *out) {
  __shared__ double sh[256];
  int q = blockIdx.x;
  double s = 0.0;
  for (int j = threadIdx.x; j < jmax; j += blockDim.x) s += ej[(size_t)q * jmax + j];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[q] = sh[0];
}

// ---------------------------------------------------------------------------
static Fields fields(Ctx &c) { return Fields{c.d_f, c.fsize()}; }

void rj_explicit(Ctx &c, bool euler) {
  k_explicit<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(c.rj_args(), fields(c), euler ? 1 : 0);
}

void rj_implicit(Ctx &c) {
  RJArgs a = c.rj_args();
  const ImpLU lup{{c.d_lu_vp, c.d_lu_vt, c.d_lu_t, c.d_lu_bs, c.d_lu_bt},
                  {c.d_pv_vp, c.d_pv_vt, c.d_pv_t, c.d_pv_bs, c.d_pv_bt}};
  const int4 *tiles = reinterpret_cast<const int4 *>(c.d_imp_map);
  k_implicit<9><<<c.imp_slots, IMP_LD * IMP_MD, imp_smem(c.nr, 9), c.stream>>>(a, fields(c), lup, c.d_moff, tiles);
  k_implicit<5><<<dim3(c.imp_slots, 4), IMP_LD * IMP_MD, imp_smem(c.nr, 5), c.stream>>>(a, fields(c), lup,
                                                                                        c.d_moff, tiles);
  k_derived_a<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(a, fields(c));
  k_derived_b<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(a, fields(c));
}

void rj_start_derived(Ctx &c) {
  RJArgs a = c.rj_args();
  k_derived_a<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(a, fields(c));
  k_derived_b<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(a, fields(c));
}

void rj_after_transform(Ctx &c) {
  const CorTables ct{c.d_jgi1, c.d_jgi2, c.d_jei1, c.d_sw, c.d_tw};
  k_after_transform<<<dim3(cdiv(c.jmax, kThreads), c.nr), kThreads, 0, c.stream>>>(c.rj_args(), fields(c), ct);
}

void rj_temp_total(Ctx &c, double sign) {
  if (!c.p.use_ref_temp) return;
  k_temp_total<<<cdiv(c.nr, 128), 128, 0, c.stream>>>(c.rj_args(), fields(c), sign);
}

int rj_energies(Ctx &c, double out[7]) {
  k_energy_j<<<cdiv(c.jmax, 128), 128, 0, c.stream>>>(c.rj_args(), fields(c), c.d_g11, c.d_g12,
                                                      c.d_ene);
  k_energy_reduce<<<7, 256, 0, c.stream>>>(c.jmax, c.d_ene, c.d_ene + 7 * (size_t)c.jmax);
  CB2_CUDA(cudaGetLastError());
  double s[7];
  CB2_CUDA(cudaMemcpyAsync(s, c.d_ene + 7 * (size_t)c.jmax, 7 * sizeof(double),
                           cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  double ri = c.h_r[c.kin], ro = c.h_r[c.kout];
  double avol = 3.0 / (ro * ro * ro - ri * ri * ri);
  for (int q = 0; q < 7; q++) out[q] = avol * s[q];
  for (int q = 0; q < 7; q++)
    if (!std::isfinite(out[q])) {
      set_error("non-finite value in the energy diagnostics");
      return CB2_ERR_NAN;
    }
  return 0;
}

// per-(l,m) radial integrals ej[q][jj] grouped by degree l (kind 0), order
// |m| (kind 1) and l - |m| (kind 2): one thread per (kind, q, group g) sums
// its modes in a fixed order (sum_sph_rms_data.f90 set_sum_table_4_sph_spectr,
// sum_sph_v_rms_by_degree)
__global__ void k_energy_group(int L, int jmax, const int *moff, const double *ej, double *out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y, kind = blockIdx.z;
  if (g > L) return;
  const double *e = ej + (size_t)q * jmax;
  double s = 0.0;
  if (kind == 0) {
    for (int m = 0; m <= g; m++) {
      s += e[moff[m] + (g - m)];
      if (m > 0) s += e[moff[m] + (L + 1 - m) + (g - m)];
    }
  } else if (kind == 1) {
    for (int l = g; l <= L; l++) {
      s += e[moff[g] + (l - g)];
      if (g > 0) s += e[moff[g] + (L + 1 - g) + (l - g)];
    }
  } else {
    for (int m = 0; m + g <= L; m++) {
      s += e[moff[m] + g];
      if (m > 0) s += e[moff[m] + (L + 1 - m) + g];
    }
  }
  out[((size_t)kind * 7 + q) * (L + 1) + g] = s;
}

int rj_energy_spectra(Ctx &c, double *out_l, double *out_m, double *out_lm) {
  k_energy_j<<<cdiv(c.jmax, 128), 128, 0, c.stream>>>(c.rj_args(), fields(c), c.d_g11, c.d_g12, c.d_ene);
  // the grouped sums go to the temporary slot array (3 x 7 x (L+1) << nr jmax)
  double *grp = c.d_tmp;
  k_energy_group<<<dim3(cdiv(c.L + 1, 128), 7, 3), 128, 0, c.stream>>>(c.L, c.jmax, c.d_moff, c.d_ene, grp);
  CB2_CUDA(cudaGetLastError());
  const size_t n = 7 * (size_t)(c.L + 1);
  std::vector<double> h(3 * n);
  CB2_CUDA(cudaMemcpyAsync(h.data(), grp, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  const double ri = c.h_r[c.kin], ro = c.h_r[c.kout];
  const double avol = 3.0 / (ro * ro * ro - ri * ri * ri);
  double *outs[3] = {out_l, out_m, out_lm};
  for (int kind = 0; kind < 3; kind++)
    for (size_t i = 0; i < n; i++) {
      const double v = avol * h[kind * n + i];
      if (!std::isfinite(v)) {
        set_error("non-finite value in the energy spectra");
        return CB2_ERR_NAN;
      }
      outs[kind][i] = v;
    }
  return 0;
}

// The same diagnostics with caller-provided device scratch of at least
// 7 * jmax + 7 doubles (per-(l,m) partial sums, then the 7 totals).  Every
// element the kernels read is written first in the same call, so the
// scratch needs no clearing.
int rj_energies_scratch(Ctx &c, double *scratch, double out[7]) {
  double *sums = scratch + 7 * (size_t)c.jmax;
  k_energy_j<<<cdiv(c.jmax, 128), 128, 0, c.stream>>>(c.rj_args(), fields(c), c.d_g11, c.d_g12, scratch);
  k_energy_reduce<<<7, 256, 0, c.stream>>>(c.jmax, scratch, sums);
  CB2_CUDA(cudaGetLastError());
  double s[7];
  CB2_CUDA(cudaMemcpyAsync(s, sums, 7 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  double ri = c.h_r[c.kin], ro = c.h_r[c.kout];
  double avol = 3.0 / (ro * ro * ro - ri * ri * ri);
  for (int q = 0; q < 7; q++) out[q] = avol * s[q];
  for (int q = 0; q < 7; q++)
    if (!std::isfinite(out[q])) {
      set_error("non-finite value in the energy diagnostics");
      return CB2_ERR_NAN;
    }
  return 0;
}

}  // namespace cb2
