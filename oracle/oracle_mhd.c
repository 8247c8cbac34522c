/*
 * oracle_mhd.c -- Crank-Nicolson / Adams-Bashforth time step in (r, l, m)
 * space of the CPU oracle (test infrastructure, see calypso_oracle.h).
 *
 * Boundary conditions restated here are the ones of the benchmark
 * configurations: non-slip walls (velocity), fixed temperature, insulating
 * magnetic boundaries at both the ICB and the CMB, the ICB at radial node 0
 * and the CMB at node nr-1.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

#define FLD(o, s) ((o)->f[(s)])
#define AT(o, k, j) ((size_t)(k) * (o)->jmax + (j))

/* ---------------------------------------------------------------------- */
/* banded LU with the reference's pivoting rules.  Bands are stored like
 * the Fortran arrays, column-major: lu[(col-1)*nb + (band-1)], 1-based
 * band and column indices (F/SOLVER_src/direct_solver/m_ludcmp_3band.f90,
 * m_ludcmp_band.f90, lubksb_357band_mul.f90). */
#define B3(a, b, c) (a)[((c) - 1) * 3 + ((b) - 1)]
#define L5(a, b, c) (a)[((c) - 1) * 5 + ((b) - 1)]
#define B5(a, b, c) (a)[((c) - 1) * 5 + ((b) - 1)]
#define L9(a, b, c) (a)[((c) - 1) * 9 + ((b) - 1)]

int calo_ludcmp_3band(int n, const double *band_a, double *lu, int *ipiv) {
  const double TINY = 1.0e-30;
  double *vwk = calloc(n + 1, sizeof(double));
  int *idx = calloc(n + 1, sizeof(int));
  for (int i = 0; i < 5 * n; i++) lu[i] = 0.0;
  L5(lu, 3, 1) = B3(band_a, 2, 1);
  L5(lu, 4, 1) = B3(band_a, 3, 1);
  for (int j = 2; j <= n - 1; j++) {
    L5(lu, 2, j) = B3(band_a, 1, j);
    L5(lu, 3, j) = B3(band_a, 2, j);
    L5(lu, 4, j) = B3(band_a, 3, j);
  }
  L5(lu, 2, n) = B3(band_a, 1, n);
  L5(lu, 3, n) = B3(band_a, 2, n);
  for (int i = 1; i <= n; i++) {
    double aamax = fabs(L5(lu, 3, i));
    if (i < n && fabs(L5(lu, 2, i + 1)) > aamax) aamax = fabs(L5(lu, 2, i + 1));
    if (i > 1 && fabs(L5(lu, 4, i - 1)) > aamax) aamax = fabs(L5(lu, 4, i - 1));
    if (aamax == 0.0) { free(vwk); free(idx); return 100; }
    vwk[i] = 1.0 / aamax;
    idx[i] = i;
  }
  for (int j = 1; j <= n; j++) {
    if (j == 2) {
      L5(lu, 3, j) = L5(lu, 3, j) - L5(lu, 4, j - 1) * L5(lu, 2, j);
    } else if (j > 2) {
      L5(lu, 2, j) = L5(lu, 2, j) - L5(lu, 4, j - 2) * L5(lu, 1, j);
      L5(lu, 3, j) = L5(lu, 3, j) - L5(lu, 5, j - 2) * L5(lu, 1, j)
                                  - L5(lu, 4, j - 1) * L5(lu, 2, j);
    }
    ipiv[j - 1] = j;
    if (j < n) {
      double aamax = vwk[j] * fabs(L5(lu, 3, j));
      if (j > 1) L5(lu, 4, j) = L5(lu, 4, j) - L5(lu, 5, j - 1) * L5(lu, 2, j);
      double dum = vwk[j + 1] * fabs(L5(lu, 4, j));
      if (dum >= aamax && j <= idx[j]) {
        int k = idx[j + 1];
        idx[j + 1] = idx[j];
        idx[j] = k;
        ipiv[j - 1] = j + 1;
        int kst = (j - 1 > 1) ? j - 1 : 1, ked = (j + 2 < n) ? j + 2 : n;
        for (k = kst; k <= ked; k++) {
          double t = L5(lu, j + 4 - k, k);
          L5(lu, j + 4 - k, k) = L5(lu, j + 3 - k, k);
          L5(lu, j + 3 - k, k) = t;
        }
        vwk[j + 1] = vwk[j];
      }
    }
    if (L5(lu, 3, n) == 0.0) L5(lu, 3, n) = TINY;
    double dum = 1.0 / L5(lu, 3, j);
    if (j < n) L5(lu, 4, j) = L5(lu, 4, j) * dum;
  }
  free(vwk);
  free(idx);
  return 0;
}

/* general banded LU for 5 bands (nb1 = 2, nb2 = 4) */
int calo_ludcmp_band5(int n, const double *band_a, double *lu_in, int *ipiv) {
  const double TINY = 1.0e-30;
  const int nb1 = 2, nb2 = 4;
  double *vv = calloc(n + 1, sizeof(double));
  int *idx = calloc(n + 1, sizeof(int));
  double *lu = lu_in;
  for (int i = 1; i <= n; i++) {
    int jst = (i - nb1 > 1) ? i - nb1 : 1, jed = (i + nb1 < n) ? i + nb1 : n;
    double aamax = fabs(B5(band_a, i - jst + nb1 + 1, jst));
    for (int j = jst + 1; j <= jed; j++) {
      double v = fabs(B5(band_a, i - j + nb1 + 1, j));
      if (v > aamax) aamax = v;
    }
    if (aamax == 0.0) { free(vv); free(idx); return 100; }
    vv[i] = 1.0 / aamax;
    idx[i] = i;
  }
  for (int i = 0; i < 9 * n; i++) lu[i] = 0.0;
  for (int i = 1; i <= n; i++) {
    int jst = (i - nb1 > 1) ? i - nb1 : 1, jed = (i + nb1 < n) ? i + nb1 : n;
    for (int j = jst; j <= jed; j++)
      L9(lu, i - j + nb2 + 1, j) = B5(band_a, i - j + nb1 + 1, j);
  }
  for (int j = 1; j <= n; j++) {
    int ist = (j - nb2 > 1) ? j - nb2 : 1, ied = (j + nb1 < n) ? j + nb1 : n;
    for (int i = ist; i <= j - 1; i++) {
      int l = i - j + nb2 + 1;
      for (int k = ist; k <= i - 1; k++)
        L9(lu, l, j) = L9(lu, l, j) - L9(lu, i - k + nb2 + 1, k) * L9(lu, k - j + nb2 + 1, j);
    }
    double aamax = 0.0;
    int imax = j;
    for (int i = j; i <= ied; i++) {
      int l = i - j + nb2 + 1;
      int kst = (i - nb2 > 1) ? i - nb2 : 1;
      for (int k = kst; k <= j - 1; k++)
        L9(lu, l, j) = L9(lu, l, j) - L9(lu, i - k + nb2 + 1, k) * L9(lu, k - j + nb2 + 1, j);
      double dum = vv[i] * fabs(L9(lu, l, j));
      if (dum >= aamax && i <= idx[j] + nb1) { imax = i; aamax = dum; }
    }
    if (j != imax) {
      int k = idx[imax];
      idx[imax] = idx[j];
      idx[j] = k;
      int kst = (j - nb2 > 1) ? j - nb2 : 1, ked = (imax + nb2 < n) ? imax + nb2 : n;
      for (k = kst; k <= ked; k++) {
        int m1 = j - k + nb2 + 1, m2 = imax - k + nb2 + 1;
        long i1 = (long)(k - 1) * 9 + (m1 - 1), i2 = (long)(k - 1) * 9 + (m2 - 1);
        if (i1 < 0 || i2 < 0 || i1 >= 9L * n || i2 >= 9L * n) continue;
        double t = lu[i2];
        lu[i2] = lu[i1];
        lu[i1] = t;
      }
      vv[imax] = vv[j];
    }
    ipiv[j - 1] = imax;
    if (L9(lu, nb2 + 1, j) == 0.0) L9(lu, nb2 + 1, j) = TINY;
    if (j != n) {
      double dum = 1.0 / L9(lu, nb2 + 1, j);
      int ie = (j + nb2 < n) ? j + nb2 : n;
      for (int i = j + 1; i <= ie; i++) L9(lu, i - j + nb2 + 1, j) = L9(lu, i - j + nb2 + 1, j) * dum;
    }
  }
  free(vv);
  free(idx);
  return 0;
}

void calo_lubksb_3band(int n, const double *lu, const int *ipiv, double *x) {
  /* x is 1-based in the formulas below: X(i) = x[i-1] */
#define X(i) x[(i) - 1]
  for (int i = 1; i <= n; i++) {
    int ll = ipiv[i - 1];
    double s = X(ll);
    X(ll) = X(i);
    X(i) = s;
  }
  X(2) = X(2) - L5(lu, 4, 1) * X(1);
  for (int i = 3; i <= n; i++)
    X(i) = X(i) - L5(lu, 5, i - 2) * X(i - 2) - L5(lu, 4, i - 1) * X(i - 1);
  X(n) = X(n) / L5(lu, 3, n);
  X(n - 1) = (X(n - 1) - L5(lu, 2, n) * X(n)) / L5(lu, 3, n - 1);
  for (int i = n - 2; i >= 1; i--)
    X(i) = (X(i) - L5(lu, 2, i + 1) * X(i + 1) - L5(lu, 1, i + 2) * X(i + 2)) / L5(lu, 3, i);
}

void calo_lubksb_5band(int n, const double *lu, const int *ipiv, double *x) {
  for (int i = 1; i <= n; i++) {
    int ll = ipiv[i - 1];
    double s = X(ll);
    X(ll) = X(i);
    X(i) = s;
  }
  X(2) = X(2) - L9(lu, 6, 1) * X(1);
  X(3) = X(3) - L9(lu, 7, 1) * X(1) - L9(lu, 6, 2) * X(2);
  X(4) = X(4) - L9(lu, 8, 1) * X(1) - L9(lu, 7, 2) * X(2) - L9(lu, 6, 3) * X(3);
  for (int i = 5; i <= n; i++)
    X(i) = X(i) - L9(lu, 9, i - 4) * X(i - 4) - L9(lu, 8, i - 3) * X(i - 3)
                - L9(lu, 7, i - 2) * X(i - 2) - L9(lu, 6, i - 1) * X(i - 1);
  X(n) = X(n) / L9(lu, 5, n);
  X(n - 1) = (X(n - 1) - L9(lu, 4, n) * X(n)) / L9(lu, 5, n - 1);
  X(n - 2) = (X(n - 2) - L9(lu, 4, n - 1) * X(n - 1) - L9(lu, 3, n) * X(n)) / L9(lu, 5, n - 2);
  X(n - 3) = (X(n - 3) - L9(lu, 4, n - 2) * X(n - 2) - L9(lu, 3, n - 1) * X(n - 1)
              - L9(lu, 2, n) * X(n)) / L9(lu, 5, n - 3);
  for (int i = n - 4; i >= 1; i--)
    X(i) = (X(i) - L9(lu, 4, i + 1) * X(i + 1) - L9(lu, 3, i + 2) * X(i + 2)
            - L9(lu, 2, i + 3) * X(i + 3) - L9(lu, 1, i + 4) * X(i + 4)) / L9(lu, 5, i);
#undef X
}

/* ---------------------------------------------------------------------- */
/* radial operator matrices, per degree l (F/MHD_src/sph_MHD/
 * const_r_mat_4_vector_sph.f90, const_r_mat_4_scalar_sph.f90,
 * set_radial_mat_sph.f90, set_sph_scalar_mat_bc.f90, set_sph_magne_mat_bc.f90,
 * F/SOLVER_src/direct_solver/mat_product_3band_mul.f90) */
static void unit_time_evo(int n, double *m3) {
  for (int i = 0; i < 3 * n; i++) m3[i] = 0.0;
  for (int k = 1; k <= n; k++) B3(m3, 2, k) = 1.0;
}

static void unit_poisson(int n, int kin, int kout, double *m3) {
  for (int i = 0; i < 3 * n; i++) m3[i] = 0.0;
  for (int k = 1; k <= n; k++) B3(m3, 2, k) = (k < kin || k > kout) ? 1.0 : 0.0;
}

/* kin/kout 1-based in the matrix helpers */
static void add_vector_poisson(const cal_oracle *o, int kin, int kout, double g3,
                               double c, double *m3) {
  for (int k = kin + 1; k <= kout - 1; k++) {
    int kk = k - 1;
    B3(m3, 3, k - 1) = B3(m3, 3, k - 1) - c * o->d2[0][kk];
    B3(m3, 2, k) = B3(m3, 2, k) - c * (o->d2[1][kk] - g3 * o->ar2[kk]);
    B3(m3, 1, k + 1) = B3(m3, 1, k + 1) - c * o->d2[2][kk];
  }
}

static void add_scalar_poisson(const cal_oracle *o, int kin, int kout, double g3,
                               double c, double *m3) {
  for (int k = kin + 1; k <= kout - 1; k++) {
    int kk = k - 1;
    B3(m3, 3, k - 1) = B3(m3, 3, k - 1)
        - c * (o->d2[0][kk] + 2.0 * o->ar1[kk] * o->d1[0][kk]);
    B3(m3, 2, k) = B3(m3, 2, k)
        - c * (o->d2[1][kk] + 2.0 * o->ar1[kk] * o->d1[1][kk] - g3 * o->ar2[kk]);
    B3(m3, 1, k + 1) = B3(m3, 1, k + 1)
        - c * (o->d2[2][kk] + 2.0 * o->ar1[kk] * o->d1[2][kk]);
  }
}

static void fix_fld_icb(int kin, double *m3) { B3(m3, 2, kin) = 1.0; B3(m3, 1, kin + 1) = 0.0; }
static void fix_fld_cmb(int kout, double *m3) { B3(m3, 3, kout - 1) = 0.0; B3(m3, 2, kout) = 1.0; }

static void fix_flux_icb(const calo_bc *b, int kin, double g3, double c, double *m3) {
  B3(m3, 2, kin) = B3(m3, 2, kin) - c * (b->fix_dr_icb[1][3] - g3 * b->r_icb[2]);
  B3(m3, 1, kin + 1) = B3(m3, 1, kin + 1) - c * b->fix_dr_icb[2][3];
}

static void fix_flux_cmb(const calo_bc *b, int kout, double g3, double c, double *m3) {
  B3(m3, 3, kout - 1) = B3(m3, 3, kout - 1) - c * b->fix_dr_cmb[0][3];
  B3(m3, 2, kout) = B3(m3, 2, kout) - c * (b->fix_dr_cmb[1][3] - g3 * b->r_cmb[2]);
}

static void mat_product_3band(int n, int kst, int ked, const double *al,
                              const double *ar, double *ap) {
  for (int i = 0; i < 5 * n; i++) ap[i] = 0.0;
  for (int k = 1; k < kst; k++) B5(ap, 3, k) = 1.0;
  for (int k = ked + 1; k <= n; k++) B5(ap, 3, k) = 1.0;
  for (int k = kst + 2; k <= ked - 2; k++) {
    B5(ap, 5, k - 2) = B3(al, 3, k - 1) * B3(ar, 3, k - 2);
    B5(ap, 4, k - 1) = B3(al, 3, k - 1) * B3(ar, 2, k - 1) + B3(al, 2, k) * B3(ar, 3, k - 1);
    B5(ap, 3, k) = B3(al, 3, k - 1) * B3(ar, 1, k) + B3(al, 2, k) * B3(ar, 2, k)
                 + B3(al, 1, k + 1) * B3(ar, 3, k);
    B5(ap, 2, k + 1) = B3(al, 2, k) * B3(ar, 1, k + 1) + B3(al, 1, k + 1) * B3(ar, 2, k + 1);
    B5(ap, 1, k + 2) = B3(al, 1, k + 1) * B3(ar, 1, k + 2);
  }
  int k = kst;
  B5(ap, 3, k) = 1.0;
  B5(ap, 2, k + 1) = 0.0;
  B5(ap, 1, k + 2) = 0.0;
  k = kst + 1;
  B5(ap, 4, k - 1) = B3(al, 3, k - 1) * B3(ar, 2, k - 1) + B3(al, 2, k) * B3(ar, 3, k - 1);
  B5(ap, 3, k) = B3(al, 3, k - 1) * B3(ar, 1, k) + B3(al, 2, k) * B3(ar, 2, k)
               + B3(al, 1, k + 1) * B3(ar, 3, k);
  B5(ap, 2, k + 1) = B3(al, 2, k) * B3(ar, 1, k + 1) + B3(al, 1, k + 1) * B3(ar, 2, k + 1);
  B5(ap, 1, k + 2) = B3(al, 1, k + 1) * B3(ar, 1, k + 2);
  k = ked - 1;
  B5(ap, 5, k - 2) = B3(al, 3, k - 1) * B3(ar, 3, k - 2);
  B5(ap, 4, k - 1) = B3(al, 3, k - 1) * B3(ar, 2, k - 1) + B3(al, 2, k) * B3(ar, 3, k - 1);
  B5(ap, 3, k) = B3(al, 3, k - 1) * B3(ar, 1, k) + B3(al, 2, k) * B3(ar, 2, k)
               + B3(al, 1, k + 1) * B3(ar, 3, k);
  B5(ap, 2, k + 1) = B3(al, 2, k) * B3(ar, 1, k + 1) + B3(al, 1, k + 1) * B3(ar, 2, k + 1);
  k = ked;
  B5(ap, 5, k - 2) = 0.0;
  B5(ap, 4, k - 1) = 0.0;
  B5(ap, 3, k) = 1.0;
}

static void alloc_lu3(calo_lu3 *a, int n) {
  a->n = n;
  a->lu = calloc(5 * n, sizeof(double));
  a->piv = calloc(n, sizeof(int));
}

static void alloc_lu5(calo_lu5 *a, int n) {
  a->n = n;
  a->lu = calloc(9 * n, sizeof(double));
  a->piv = calloc(n, sizeof(int));
}

static int build_matrices(cal_oracle *o) {
  int n = o->nr, L = o->L, kin = o->kin + 1, kout = o->kout + 1;
  const calo_bc *b = &o->bc;
  double dt = o->p.dt;
  o->vp_lu = calloc(L + 1, sizeof(calo_lu5));
  o->vt_lu = calloc(L + 1, sizeof(calo_lu3));
  o->bs_lu = calloc(L + 1, sizeof(calo_lu3));
  o->bt_lu = calloc(L + 1, sizeof(calo_lu3));
  o->temp_lu = calloc(L + 1, sizeof(calo_lu3));
  int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
  for (int l = 0; l <= L; l++) {
    double g3 = (double)(l * (l + 1)), gl = (double)l;
    double *vt = malloc(3 * n * sizeof(double)), *wt = malloc(3 * n * sizeof(double));
    double *vs = malloc(3 * n * sizeof(double)), *vp = malloc(5 * n * sizeof(double));
    double *m3 = malloc(3 * n * sizeof(double));
    /* velocity (const_radial_mat_vort_2step), non-slip walls */
    double cv = o->p.coef_imp_v * o->p.coef_d_velo * dt;
    unit_time_evo(n, vt);
    unit_time_evo(n, wt);
    unit_poisson(n, kin, kout, vs);
    add_vector_poisson(o, kin, kout, g3, cv, vt);
    add_vector_poisson(o, kin, kout, g3, cv, wt);
    add_vector_poisson(o, kin, kout, g3, 1.0, vs);
    fix_flux_icb(b, kin, g3, cv, wt);
    fix_fld_icb(kin, vt);
    fix_flux_icb(b, kin, g3, 1.0, vs);
    fix_flux_cmb(b, kout, g3, cv, wt);
    fix_fld_cmb(kout, vt);
    fix_flux_cmb(b, kout, g3, 1.0, vs);
    mat_product_3band(n, kin, kout, wt, vs, vp);
    alloc_lu5(&o->vp_lu[l], n);
    alloc_lu3(&o->vt_lu[l], n);
    err |= calo_ludcmp_band5(n, vp, o->vp_lu[l].lu, o->vp_lu[l].piv);
    err |= calo_ludcmp_3band(n, vt, o->vt_lu[l].lu, o->vt_lu[l].piv);
    /* magnetic field (const_radial_mat_4_magne_sph), insulating walls */
    double cb = o->p.coef_imp_b * o->p.coef_d_magne * dt;
    unit_time_evo(n, m3);
    add_vector_poisson(o, kin, kout, g3, cb, m3);
    B3(m3, 2, kin) = B3(m3, 2, kin)
        - cb * (b->fix_dr_icb[1][3] - g3 * b->r_icb[2]
                + (gl + 1.0) * b->r_icb[1] * b->fix_dr_icb[0][3]);
    B3(m3, 1, kin + 1) = B3(m3, 1, kin + 1) - cb * b->fix_dr_icb[2][3];
    B3(m3, 3, kout - 1) = B3(m3, 3, kout - 1) - cb * b->fix_dr_cmb[0][3];
    B3(m3, 2, kout) = B3(m3, 2, kout)
        - cb * (b->fix_dr_cmb[1][3] - g3 * b->r_cmb[2] - gl * b->r_cmb[1] * b->fix_dr_cmb[2][3]);
    alloc_lu3(&o->bs_lu[l], n);
    err |= calo_ludcmp_3band(n, m3, o->bs_lu[l].lu, o->bs_lu[l].piv);
    unit_time_evo(n, m3);
    add_vector_poisson(o, kin, kout, g3, cb, m3);
    fix_fld_icb(kin, m3);
    fix_fld_cmb(kout, m3);
    alloc_lu3(&o->bt_lu[l], n);
    err |= calo_ludcmp_3band(n, m3, o->bt_lu[l].lu, o->bt_lu[l].piv);
    /* temperature (const_radial_mat_4_scalar_sph), fixed values */
    double ct = o->p.coef_imp_t * o->p.coef_d_temp * dt;
    unit_time_evo(n, m3);
    add_scalar_poisson(o, kin, kout, g3, ct, m3);
    fix_fld_icb(kin, m3);
    fix_fld_cmb(kout, m3);
    alloc_lu3(&o->temp_lu[l], n);
    err |= calo_ludcmp_3band(n, m3, o->temp_lu[l].lu, o->temp_lu[l].piv);
    free(vt); free(wt); free(vs); free(vp); free(m3);
  }
  return err;
}

/* solve all j of degree l for one field column (radial stride jmax) */
static void solve3_all(cal_oracle *o, calo_lu3 *lus, double *fld) {
  int n = o->nr;
#pragma omp parallel
  {
    double *x = malloc(n * sizeof(double));
#pragma omp for schedule(static)
    for (int j = 0; j < o->jmax; j++) {
      calo_lu3 *a = &lus[o->jl[j]];
      for (int k = 0; k < n; k++) x[k] = fld[AT(o, k, j)];
      calo_lubksb_3band(n, a->lu, a->piv, x);
      for (int k = 0; k < n; k++) fld[AT(o, k, j)] = x[k];
    }
    free(x);
  }
}

static void solve5_all(cal_oracle *o, calo_lu5 *lus, double *fld) {
  int n = o->nr;
#pragma omp parallel
  {
    double *x = malloc(n * sizeof(double));
#pragma omp for schedule(static)
    for (int j = 0; j < o->jmax; j++) {
      calo_lu5 *a = &lus[o->jl[j]];
      for (int k = 0; k < n; k++) x[k] = fld[AT(o, k, j)];
      calo_lubksb_5band(n, a->lu, a->piv, x);
      for (int k = 0; k < n; k++) fld[AT(o, k, j)] = x[k];
    }
    free(x);
  }
}

/* ---------------------------------------------------------------------- */
/* rj-space operators (F/MHD_src/sph_MHD/cal_sph_exp_rotation.f90,
 * cal_sph_exp_diffusion.f90, const_sph_rotation.f90, const_sph_diffusion.f90,
 * const_sph_radial_grad.f90, set_sph_exp_rigid_{ICB,CMB}.f90,
 * cal_sph_exp_nod_{icb,cmb}_ins.f90, cal_sph_exp_fixed_scalar.f90) */
static inline double D1(const cal_oracle *o, const double *f, int k, int j) {
  return o->d1[0][k] * f[AT(o, k - 1, j)] + o->d1[1][k] * f[AT(o, k, j)]
       + o->d1[2][k] * f[AT(o, k + 1, j)];
}
static inline double D2(const cal_oracle *o, const double *f, int k, int j) {
  return o->d2[0][k] * f[AT(o, k - 1, j)] + o->d2[1][k] * f[AT(o, k, j)]
       + o->d2[2][k] * f[AT(o, k + 1, j)];
}

/* velocity gradient + vorticity with non-slip walls
 * (const_grad_vp_and_vorticity; cal_sph_nod_icb_rigid_velo2/rot2,
 *  cal_sph_nod_cmb_rigid_v_and_w, cal_sph_diff_pol_and_rot2) */
static void grad_vp_and_vorticity(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double *uS = FLD(o, CALO_VELO), *udS = FLD(o, CALO_VELO + 1), *uT = FLD(o, CALO_VELO + 2);
  double *wS = FLD(o, CALO_VORT), *wdS = FLD(o, CALO_VORT + 1), *wT = FLD(o, CALO_VORT + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    for (int k = 0; k <= ki; k++) {
      uS[AT(o, k, j)] = 0.0; udS[AT(o, k, j)] = 0.0; uT[AT(o, k, j)] = 0.0 * b->r_icb[1];
    }
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d2s = b->fix_dr_icb[1][3] * uS[i0] + b->fix_dr_icb[2][3] * uS[i1];
    double d1t = b->fix_fld_icb[0][2] * uT[i0] + b->fix_fld_icb[1][2] * uT[i1]
               + b->fix_fld_icb[2][2] * uT[i2];
    wS[i0] = uT[i0];
    wdS[i0] = d1t;
    wT[i0] = -(d2s - o->g3[j] * b->r_icb[2] * uS[i0]);
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    uS[c0] = 0.0; udS[c0] = 0.0; uT[c0] = 0.0 * b->r_cmb[1];
    d2s = b->fix_dr_cmb[0][3] * uS[c1];
    d1t = b->fix_fld_cmb[2][2] * uT[c2] + b->fix_fld_cmb[1][2] * uT[c1]
        + b->fix_fld_cmb[0][2] * uT[c0];
    wS[c0] = uT[c0];
    wdS[c0] = d1t;
    wT[c0] = -d2s;
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      udS[a] = D1(o, uS, k, j);
      wS[a] = uT[a];
      wdS[a] = D1(o, uT, k, j);
      wT[a] = -D2(o, uS, k, j) + o->g3[j] * o->ar2[k] * uS[a];
    }
  }
}

/* magnetic gradient + current with insulating walls
 * (const_grad_bp_and_current; cal_sph_nod_{icb,cmb}_ins_b_and_j) */
static void grad_bp_and_current(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double *bS = FLD(o, CALO_MAGNE), *bdS = FLD(o, CALO_MAGNE + 1), *bT = FLD(o, CALO_MAGNE + 2);
  double *jS = FLD(o, CALO_CURRENT), *jdS = FLD(o, CALO_CURRENT + 1), *jT = FLD(o, CALO_CURRENT + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double gl = o->gl[j], g3 = o->g3[j];
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d1s = (gl + 1.0) * b->r_icb[1] * bS[i0];
    double d2s = ((gl + 1.0) * b->r_icb[1] * b->fix_dr_icb[0][3] + b->fix_dr_icb[1][3]) * bS[i0]
               + b->fix_dr_icb[2][3] * bS[i1];
    double d1t = b->fix_fld_icb[1][2] * bT[i1] + b->fix_fld_icb[2][2] * bT[i2];
    bdS[i0] = d1s;
    bT[i0] = 0.0;
    jS[i0] = 0.0;
    jdS[i0] = d1t;
    jT[i0] = -(d2s - g3 * b->r_icb[2] * bS[i0]);
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    d1s = -gl * b->r_cmb[1] * bS[c0];
    d2s = b->fix_dr_cmb[0][3] * bS[c1]
        + (b->fix_dr_cmb[1][3] - gl * b->r_cmb[1] * b->fix_dr_cmb[2][3]) * bS[c0];
    d1t = b->fix_fld_cmb[2][2] * bT[c2] + b->fix_fld_cmb[1][2] * bT[c1];
    bdS[c0] = d1s;
    bT[c0] = 0.0;
    jS[c0] = 0.0;
    jdS[c0] = d1t;
    jT[c0] = -(d2s - g3 * b->r_cmb[2] * bS[c0]);
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      bdS[a] = D1(o, bS, k, j);
      jS[a] = bT[a];
      jdS[a] = D1(o, bT, k, j);
      jT[a] = -D2(o, bS, k, j) + g3 * o->ar2[k] * bS[a];
    }
  }
}

/* vorticity diffusion (const_sph_vorticirty_diffusion with non-slip walls) */
static void vort_diffusion(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double c = o->p.coef_d_velo;
  double *wS = FLD(o, CALO_VORT), *wT = FLD(o, CALO_VORT + 2);
  double *dS = FLD(o, CALO_WDIFF), *ddS = FLD(o, CALO_WDIFF + 1), *dT = FLD(o, CALO_WDIFF + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j];
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      dS[a] = c * (D2(o, wS, k, j) - g3 * o->ar2[k] * wS[a]);
      dT[a] = c * (D2(o, wT, k, j) - g3 * o->ar2[k] * wT[a]);
    }
    for (int k = ki + 1; k <= ko - 1; k++) ddS[AT(o, k, j)] = D1(o, dS, k, j);
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d2s = b->fix_fld_icb[0][3] * wS[i0] + b->fix_fld_icb[1][3] * wS[i1]
               + b->fix_fld_icb[2][3] * wS[i2];
    double d2t = b->fix_fld_icb[0][3] * wT[i0] + b->fix_fld_icb[1][3] * wT[i1]
               + b->fix_fld_icb[2][3] * wT[i2];
    dS[i0] = c * (d2s - g3 * b->r_icb[2] * wS[i0]);
    dT[i0] = c * (d2t - g3 * b->r_icb[2] * wT[i0]);
    ddS[i0] = b->fix_fld_icb[0][2] * dS[i0] + b->fix_fld_icb[1][2] * dS[i1]
            + b->fix_fld_icb[2][2] * dS[i2];
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    d2s = b->fix_fld_cmb[2][3] * wS[c2] + b->fix_fld_cmb[1][3] * wS[c1]
        + b->fix_fld_cmb[0][3] * wS[c0];
    d2t = b->fix_fld_cmb[2][3] * wT[c2] + b->fix_fld_cmb[1][3] * wT[c1]
        + b->fix_fld_cmb[0][3] * wT[c0];
    dS[c0] = c * (d2s - g3 * b->r_cmb[2] * wS[c0]);
    dT[c0] = c * (d2t - g3 * b->r_cmb[2] * wT[c0]);
    ddS[c0] = b->fix_fld_cmb[2][2] * dS[c2] + b->fix_fld_cmb[1][2] * dS[c1]
            + b->fix_fld_cmb[0][2] * dS[c0];
  }
}

/* magnetic diffusion from the current (const_sph_mag_diffuse_by_j) */
static void mag_diffusion(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double c = o->p.coef_d_magne;
  double *bS = FLD(o, CALO_MAGNE), *bT = FLD(o, CALO_MAGNE + 2);
  double *jS = FLD(o, CALO_CURRENT), *jT = FLD(o, CALO_CURRENT + 2);
  double *dS = FLD(o, CALO_BDIFF), *ddS = FLD(o, CALO_BDIFF + 1), *dT = FLD(o, CALO_BDIFF + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j], gl = o->gl[j];
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      dS[a] = -c * jT[a];
      ddS[a] = -c * D1(o, jT, k, j);
      dT[a] = c * (D2(o, jS, k, j) - g3 * o->ar2[k] * jS[a]);
    }
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d2s = ((gl + 1.0) * b->r_icb[1] * b->fix_dr_icb[0][3] + b->fix_dr_icb[1][3]) * bS[i0]
               + b->fix_dr_icb[2][3] * bS[i1];
    double d2t = b->fix_fld_icb[0][3] * bT[i0] + b->fix_fld_icb[1][3] * bT[i1]
               + b->fix_fld_icb[2][3] * bT[i2];
    dS[i0] = c * (d2s - g3 * b->r_icb[2] * bS[i0]);
    dT[i0] = c * (d2t - g3 * b->r_icb[2] * bT[i0]);
    ddS[i0] = b->fix_fld_icb[0][2] * dS[i0] + b->fix_fld_icb[1][2] * dS[i1]
            + b->fix_fld_icb[2][2] * dS[i2];
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    d2s = b->fix_dr_cmb[0][3] * bS[c1]
        + (b->fix_dr_cmb[1][3] - gl * b->r_cmb[1] * b->fix_dr_cmb[2][3]) * bS[c0];
    d2t = b->fix_fld_cmb[2][3] * bT[c2] + b->fix_fld_cmb[1][3] * bT[c1]
        + b->fix_fld_cmb[0][3] * bT[c0];
    dS[c0] = c * (d2s - g3 * b->r_cmb[2] * bS[c0]);
    dT[c0] = c * (d2t - g3 * b->r_cmb[2] * bT[c0]);
    ddS[c0] = b->fix_fld_cmb[2][2] * dS[c2] + b->fix_fld_cmb[1][2] * dS[c1]
            + b->fix_fld_cmb[0][2] * dS[c0];
  }
}

static double icb_fld(const cal_oracle *o, int j) { return (j == 0) ? o->temp_icb_fld : 0.0; }
static double cmb_fld(const cal_oracle *o, int j) { return (j == 0) ? o->temp_cmb_fld : 0.0; }

/* thermal diffusion with fixed boundary values (const_sph_scalar_diffusion);
 * the boundary routines also reset T at the walls to the fixed values */
static void temp_diffusion(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double c = o->p.coef_d_temp;
  double *T = FLD(o, CALO_TEMP), *D = FLD(o, CALO_TDIFF);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j];
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      D[a] = c * (D2(o, T, k, j) + 2.0 * o->ar1[k] * D1(o, T, k, j) - g3 * o->ar2[k] * T[a]);
    }
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double fb = icb_fld(o, j);
    double d1t = b->fix_fld_icb[0][2] * fb + b->fix_fld_icb[1][2] * T[i1]
               + b->fix_fld_icb[2][2] * T[i2];
    double d2t = b->fix_fld_icb[0][3] * fb + b->fix_fld_icb[1][3] * T[i1]
               + b->fix_fld_icb[2][3] * T[i2];
    T[i0] = fb;
    D[i0] = c * (d2t + 2.0 * b->r_icb[1] * d1t - g3 * b->r_icb[2] * T[i0]);
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    fb = cmb_fld(o, j);
    d1t = b->fix_fld_cmb[2][2] * T[c2] + b->fix_fld_cmb[1][2] * T[c1] + b->fix_fld_cmb[0][2] * fb;
    d2t = b->fix_fld_cmb[2][3] * T[c2] + b->fix_fld_cmb[1][3] * T[c1] + b->fix_fld_cmb[0][3] * fb;
    T[c0] = fb;
    D[c0] = c * (d2t + 2.0 * b->r_cmb[1] * d1t - g3 * b->r_cmb[2] * T[c0]);
  }
}

/* buoyancy (cal_rot_buoyancy_sph_MHD): tor slot = c_buo T r */
static void rot_buoyancy(cal_oracle *o) {
  double *T = FLD(o, CALO_TEMP), *R = FLD(o, CALO_ROTBUO + 2);
#pragma omp parallel for schedule(static)
  for (int k = o->kin; k <= o->kout; k++)
    for (int j = 0; j < o->jmax; j++)
      R[AT(o, k, j)] = o->p.coef_buo * T[AT(o, k, j)] * o->r[k];
}

/* rotation of a forcing vector with non-slip-wall boundary rows
 * (const_sph_force_rot2: cal_sph_nod_{icb,cmb}_rigid_rot2 +
 *  cal_sph_nod_vect_w_div_rot2) */
static void force_rot(cal_oracle *o, int sf, int sr) {
  const calo_bc *b = &o->bc;
  double *fS = FLD(o, sf), *fdS = FLD(o, sf + 1), *fT = FLD(o, sf + 2);
  double *rS = FLD(o, sr), *rdS = FLD(o, sr + 1), *rT = FLD(o, sr + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j];
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d2s = b->fix_dr_icb[1][3] * fS[i0] + b->fix_dr_icb[2][3] * fS[i1];
    double d1t = b->fix_fld_icb[0][2] * fT[i0] + b->fix_fld_icb[1][2] * fT[i1]
               + b->fix_fld_icb[2][2] * fT[i2];
    rS[i0] = fT[i0];
    rdS[i0] = d1t;
    rT[i0] = -(d2s - g3 * b->r_icb[2] * fS[i0]);
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    d2s = b->fix_dr_cmb[0][3] * fS[c1] + b->fix_dr_cmb[1][3] * fS[c0];
    d1t = b->fix_fld_cmb[2][2] * fT[c2] + b->fix_fld_cmb[1][2] * fT[c1]
        + b->fix_fld_cmb[0][2] * fT[c0];
    rS[c0] = fT[c0];
    rdS[c0] = d1t;
    rT[c0] = -(d2s - g3 * b->r_cmb[2] * fS[c0]);
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      rS[a] = fT[a];
      rdS[a] = D1(o, fT, k, j);
      rT[a] = -D1(o, fdS, k, j) + g3 * o->ar2[k] * fS[a];
    }
  }
}

/* magnetic induction = rot(u x B) with insulating walls (const_sph_rotation_uxb) */
static void induction_rot(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double *fS = FLD(o, CALO_VPIND), *fdS = FLD(o, CALO_VPIND + 1), *fT = FLD(o, CALO_VPIND + 2);
  double *rS = FLD(o, CALO_INDUCT), *rdS = FLD(o, CALO_INDUCT + 1), *rT = FLD(o, CALO_INDUCT + 2);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j], gl = o->gl[j];
    size_t i0 = AT(o, ki, j), c0 = AT(o, ko, j);
    rS[i0] = fT[i0];
    rdS[i0] = (gl + 1.0) * b->r_icb[1] * fT[i0];
    rT[i0] = 0.0;
    rS[c0] = fT[c0];
    rdS[c0] = -gl * b->r_cmb[1] * fT[c0];
    rT[c0] = 0.0;
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      rS[a] = fT[a];
      rdS[a] = D1(o, fT, k, j);
      rT[a] = -D1(o, fdS, k, j) + g3 * o->ar2[k] * fS[a];
    }
  }
}

/* heat advection = div(u T) with fixed-temperature walls
 * (const_sph_scalar_advect, cal_sph_div_flux_4_fix_in/out) plus the
 * advection of the reference profile (add_reftemp_advect_sph_MHD) */
static void heat_advect(cal_oracle *o) {
  const calo_bc *b = &o->bc;
  double *fS = FLD(o, CALO_HFLUX), *fdS = FLD(o, CALO_HFLUX + 1);
  double *H = FLD(o, CALO_HADV), *uS = FLD(o, CALO_VELO);
  int ki = o->kin, ko = o->kout;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < o->jmax; j++) {
    double g3 = o->g3[j], gm = (g3 > 0.5) ? g3 : 0.5;
    for (int k = ki + 1; k <= ko - 1; k++) {
      size_t a = AT(o, k, j);
      H[a] = (D1(o, fS, k, j) - fdS[a]) * gm * o->ar2[k];
    }
    size_t i0 = AT(o, ki, j), i1 = AT(o, ki + 1, j), i2 = AT(o, ki + 2, j);
    double d1s = b->fix_fld_icb[0][2] * icb_fld(o, j) + b->fix_fld_icb[1][2] * fS[i1]
               + b->fix_fld_icb[2][2] * fS[i2];
    H[i0] = (d1s - fdS[i0]) * gm * b->r_icb[2];
    size_t c0 = AT(o, ko, j), c1 = AT(o, ko - 1, j), c2 = AT(o, ko - 2, j);
    d1s = b->fix_fld_cmb[2][2] * fS[c2] + b->fix_fld_cmb[1][2] * fS[c1]
        + b->fix_fld_cmb[0][2] * cmb_fld(o, j);
    H[c0] = (d1s - fdS[c0]) * gm * b->r_cmb[2];
    if (o->p.use_ref_temp) {
      for (int k = ki; k <= ko; k++) {
        size_t a = AT(o, k, j);
        H[a] = H[a] + o->p.coef_temp * g3 * o->ar2[k] * o->reft1[k] * uS[a];
      }
    }
  }
}

/* Coriolis term in spectral space (F/MHD_src/sph_MHD/sum_coriolis_terms_rlm.f90
 * sum_rot_coriolis_rlm_10) from the velocity and vorticity spectra */
static void coriolis(cal_oracle *o) {
  double *vS = FLD(o, CALO_VELO), *vdS = FLD(o, CALO_VELO + 1);
  double *wS = FLD(o, CALO_VORT), *wdS = FLD(o, CALO_VORT + 1), *wT = FLD(o, CALO_VORT + 2);
  double *cS = FLD(o, CALO_ROTCOR), *cdS = FLD(o, CALO_ROTCOR + 1), *cT = FLD(o, CALO_ROTCOR + 2);
  double cc = o->p.coef_cor;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < o->nr; k++) {
    double a1 = o->ar1[k], o0 = o->om[0][k], o1 = o->om[1][k], o2 = o->om[2][k];
    for (int j = 0; j < o->jmax; j++) {
      size_t i11 = AT(o, k, o->jgi1[j]), i21 = AT(o, k, o->jgi2[j]), i12 = AT(o, k, o->jei1[j]);
      double dvp1 = vdS[i11], dvp2 = vdS[i21], wp_l1 = wS[i12];
      double vp1 = vS[i11], vp2 = vS[i21];
      double d2vp_l1 = a1 * a1 * o->g3rlm[j] * vS[i12] - wT[i12];
      double vp_l1 = vS[i12];
      double wp1 = wS[i11], wp2 = wS[i21];
      double dwp1 = wdS[i11] - 2.0 * a1 * wS[i11];
      double dwp2 = wdS[i21] - 2.0 * a1 * wS[i21];
      double p = o->sw[0][j] * o0 * dvp1 + o->sw[1][j] * o0 * dvp2 + o->sw[4][j] * o0 * wp_l1
               + o->sw[2][j] * o1 * vp1 + o->sw[3][j] * o1 * vp2;
      double t = o->tw[0][j] * o0 * d2vp_l1 - o->tw[2][j] * o2 * vp_l1
               + o->tw[4][j] * o1 * wp1 + o->tw[5][j] * o1 * wp2
               + o->tw[6][j] * o0 * dwp1 + o->tw[7][j] * o0 * dwp2;
      size_t a = AT(o, k, j);
      cS[a] = -cc * p * a1 * a1;
      cdS[a] = 0.0;
      cT[a] = -cc * t * a1 * a1;
    }
  }
}

/* nonlinear: pseudo-spectral products, their rotation / divergence, the
 * Coriolis term and the force sum (F/MHD_src/sph_MHD/cal_nonlinear.f90) */
static void nonlinear(cal_oracle *o) {
  coriolis(o);
  calo_nonlinear_transforms(o);
  force_rot(o, CALO_MADV, CALO_ROTINERT);
  force_rot(o, CALO_LOR, CALO_ROTLOR);
  induction_rot(o);
  heat_advect(o);
  double *fS = FLD(o, CALO_FORCES), *fT = FLD(o, CALO_FORCES + 2);
  size_t n = (size_t)o->nr * o->jmax;
#pragma omp parallel for schedule(static)
  for (size_t a = 0; a < n; a++) {
    fS[a] = -FLD(o, CALO_ROTINERT)[a] + FLD(o, CALO_ROTCOR)[a] + FLD(o, CALO_ROTLOR)[a];
    fT[a] = -FLD(o, CALO_ROTINERT + 2)[a] + FLD(o, CALO_ROTCOR + 2)[a]
          + FLD(o, CALO_ROTLOR + 2)[a] + FLD(o, CALO_ROTBUO + 2)[a];
  }
}

static void delete_l0(cal_oracle *o, int s) {
  for (int k = 0; k < o->nr; k++) {
    FLD(o, s)[AT(o, k, 0)] = 0.0;
    FLD(o, s + 2)[AT(o, k, 0)] = 0.0;
  }
}

/* Crank-Nicolson solves (F/MHD_src/sph_MHD/cal_sol_sph_fluid_crank.f90) and
 * the derived fields of the new state (cal_sol_sph_MHD_crank.f90:44-101) */
static void implicit_solve(cal_oracle *o) {
  size_t n = (size_t)o->nr * o->jmax;
  double *uS = FLD(o, CALO_VELO), *udS = FLD(o, CALO_VELO + 1), *uT = FLD(o, CALO_VELO + 2);
  /* velocity from vorticity: S <- tor(w), T <- pol(w) */
  for (size_t a = 0; a < n; a++) {
    uS[a] = FLD(o, CALO_VORT + 2)[a];
    uT[a] = FLD(o, CALO_VORT)[a];
  }
  delete_l0(o, CALO_VELO);
  for (int j = 0; j < o->jmax; j++) {
    for (int k = 0; k <= o->kin; k++) {
      uS[AT(o, k, j)] = 0.0; udS[AT(o, k, j)] = 0.0; uT[AT(o, k, j)] = 0.0;
    }
    uS[AT(o, o->kout, j)] = 0.0; udS[AT(o, o->kout, j)] = 0.0; uT[AT(o, o->kout, j)] = 0.0;
  }
  solve5_all(o, o->vp_lu, uS);
  solve3_all(o, o->vt_lu, uT);
  grad_vp_and_vorticity(o);
  /* temperature with fixed boundary values */
  double *T = FLD(o, CALO_TEMP);
  for (int j = 0; j < o->jmax; j++) {
    for (int k = o->kout; k < o->nr; k++) T[AT(o, k, j)] = cmb_fld(o, j);
    for (int k = 0; k <= o->kin; k++) T[AT(o, k, j)] = icb_fld(o, j);
  }
  solve3_all(o, o->temp_lu, T);
  /* magnetic field with insulating boundaries */
  double *bS = FLD(o, CALO_MAGNE), *bdS = FLD(o, CALO_MAGNE + 1), *bT = FLD(o, CALO_MAGNE + 2);
  delete_l0(o, CALO_MAGNE);
  for (int j = 0; j < o->jmax; j++) {
    size_t i0 = AT(o, o->kin, j), c0 = AT(o, o->kout, j);
    bdS[i0] = (o->gl[j] + 1.0) * o->bc.r_icb[1] * bS[i0];
    bT[i0] = 0.0;
    bdS[c0] = -o->gl[j] * o->bc.r_cmb[1] * bS[c0];
    bT[c0] = 0.0;
  }
  solve3_all(o, o->bs_lu, bS);
  solve3_all(o, o->bt_lu, bT);
  grad_bp_and_current(o);
  vort_diffusion(o);
  rot_buoyancy(o);
  temp_diffusion(o);
  mag_diffusion(o);
}

/* explicit Euler (first step) or Adams-Bashforth 2 update
 * (cal_momentum_eq_explicit.f90, cal_vorticity_terms_adams.f90,
 *  cal_explicit_terms.f90, cal_diff_adv_src_explicit.f90) */
static void explicit_update(cal_oracle *o, int euler) {
  const double adam_0 = 3.0 / 2.0, adam_1 = -1.0 / 2.0, dt = o->p.dt;
  double cev = o->coef_exp_v, ceb = o->coef_exp_b, cet = o->coef_exp_t;
  size_t n = (size_t)o->nr * o->jmax;
  size_t ist = (size_t)o->kin * o->jmax, ied = (size_t)(o->kout + 1) * o->jmax;
  double *wS = FLD(o, CALO_VORT), *wT = FLD(o, CALO_VORT + 2);
  double *dwS = FLD(o, CALO_WDIFF), *dwT = FLD(o, CALO_WDIFF + 2);
  double *fS = FLD(o, CALO_FORCES), *fT = FLD(o, CALO_FORCES + 2);
  double *pS = FLD(o, CALO_PREMOM), *pT = FLD(o, CALO_PREMOM + 2);
  double *bS = FLD(o, CALO_MAGNE), *bT = FLD(o, CALO_MAGNE + 2);
  double *dbS = FLD(o, CALO_BDIFF), *dbT = FLD(o, CALO_BDIFF + 2);
  double *iS = FLD(o, CALO_INDUCT), *iT = FLD(o, CALO_INDUCT + 2);
  double *qS = FLD(o, CALO_PREUXB), *qT = FLD(o, CALO_PREUXB + 2);
  double *T = FLD(o, CALO_TEMP), *dT = FLD(o, CALO_TDIFF), *H = FLD(o, CALO_HADV);
  double *pH = FLD(o, CALO_PREHEAT);
  if (euler) {
    for (size_t a = ist; a < ied; a++) {
      wS[a] = wS[a] + dt * (cev * dwS[a] + fS[a]);
      wT[a] = wT[a] + dt * (cev * dwT[a] + fT[a]);
    }
    for (size_t a = ist; a < ied; a++) T[a] = T[a] + dt * (cet * dT[a] - H[a]);
    for (size_t a = 0; a < n; a++) {
      bS[a] = bS[a] + dt * (ceb * dbS[a] + iS[a]);
      bT[a] = bT[a] + dt * (ceb * dbT[a] + iT[a]);
    }
    for (size_t a = 0; a < n; a++) { pS[a] = fS[a]; pT[a] = fT[a]; }
    for (size_t a = ist; a < ied; a++) pH[a] = -H[a];
    for (size_t a = 0; a < n; a++) { qS[a] = iS[a]; qT[a] = iT[a]; }
  } else {
    for (size_t a = ist; a < ied; a++) {
      wS[a] = wS[a] + dt * (cev * dwS[a] + adam_0 * fS[a] + adam_1 * pS[a]);
      wT[a] = wT[a] + dt * (cev * dwT[a] + adam_0 * fT[a] + adam_1 * pT[a]);
      pS[a] = fS[a];
      pT[a] = fT[a];
    }
    for (size_t a = 0; a < n; a++) {
      bS[a] = bS[a] + dt * (ceb * dbS[a] + adam_0 * iS[a] + adam_1 * qS[a]);
      bT[a] = bT[a] + dt * (ceb * dbT[a] + adam_0 * iT[a] + adam_1 * qT[a]);
      qS[a] = iS[a];
      qT[a] = iT[a];
    }
    for (size_t a = ist; a < ied; a++) {
      T[a] = T[a] + dt * (cet * dT[a] - adam_0 * H[a] + adam_1 * pH[a]);
      pH[a] = -H[a];
    }
  }
}

/* volume mean square energies (F/PARALLEL_src/SPH_SHELL_src/
 * cal_rms_by_sph_spectr.f90, sum_sph_rms_data.f90, cal_ave_4_rms_vector_sph.f90,
 * F/SERIAL_src/SPH_SPECTR_src/radial_int_for_sph_spec.f90) */
static void rms_vector(const cal_oracle *o, int s, double out[3]) {
  int ki = o->kin, ko = o->kout, L = o->L;
  double *vl = calloc(3 * (L + 1), sizeof(double));
  double *f = malloc(o->nr * 3 * sizeof(double));
  for (int j = 0; j < o->jmax; j++) {
    for (int k = 0; k < o->nr; k++) {
      size_t a = AT(o, k, j);
      double S = FLD(o, s)[a], dS = FLD(o, s + 1)[a], T = FLD(o, s + 2)[a];
      double a1 = o->ar1[k];
      if (j == 0) {
        f[3 * k + 0] = (0.5 * S) * (0.5 * S) * a1 * a1;
        f[3 * k + 1] = 0.0;
      } else {
        f[3 * k + 0] = o->g12[j] * (o->g3[j] * a1 * a1 * S * S + dS * dS);
        f[3 * k + 1] = o->g12[j] * T * T;
      }
      f[3 * k + 2] = f[3 * k + 0] + f[3 * k + 1];
      for (int c = 0; c < 3; c++) f[3 * k + c] = 0.5 * f[3 * k + c];
    }
    for (int c = 0; c < 3; c++) {
      double fi = 0.0;
      for (int kr = ki; kr < ko; kr++)
        fi = fi + 0.5 * (o->r[kr + 1] - o->r[kr]) * (f[3 * kr + c] + f[3 * (kr + 1) + c]);
      vl[c * (L + 1) + o->jl[j]] += fi;
    }
  }
  double avol = 3.0 / (pow(o->r[ko], 3) - pow(o->r[ki], 3));
  for (int c = 0; c < 3; c++) {
    double t = vl[c * (L + 1) + 0];
    for (int l = 1; l <= L; l++) t = t + vl[c * (L + 1) + l];
    out[c] = avol * t;
  }
  free(vl);
  free(f);
}

static double rms_scalar(const cal_oracle *o, int s) {
  int ki = o->kin, ko = o->kout, L = o->L;
  double *vl = calloc(L + 1, sizeof(double));
  double *f = malloc(o->nr * sizeof(double));
  for (int j = 0; j < o->jmax; j++) {
    for (int k = 0; k < o->nr; k++) {
      double v = FLD(o, s)[AT(o, k, j)];
      f[k] = v * v * o->g11[j] * o->r[k] * o->r[k];
    }
    double fi = 0.0;
    for (int kr = ki; kr < ko; kr++) fi = fi + 0.5 * (o->r[kr + 1] - o->r[kr]) * (f[kr] + f[kr + 1]);
    vl[o->jl[j]] += fi;
  }
  double avol = 3.0 / (pow(o->r[ko], 3) - pow(o->r[ki], 3));
  double t = vl[0];
  for (int l = 1; l <= L; l++) t = t + vl[l];
  free(vl);
  free(f);
  return avol * t;
}

static void compute_energies(cal_oracle *o, double out[7]) {
  double v[3], b[3];
  rms_vector(o, CALO_VELO, v);
  double t = rms_scalar(o, CALO_TEMP);
  rms_vector(o, CALO_MAGNE, b);
  out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; out[3] = t;
  out[4] = b[0]; out[5] = b[1]; out[6] = b[2];
}

/* total temperature for output and back to the perturbation
 * (set_reference_sph_mhd.f90 trans_per_temp_to_temp_sph /
 *  sync_temp_by_per_temp_sph), with the energies evaluated in between */
static void output_stage(cal_oracle *o, double ene[7]) {
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) FLD(o, CALO_TEMP)[AT(o, k, 0)] += o->reft0[k];
  compute_energies(o, ene);
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) FLD(o, CALO_TEMP)[AT(o, k, 0)] -= o->reft0[k];
}

/* Volume spectra of the seven energies grouped by degree l, order |m| and
 * l - |m| (sum_sph_rms_data.f90 set_sum_table_4_sph_spectr and
 * sum_sph_v_rms_by_degree: per-j radial integrals of rms_vector /
 * rms_scalar added into the group of their j, times 1/volume), with the
 * total temperature as calo_energies.  out_x[q * (L+1) + g]. */
int calo_energy_spectra(cal_oracle *o, double *out_l, double *out_m, double *out_lm) {
  int ki = o->kin, ko = o->kout, L = o->L;
  size_t n = 7 * (size_t)(L + 1);
  memset(out_l, 0, n * sizeof(double));
  memset(out_m, 0, n * sizeof(double));
  memset(out_lm, 0, n * sizeof(double));
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) FLD(o, CALO_TEMP)[AT(o, k, 0)] += o->reft0[k];
  double *f = malloc(o->nr * 7 * sizeof(double));
  for (int j = 0; j < o->jmax; j++) {
    for (int k = 0; k < o->nr; k++) {
      size_t a = AT(o, k, j);
      double a1 = o->ar1[k];
      for (int v = 0; v < 2; v++) {
        int s = v ? CALO_MAGNE : CALO_VELO, q0 = v ? 4 : 0;
        double S = FLD(o, s)[a], dS = FLD(o, s + 1)[a], T = FLD(o, s + 2)[a], p, t;
        if (j == 0) {
          p = (0.5 * S) * (0.5 * S) * a1 * a1;
          t = 0.0;
        } else {
          p = o->g12[j] * (o->g3[j] * a1 * a1 * S * S + dS * dS);
          t = o->g12[j] * T * T;
        }
        f[7 * k + q0] = 0.5 * p;
        f[7 * k + q0 + 1] = 0.5 * t;
        f[7 * k + q0 + 2] = 0.5 * (p + t);
      }
      double tv = FLD(o, CALO_TEMP)[a];
      f[7 * k + 3] = tv * tv * o->g11[j] * o->r[k] * o->r[k];
    }
    int l = o->jl[j], m = abs(o->jm[j]);
    for (int q = 0; q < 7; q++) {
      double fi = 0.0;
      for (int kr = ki; kr < ko; kr++)
        fi = fi + 0.5 * (o->r[kr + 1] - o->r[kr]) * (f[7 * kr + q] + f[7 * (kr + 1) + q]);
      out_l[q * (L + 1) + l] += fi;
      out_m[q * (L + 1) + m] += fi;
      out_lm[q * (L + 1) + (l - m)] += fi;
    }
  }
  free(f);
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) FLD(o, CALO_TEMP)[AT(o, k, 0)] -= o->reft0[k];
  double avol = 3.0 / (pow(o->r[ko], 3) - pow(o->r[ki], 3));
  for (size_t i = 0; i < n; i++) {
    out_l[i] *= avol;
    out_m[i] *= avol;
    out_lm[i] *= avol;
  }
  return 0;
}

/* energies of the current state without touching it (initial state) */
static void peek_energies(cal_oracle *o, double ene[7]) {
  double *save = malloc(o->nr * sizeof(double));
  for (int k = 0; k < o->nr; k++) save[k] = FLD(o, CALO_TEMP)[AT(o, k, 0)];
  output_stage(o, ene);
  for (int k = 0; k < o->nr; k++) FLD(o, CALO_TEMP)[AT(o, k, 0)] = save[k];
  free(save);
}

/* ---------------------------------------------------------------------- */
cal_oracle *calo_create(const calo_params *p) {
  cal_oracle *o = calloc(1, sizeof(cal_oracle));
  o->p = *p;
  o->L = p->ltr;
  o->nth = p->nth;
  o->nph = p->nph;
  o->nr = p->nr;
  o->jmax = (p->ltr + 1) * (p->ltr + 1);
  o->kin = 0;
  o->kout = p->nr - 1;
  if (p->nthreads > 0) {
#ifdef _OPENMP
    extern void omp_set_num_threads(int);
    omp_set_num_threads(p->nthreads);
#endif
  }
  if (o->nr < 5 || o->nth < 2 || o->nph < 4) { free(o); return NULL; }
  calo_setup_grid(o);
  calo_setup_coriolis(o);
  o->coef_exp_v = 1.0 - p->coef_imp_v;
  o->coef_exp_t = 1.0 - p->coef_imp_t;
  o->coef_exp_b = 1.0 - p->coef_imp_b;
  /* fixed temperature of the perturbation (adjust_sph_temp_bc_by_reftemp) */
  o->temp_icb_fld = p->temp_icb - (p->use_ref_temp ? o->reft0[o->kin] : 0.0);
  o->temp_cmb_fld = p->temp_cmb - (p->use_ref_temp ? o->reft0[o->kout] : 0.0);
  if (build_matrices(o)) { calo_destroy(o); return NULL; }
  size_t n = (size_t)o->nr * o->jmax;
  for (int s = 0; s < CALO_NFIELD; s++) o->f[s] = calloc(n, sizeof(double));
  o->fft_plan = calo_fft_plan(o->nph);
  return o;
}

void calo_destroy(cal_oracle *o) {
  if (!o) return;
  for (int s = 0; s < CALO_NFIELD; s++) free(o->f[s]);
  for (int l = 0; o->vp_lu && l <= o->L; l++) {
    free(o->vp_lu[l].lu); free(o->vp_lu[l].piv);
    free(o->vt_lu[l].lu); free(o->vt_lu[l].piv);
    free(o->bs_lu[l].lu); free(o->bs_lu[l].piv);
    free(o->bt_lu[l].lu); free(o->bt_lu[l].piv);
    free(o->temp_lu[l].lu); free(o->temp_lu[l].piv);
  }
  free(o->vp_lu); free(o->vt_lu); free(o->bs_lu); free(o->bt_lu); free(o->temp_lu);
  free(o->jgi1); free(o->jgi2); free(o->jei1); free(o->gi1); free(o->gi2); free(o->ei1);
  for (int i = 0; i < 6; i++) free(o->sw[i]);
  for (int i = 0; i < 8; i++) free(o->tw[i]);
  calo_fft_free(o->fft_plan);
  calo_free_grid(o);
  free(o);
}

int calo_jmax(const cal_oracle *o) { return o->jmax; }
int calo_istep(const cal_oracle *o) { return o->istep; }

/* a small portable generator for the seeded initial state */
static unsigned long long rng_next(unsigned long long *s) {
  unsigned long long z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double rng_uniform(unsigned long long *s) {
  return (double)(rng_next(s) >> 11) * (1.0 / 9007199254740992.0);
}

int calo_init_fields(cal_oracle *o, int kind, unsigned seed) {
  size_t n = (size_t)o->nr * o->jmax;
  for (int s = 0; s < CALO_NFIELD; s++) memset(o->f[s], 0, n * sizeof(double));
  double pi = 4.0 * atan(1.0);
  double ri = o->r[o->kin], ro = o->r[o->kout], shell = ro - ri;
  double *T = FLD(o, CALO_TEMP);
  /* total temperature: reference profile in l = 0 (set_ini_reference_temp_sph) */
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) T[AT(o, k, 0)] = o->reft0[k];
  if (kind == 1) {
    /* m = l = 4 thermal perturbation (set_initial_temp_sph, isig = 400) */
    int jj = calo_j(4, 4);
    if (jj < o->jmax)
      for (int k = o->kin; k <= o->kout; k++) {
        double xr = 2.0 * o->r[k] - 1.0 * (ro + ri) / shell;
        double x2 = xr * xr, x4 = x2 * x2, x6 = x4 * x2;
        T[AT(o, k, jj)] = (1.0 - 3.0 * x2 + 3.0 * x4 - x6) * 0.1 * 3.0 / sqrt(2.0 * pi);
      }
    /* initial_b_dynamobench_1 (initial_magne_dynamobench.f90:30-80) */
    int js = calo_j(1, 0), jt = calo_j(2, 0);
    for (int k = o->kin; k <= o->kout; k++) {
      double rr = o->r[k];
      if (js < o->jmax) {
        FLD(o, CALO_MAGNE)[AT(o, k, js)] =
            (5.0 / 8.0) * (-3.0 * rr * rr * rr + 4.0 * ro * rr * rr - ri * ri * ri * ri / rr);
        FLD(o, CALO_MAGNE + 1)[AT(o, k, js)] =
            (5.0 / 8.0) * (-9.0 * rr * rr + 8.0 * ro * rr + ri * ri * ri * ri / (rr * rr));
        FLD(o, CALO_CURRENT + 2)[AT(o, k, js)] = (5.0 * 3.0 / 2.0) * rr;
      }
      if (jt < o->jmax) {
        double bt = (10.0 / 3.0) * rr * sin(pi * (rr - ri));
        FLD(o, CALO_MAGNE + 2)[AT(o, k, jt)] = bt;
        FLD(o, CALO_CURRENT)[AT(o, k, jt)] = bt;
        FLD(o, CALO_CURRENT + 1)[AT(o, k, jt)] =
            (10.0 / 3.0) * (sin(pi * (rr - ri)) + pi * rr * cos(pi * (rr - ri)));
      }
    }
  } else if (kind == 2) {
    /* seeded thermal perturbation of amplitude 0.1 on random l <= 8 modes
     * with the benchmark radial profile, plus a weak random dipole-dominated
     * poloidal seed field (no reference counterpart; identical on the
     * oracle and the CUDA path because both use this generator) */
    unsigned long long st = 0x5DEECE66DULL ^ ((unsigned long long)seed << 17);
    int lmax = (o->L < 8) ? o->L : 8;
    for (int l = 1; l <= lmax; l++)
      for (int m = -l; m <= l; m++) {
        double amp = 0.1 * (2.0 * rng_uniform(&st) - 1.0) / sqrt((double)(2 * l + 1));
        int j = calo_j(l, m);
        for (int k = o->kin; k <= o->kout; k++) {
          double xr = 2.0 * o->r[k] - 1.0 * (ro + ri) / shell;
          double x2 = xr * xr, x4 = x2 * x2, x6 = x4 * x2;
          T[AT(o, k, j)] = amp * (1.0 - 3.0 * x2 + 3.0 * x4 - x6);
        }
      }
    int lb = (o->L < 3) ? o->L : 3;
    for (int l = 1; l <= lb; l++)
      for (int m = -l; m <= l; m++) {
        double amp = (l == 1 && m == 0 ? 1.0e-2 : 1.0e-3) * (2.0 * rng_uniform(&st) - 1.0);
        int j = calo_j(l, m);
        for (int k = o->kin; k <= o->kout; k++) {
          double rr = o->r[k];
          FLD(o, CALO_MAGNE)[AT(o, k, j)] =
              amp * (-3.0 * rr * rr * rr + 4.0 * ro * rr * rr - ri * ri * ri * ri / rr);
        }
      }
  } else {
    return 1;
  }
  /* perturbation temperature (sync_temp_by_per_temp_sph) */
  if (o->p.use_ref_temp)
    for (int k = 0; k < o->nr; k++) T[AT(o, k, 0)] -= o->reft0[k];
  return calo_start(o);
}

int calo_start(cal_oracle *o) {
  /* set_sph_field_to_start (cal_sol_sph_MHD_crank.f90:106-136) */
  grad_vp_and_vorticity(o);
  vort_diffusion(o);
  rot_buoyancy(o);
  temp_diffusion(o);
  grad_bp_and_current(o);
  mag_diffusion(o);
  nonlinear(o);
  o->istep = 0;
  o->time = 0.0;
  peek_energies(o, o->ene);
  return 0;
}

int calo_step(cal_oracle *o, int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    o->istep += 1;
    o->time += o->p.dt;
    explicit_update(o, o->istep == 1);
    implicit_solve(o);
    nonlinear(o);
    output_stage(o, o->ene);
  }
  return 0;
}

int calo_energies(cal_oracle *o, double out[7]) {
  for (int i = 0; i < 7; i++) out[i] = o->ene[i];
  return 0;
}

int calo_get_field(const cal_oracle *o, int slot, double *buf) {
  if (slot < 0 || slot >= CALO_NFIELD) return 1;
  memcpy(buf, o->f[slot], (size_t)o->nr * o->jmax * sizeof(double));
  return 0;
}

int calo_set_field(cal_oracle *o, int slot, const double *buf) {
  if (slot < 0 || slot >= CALO_NFIELD) return 1;
  memcpy(o->f[slot], buf, (size_t)o->nr * o->jmax * sizeof(double));
  return 0;
}

int calo_get_gauss(const cal_oracle *o, double *colat, double *weight) {
  memcpy(colat, o->colat, o->nth * sizeof(double));
  memcpy(weight, o->wgt, o->nth * sizeof(double));
  return 0;
}

int calo_get_radius(const cal_oracle *o, double *r) {
  memcpy(r, o->r, o->nr * sizeof(double));
  return 0;
}

int calo_get_plm(const cal_oracle *o, int l, int m, double *p, double *dp) {
  if (m < 0 || m > l || l > o->L) return 1;
  int nl = o->L + 1 - m;
  for (int i = 0; i < o->nth; i++) {
    p[i] = o->pm[m][(size_t)i * nl + (l - m)];
    dp[i] = o->dpm[m][(size_t)i * nl + (l - m)];
  }
  return 0;
}

int calo_get_gaunt(const cal_oracle *o, int j, double *gi, double *ei) {
  if (j < 0 || j >= o->jmax) return 1;
  gi[0] = o->gi1[j];
  gi[1] = o->gi2[j];
  ei[0] = o->ei1[j];
  return 0;
}
