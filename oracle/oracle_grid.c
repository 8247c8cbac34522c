/*
 * oracle_grid.c -- radial grid, finite-difference weights, Gauss-Legendre
 * nodes, Schmidt quasi-normalised Legendre functions and harmonic
 * normalisations of the CPU oracle (test infrastructure, see
 * calypso_oracle.h).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* determinant and adjugate inverse of a 3x3 matrix, a[i][j] row i col j
 * (F/SERIAL_src/BASE/cal_inverse_small_matrix.f90:176-218) */
static double det33(const double a[3][3]) {
  return a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2])
       - a[0][1] * (a[1][0] * a[2][2] - a[2][0] * a[1][2])
       + a[0][2] * (a[1][0] * a[2][1] - a[2][0] * a[1][1]);
}

static int inv33(const double a[3][3], double ainv[3][3]) {
  double det = det33(a);
  if (fabs(det) < 1.0e-40) return 1;
  double adet = 1.0 / det;
  for (int kj = 0; kj < 3; kj++) {
    for (int ki = 0; ki < 3; ki++) {
      double t[2][2];
      int jj = 0;
      for (int j = 0; j < 3; j++) {
        if (j == kj) continue;
        int ii = 0;
        for (int i = 0; i < 3; i++) {
          if (i == ki) continue;
          t[ii][jj] = a[i][j];
          ii++;
        }
        jj++;
      }
      double d = t[0][0] * t[1][1] - t[1][0] * t[0][1];
      double s = ((ki + kj) % 2 == 0) ? 1.0 : -1.0;
      ainv[kj][ki] = s * d * adet;
    }
  }
  return 0;
}

/* Chebyshev / equidistant radial grid of the fluid shell
 * (F/SERIAL_src/SPH_SPECTR_src/set_radial_grid_sph_shell.f90:40-111) */
static void set_radius(cal_oracle *o) {
  int nr = o->nr, nri = nr - 1;
  double ri = o->p.r_icb, ro = o->p.r_cmb, shell = ro - ri;
  double pi = 4.0 * atan(1.0);
  for (int k = 0; k < nr; k++) {
    if (o->p.radial_grid_type == 1)
      o->r[k] = ri + 0.5 * shell * (1.0 - cos(pi * (double)k / (double)nri));
    else
      o->r[k] = ri + (ro - ri) * (double)k / (double)nri;
    o->ar1[k] = 1.0 / o->r[k];
    o->ar2[k] = o->ar1[k] * o->ar1[k];
  }
}

/* 2nd-order FDM weights on the non-uniform grid
 * (F/SERIAL_src/SPH_SPECTR_src/set_radius_func_noequi.f90:120-230,
 *  F/SERIAL_src/SPH_SPECTR_src/m_fdm_coefs.f90 copy_fdm_nod_coefs_from_mat) */
static void set_fdm(cal_oracle *o) {
  int nr = o->nr;
  double *dr = calloc(nr, sizeof(double));
  for (int k = 1; k < nr - 1; k++) dr[k] = o->r[k + 1] - o->r[k];
  dr[nr - 1] = o->r[nr - 1] - o->r[nr - 2];
  dr[0] = o->r[1] - o->r[0];
  for (int k = 0; k < nr; k++) {
    double dp, dn;
    if (k == 0) { dp = dr[0]; dn = dr[0]; }
    else if (k == nr - 1) { dp = dr[k]; dn = dr[k]; }
    else { dp = dr[k]; dn = dr[k - 1]; }
    double a[3][3] = {{1.0, 0.0, 0.0},
                      {1.0, dp, 0.5 * dp * dp},
                      {1.0, -dn, 0.5 * dn * dn}};
    double m[3][3];
    inv33(a, m);
    o->d1[0][k] = m[1][2]; o->d1[1][k] = m[1][0]; o->d1[2][k] = m[1][1];
    o->d2[0][k] = m[2][2]; o->d2[1][k] = m[2][0]; o->d2[2][k] = m[2][1];
  }
  free(dr);
}

/* one-sided boundary weights (F/MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90) */
static void set_bc_fdm(cal_oracle *o) {
  calo_bc *b = &o->bc;
  int ki = o->kin, ko = o->kout;
  double *r = o->r, m[3][3];
  memset(b, 0, sizeof(*b));
  {  /* fixed field at ICB: unknowns (f, f', f''), data (f0, f1, f2) */
    double d1 = r[ki + 1] - r[ki], d2 = r[ki + 2] - r[ki];
    double a[3][3] = {{1, 0, 0}, {1, d1, d1 * d1 / 2.0}, {1, d2, d2 * d2 / 2.0}};
    inv33(a, m);
    for (int c = 0; c < 3; c++) {
      b->fix_fld_icb[0][c + 1] = m[c][0];
      b->fix_fld_icb[1][c + 1] = m[c][1];
      b->fix_fld_icb[2][c + 1] = m[c][2];
    }
  }
  {  /* fixed gradient at ICB: unknowns (f', f, f''), data (f'0, f0, f1) */
    double d1 = r[ki + 1] - r[ki];
    double a[3][3] = {{1, 0, 0}, {0, 1, 0}, {d1, 1, d1 * d1 / 2.0}};
    inv33(a, m);
    for (int c = 0; c < 3; c++) {
      b->fix_dr_icb[0][c + 1] = m[c][0];   /* index -1 */
      b->fix_dr_icb[1][c + 1] = m[c][1];   /* index  0 */
      b->fix_dr_icb[2][c + 1] = m[c][2];   /* index  1 */
    }
  }
  {  /* fixed field at CMB: data (f0, f-1, f-2) */
    double d1 = r[ko] - r[ko - 1], d2 = r[ko] - r[ko - 2];
    double a[3][3] = {{1, 0, 0}, {1, -d1, d1 * d1 / 2.0}, {1, -d2, d2 * d2 / 2.0}};
    inv33(a, m);
    for (int c = 0; c < 3; c++) {
      b->fix_fld_cmb[0][c + 1] = m[c][0];
      b->fix_fld_cmb[1][c + 1] = m[c][1];
      b->fix_fld_cmb[2][c + 1] = m[c][2];
    }
  }
  {  /* fixed gradient at CMB: unknowns (f, f', f''), data (f0, f'0, f-1) */
    double d1 = r[ko] - r[ko - 1];
    double a[3][3] = {{1, 0, 0}, {0, 1, 0}, {1, -d1, d1 * d1 / 2.0}};
    inv33(a, m);
    for (int c = 0; c < 3; c++) {
      b->fix_dr_cmb[0][c + 1] = m[c][2];   /* index -1 */
      b->fix_dr_cmb[1][c + 1] = m[c][0];   /* index  0 */
      b->fix_dr_cmb[2][c + 1] = m[c][1];   /* index  1 */
    }
  }
  b->r_icb[0] = r[ki]; b->r_icb[1] = o->ar1[ki]; b->r_icb[2] = o->ar2[ki];
  b->r_cmb[0] = r[ko]; b->r_cmb[1] = o->ar1[ko]; b->r_cmb[2] = o->ar2[ko];
}

/* Gauss-Legendre nodes by Newton iteration, index 0 near x = -1
 * (F/SERIAL_src/gauss_integration/m_gauss_points.f90:117-210) */
static void set_gauss(cal_oracle *o) {
  int n = o->nth;
  double pi = 4.0 * atan(1.0);
  double *x = malloc(n * sizeof(double)), *w = malloc(n * sizeof(double));
  int mh = (n + 1 - (n + 1) % 2) / 2;
  for (int i = 1; i <= mh; i++) {
    double z = cos(pi * ((double)i - 0.25) / ((double)n + 0.5));
    double pp, z1;
    for (;;) {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; j++) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * (double)j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
      }
      pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (fabs(z - z1) < 3.0e-12) break;
    }
    x[i - 1] = 0.5 - 0.5 * z;
    x[n - i] = 0.5 + 0.5 * z;
    w[i - 1] = 2.0 * 0.5 / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
  for (int i = 0; i < n; i++) {
    double xx = x[i] * 2.0 - 1.0;
    o->wgt[i] = w[i] * 2.0;
    o->colat[i] = acos(xx);
    o->asin_t[i] = 1.0 / sin(o->colat[i]);
  }
  free(x);
  free(w);
}

/* Schmidt quasi-normalised P_l^m(cos theta), l = m..ltr, into p[0..ltr]
 * (F/SERIAL_src/spherical_harmonics/schmidt_fix_m.f90:62-142) */
static void schmidt_m(int ltr, int m, double theta, double *p, double *df) {
  if (m < 0) {
    for (int l = 0; l <= ltr; l++) p[l] = 0.0;
  } else if (m == 0) {
    p[0] = 1.0;
    if (ltr >= 1) p[1] = cos(theta);
    for (int l = 2; l <= ltr; l++)
      p[l] = p[l - 1] * (double)(2 * l - 1) / (double)l * cos(theta)
           - p[l - 2] * (double)(l - 1) / (double)l;
  } else {
    df[m] = 1.0;
    for (int k = 1; k <= m; k++) df[m] = df[m] * (double)(2 * k - 1) / (double)(2 * k);
    df[m + 1] = sqrt(2.0 * df[m] * (double)(2 * m + 1)) * cos(theta);
    df[m] = sqrt(2.0 * df[m]);
    if (m < ltr - 1) {
      for (int l = m + 2; l <= ltr; l++)
        df[l] = (cos(theta) * (double)(2 * l - 1) * df[l - 1]
                 - sqrt((double)((l - 1) * (l - 1) - m * m)) * df[l - 2])
                / sqrt((double)(l * l - m * m));
    }
    for (int l = m; l <= ltr; l++) {
      p[l] = df[l];
      for (int m1 = 1; m1 <= m; m1++) p[l] = p[l] * sin(theta);
    }
  }
}

/* dP/dtheta from P^{m-1} and P^{m+1}
 * (F/SERIAL_src/spherical_harmonics/schmidt_fix_m.f90:146-175) */
static void diff_schmidt_m(int ltr, int m, const double *pmn1,
                           const double *pmp1, double *dp) {
  if (m == 0) {
    dp[0] = 0.0;
    for (int l = 1; l <= ltr; l++)
      dp[l] = -sqrt((double)(l * (l + 1) / 2)) * pmp1[l];
  } else if (m == 1) {
    dp[1] = pmn1[1];
    for (int l = 2; l <= ltr; l++)
      dp[l] = 0.5 * (sqrt((double)(2 * l * (l + 1))) * pmn1[l]
                     - sqrt((double)((l - 1) * (l + 2))) * pmp1[l]);
  } else {
    dp[m] = 0.5 * sqrt((double)(2 * m)) * pmn1[m];
    for (int l = m + 1; l <= ltr; l++)
      dp[l] = 0.5 * (sqrt((double)((l + m) * (l - m + 1))) * pmn1[l]
                     - sqrt((double)((l - m) * (l + m + 1))) * pmp1[l]);
  }
}

/* P and dP/dtheta on the Gauss nodes for every order
 * (F/SERIAL_src/SPH_SPECTR_src/schmidt_poly_on_rtm_grid.f90:145-188) */
static void set_legendre(cal_oracle *o) {
  int L = o->L, nth = o->nth;
  o->pm = calloc(L + 1, sizeof(double *));
  o->dpm = calloc(L + 1, sizeof(double *));
  for (int m = 0; m <= L; m++) {
    o->pm[m] = malloc((size_t)nth * (L + 1 - m) * sizeof(double));
    o->dpm[m] = malloc((size_t)nth * (L + 1 - m) * sizeof(double));
  }
#pragma omp parallel
  {
    double *p = calloc(L + 3, sizeof(double)), *dp = calloc(L + 3, sizeof(double));
    double *pn = calloc(L + 3, sizeof(double)), *pp = calloc(L + 3, sizeof(double));
    double *df = calloc(L + 4, sizeof(double));
#pragma omp for schedule(dynamic)
    for (int m = 0; m <= L; m++) {
      int nl = L + 1 - m;
      for (int i = 0; i < nth; i++) {
        double th = o->colat[i];
        schmidt_m(L, m - 1, th, pn, df);
        schmidt_m(L, m, th, p, df);
        schmidt_m(L, m + 1, th, pp, df);
        diff_schmidt_m(L, m, pn, pp, dp);
        for (int l = m; l <= L; l++) {
          o->pm[m][i * nl + (l - m)] = p[l];
          o->dpm[m][i * nl + (l - m)] = dp[l];
        }
      }
    }
    free(p); free(dp); free(pn); free(pp); free(df);
  }
}

/* harmonic normalisations g_sph_rj(j, 1..17)
 * (F/SERIAL_src/spherical_harmonics/spherical_harmonics.f90:92-141,
 *  F/SERIAL_src/SPH_SPECTR_src/schmidt_poly_on_rtm_grid.f90:92-141) */
static void set_normalization(cal_oracle *o) {
  for (int j = 0; j < o->jmax; j++) {
    int l = o->jl[j], m = o->jm[j];
    o->gl[j] = (double)l;
    o->g3[j] = (double)(l * (l + 1));
    o->g11[j] = 1.0 / (double)(2 * l + 1);
    o->g12[j] = (double)(l * (l + 1)) / (double)(2 * l + 1);
    if (l == 0 && m == 0) {
      o->g6[j] = 1.0 / 2.0;
      o->g7[j] = 1.0;
      o->g13[j] = 1.0;
      o->g17[j] = 0.0;
      o->g3rlm[j] = 0.5;
    } else {
      o->g13[j] = 1.0 / (double)(l * (l + 1));
      o->g17[j] = (double)(2 * l + 1) / (double)(4 * l * (l + 1));
      if (m == 0) {
        o->g6[j] = (double)(2 * l + 1) / 2.0;
        o->g7[j] = (double)(2 * l + 1) / (double)(2 * l * (l + 1));
      } else {
        o->g6[j] = (double)(2 * l + 1) / 4.0;
        o->g7[j] = (double)(2 * l + 1) / (double)(4 * l * (l + 1));
      }
      o->g3rlm[j] = o->g3[j];
    }
  }
}

int calo_setup_grid(cal_oracle *o) {
  int nr = o->nr, jmax = o->jmax;
  o->jl = malloc(jmax * sizeof(int));
  o->jm = malloc(jmax * sizeof(int));
  for (int l = 0; l <= o->L; l++)
    for (int m = -l; m <= l; m++) {
      o->jl[calo_j(l, m)] = l;
      o->jm[calo_j(l, m)] = m;
    }
  double **gs[] = {&o->g3, &o->g3rlm, &o->g11, &o->g12, &o->g13, &o->g6,
                   &o->g7, &o->g17, &o->gl};
  for (unsigned i = 0; i < sizeof(gs) / sizeof(gs[0]); i++)
    *gs[i] = calloc(jmax, sizeof(double));
  o->r = calloc(nr, sizeof(double));
  o->ar1 = calloc(nr, sizeof(double));
  o->ar2 = calloc(nr, sizeof(double));
  o->reft0 = calloc(nr, sizeof(double));
  o->reft1 = calloc(nr, sizeof(double));
  for (int i = 0; i < 3; i++) {
    o->d1[i] = calloc(nr, sizeof(double));
    o->d2[i] = calloc(nr, sizeof(double));
    o->om[i] = calloc(nr, sizeof(double));
  }
  o->colat = calloc(o->nth, sizeof(double));
  o->wgt = calloc(o->nth, sizeof(double));
  o->asin_t = calloc(o->nth, sizeof(double));

  set_radius(o);
  set_fdm(o);
  set_bc_fdm(o);
  /* reference temperature (F/MHD_src/sph_MHD/set_reference_sph_mhd.f90
   * set_ref_temp_sph_mhd) */
  for (int k = 0; k < nr; k++) {
    if (o->p.use_ref_temp) {
      double dh = o->p.depth_high_t, dl = o->p.depth_low_t;
      double ht = o->p.high_temp, lt = o->p.low_temp;
      o->reft0[k] = (dh * dl * o->ar1[k] * (ht - lt) - dh * ht + dl * lt) / (dl - dh);
      o->reft1[k] = -dh * dl * o->ar2[k] * (ht - lt) / (dl - dh);
    }
  }
  /* rotation Omega_z = 1 (F/SERIAL_src/SPH_SPECTR_src/m_poloidal_rotation.f90
   * set_rotatio_spectr) */
  for (int k = 0; k < nr; k++) {
    o->om[0][k] = 0.5 * 1.0 * o->r[k] * o->r[k];
    o->om[1][k] = 1.0 * o->r[k];
    o->om[2][k] = 1.0;
  }
  set_gauss(o);
  set_legendre(o);
  set_normalization(o);
  return 0;
}

void calo_free_grid(cal_oracle *o) {
  free(o->jl); free(o->jm);
  double *ps[] = {o->g3, o->g3rlm, o->g11, o->g12, o->g13, o->g6, o->g7,
                  o->g17, o->gl, o->r, o->ar1, o->ar2, o->reft0, o->reft1,
                  o->colat, o->wgt, o->asin_t};
  for (unsigned i = 0; i < sizeof(ps) / sizeof(ps[0]); i++) free(ps[i]);
  for (int i = 0; i < 3; i++) { free(o->d1[i]); free(o->d2[i]); free(o->om[i]); }
  if (o->pm) {
    for (int m = 0; m <= o->L; m++) { free(o->pm[m]); free(o->dpm[m]); }
    free(o->pm); free(o->dpm);
  }
}
