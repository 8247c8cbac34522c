/*
 * oracle_internal.h -- private state of the CPU oracle (test infrastructure).
 * See calypso_oracle.h for the conventions.  Reference paths are relative to
 * the reference tree, F/ = src/Fortran_libraries/.
 */
#ifndef CALYPSO_ORACLE_INTERNAL_H
#define CALYPSO_ORACLE_INTERNAL_H

#include "calypso_oracle.h"

typedef struct {
  /* d/dr and d2/dr2 with fixed value at the wall (fdm2_fix_fld_ICB/CMB):
   * fld[i][c], i = 0,1,2 node offset (away from the wall), c = 1..3
   * derivative order + 1 (F/MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90) */
  double fix_fld_icb[3][4], fix_fld_cmb[3][4];
  /* fixed gradient at the wall (fdm2_fix_dr_ICB/CMB): dr[i+1][c], i=-1..1 */
  double fix_dr_icb[3][4], fix_dr_cmb[3][4];
  double r_icb[3], r_cmb[3];   /* r, 1/r, 1/r^2 at the boundary node */
} calo_bc;

typedef struct {
  /* tri-diagonal LU (ludcmp_3band): lu[5][n], pivot[n]; per degree l */
  int n;
  double *lu;  /* 5*n, lu[b*n + k], b = band row 0..4 (Fortran 1..5) */
  int *piv;    /* n (1-based row like the reference)                  */
} calo_lu3;

typedef struct {
  int n;
  double *lu;  /* 9*n, lu[b*n + k], b = 0..8 (Fortran band_lu(1..9,k)) */
  int *piv;
} calo_lu5;

struct cal_oracle {
  calo_params p;
  int L, nth, nph, nr, jmax, kin, kout;   /* kin/kout 0-based */
  int *jl, *jm;                           /* degree / order of j          */
  double *g3, *g3rlm, *g11, *g12, *g13, *g6, *g7, *g17, *gl;
  /* radial */
  double *r, *ar1, *ar2;
  double *d1[3], *d2[3];   /* d1nod_mat_fdm_2(k,-1:1) -> d1[0..2][k] */
  calo_bc bc;
  double *reft0, *reft1;   /* reftemp_rj(k,0:1)                      */
  double *om[3];           /* omega_rlm(k,0:2) for Omega_z = 1       */
  /* Gauss-Legendre colatitude and weights (index 0 near theta = pi) */
  double *colat, *wgt, *asin_t;
  /* Schmidt P and dP/dtheta: for m>=0, pm[m][i*(L+1-m) + (l-m)] */
  double **pm, **dpm;
  /* Coriolis: partner j (jgi1, jgi2, jei1) and coefficients per j */
  int *jgi1, *jgi2, *jei1;
  double *gi1, *gi2, *ei1;
  double *sw[6], *tw[8];    /* sw11 sw21 sw12 sw22 sw13 sw23 ; tw11 tw21
                               tw12 tw22 tw13 tw23 tw14 tw24          */
  /* implicit operators, factorised per degree l */
  calo_lu5 *vp_lu;   calo_lu3 *vt_lu;
  calo_lu3 *bs_lu;   calo_lu3 *bt_lu;
  calo_lu3 *temp_lu;
  double coef_exp_v, coef_exp_t, coef_exp_b;
  double temp_icb_fld, temp_cmb_fld;    /* l=0 boundary values of the
                                           perturbation temperature */
  /* fields */
  double *f[CALO_NFIELD];
  int istep;
  double time;
  double ene[7];            /* energies of the last output stage */
  int fft_n;
  void *fft_plan;
};

/* grid set-up (oracle_grid.c) */
int calo_setup_grid(cal_oracle *o);
void calo_free_grid(cal_oracle *o);
/* Gaunt integrals (oracle_gaunt.c) */
int calo_setup_coriolis(cal_oracle *o);
/* transforms (oracle_sht.c) */
void *calo_fft_plan(int n);
void calo_fft_free(void *plan);
/* inverse real DFT of a_m/b_m (m=0..L) into x[n] for two rows at once */
void calo_fourier_to_grid2(const void *plan, int n, int L,
                           const double *a0, const double *b0,
                           const double *a1, const double *b1,
                           double *x0, double *x1);
void calo_grid_to_fourier2(const void *plan, int n, int L,
                           const double *x0, const double *x1,
                           double *a0, double *b0, double *a1, double *b1);
int calo_nonlinear_transforms(cal_oracle *o);
/* linear algebra (oracle_mhd.c) */
int calo_ludcmp_3band(int n, const double *band_a, double *band_lu,
                      int *ipiv);
int calo_ludcmp_band5(int n, const double *band_a, double *band_lu,
                      int *ipiv);
void calo_lubksb_3band(int n, const double *lu, const int *ipiv, double *x);
void calo_lubksb_5band(int n, const double *lu, const int *ipiv, double *x);

static inline int calo_j(int l, int m) { return l * (l + 1) + m; }

#endif
