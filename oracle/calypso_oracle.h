/*
 * calypso_oracle.h -- CPU FP64 restatement of the Calypso time-step hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * Nothing in the product (calypso_b200/, libcalypso_b200.so) links or calls it.
 *
 * It restates, in plain C with OpenMP, the algorithm of the reference
 * (hlokavarapu/calypso, Fortran 90) for one MHD time step of a rotating
 * spherical shell: Crank-Nicolson + 2nd-order Adams-Bashforth in the
 * (r, l, m) "rj" spectral space, pseudo-spectral nonlinear terms through the
 * spherical-harmonic transform (Legendre per order m + phi FFT), Coriolis
 * force through Gaunt/Elsasser integrals in spectral space, and pivoted
 * banded LU radial solves.  Each routine cites the reference file it follows.
 *
 * Parity pin: tests/test_oracle_golden.py runs the Dynamobench case 1 set-up
 * (tests/Dynamobench_case1 of the reference) and compares the volume mean
 * square energies at steps 50 and 100 with the reference's own golden file
 * (reference/sph_pwr_volume_s.dat) at the reference's 1e-9 tolerance.
 *
 * Index conventions used everywhere in this file and in the CUDA library:
 *   j = l*(l+1) + m, 0 <= j < (L+1)^2, m<0 holds the sin(|m| phi) part
 *   radial index k = 0..nr-1 (reference k = k+1)
 *   a spectral field is stored f[k*jmax + j]   (reference d_rj(j+(k-1)*jmax))
 *   a vector field occupies 3 slots: poloidal S, dS/dr, toroidal T
 *   grid data of one component: g[(k*nth + i)*nph + p], theta index i=0 near
 *   the south pole (x=-1), as the reference's Gauss node ordering.
 */
#ifndef CALYPSO_ORACLE_H
#define CALYPSO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct calo_params {
  int ltr;              /* truncation_level_ctl                          */
  int nth;              /* ngrid_meridonal_ctl                           */
  int nph;              /* ngrid_zonal_ctl                               */
  int nr;               /* number of radial points (num_fluid_grid+1)    */
  int radial_grid_type; /* 0: equidistance, 1: Chebyshev                 */
  double r_icb, r_cmb;
  double dt;
  double coef_imp_v, coef_imp_t, coef_imp_b;
  /* coefficients of the normalised equations (construct_coefficient) */
  double coef_velo, coef_d_velo, coef_buo, coef_cor, coef_lor;
  double coef_temp, coef_d_temp;
  double coef_magne, coef_d_magne, coef_induct;
  /* reference temperature (ref_temp_ctl spherical_shell) */
  int use_ref_temp;
  double depth_high_t, depth_low_t, high_temp, low_temp;
  /* fixed temperature boundary values of the total temperature */
  double temp_icb, temp_cmb;
  int nthreads;         /* 0: OpenMP default */
} calo_params;

typedef struct cal_oracle cal_oracle;

/* field slot ids (vector fields take 3 consecutive slots: S, dS/dr, T) */
enum {
  CALO_VELO = 0, CALO_VORT = 3, CALO_MAGNE = 6, CALO_CURRENT = 9,
  CALO_TEMP = 12, CALO_WDIFF = 13, CALO_BDIFF = 16, CALO_TDIFF = 19,
  CALO_MADV = 20, CALO_LOR = 23, CALO_VPIND = 26, CALO_HFLUX = 29,
  CALO_ROTINERT = 32, CALO_ROTLOR = 35, CALO_INDUCT = 38, CALO_HADV = 41,
  CALO_ROTCOR = 42, CALO_ROTBUO = 45, CALO_FORCES = 48, CALO_PREMOM = 51,
  CALO_PREUXB = 54, CALO_PREHEAT = 57, CALO_NFIELD = 58
};

cal_oracle *calo_create(const calo_params *p);
void calo_destroy(cal_oracle *o);
int calo_jmax(const cal_oracle *o);

/* initial state: kind 1 = dynamo benchmark case 1 (set_initial_sph_dynamo,
 * initial_b_dynamobench_1); kind 2 = seeded perturbation on random l<=8 modes
 * plus weak dipole-dominated seed field (defined by this build). */
int calo_init_fields(cal_oracle *o, int kind, unsigned seed);
/* SPH_analyze_MHD repeated nsteps times (step counter continues) */
int calo_step(cal_oracle *o, int nsteps);
int calo_istep(const cal_oracle *o);
/* volume mean square of the output file sph_pwr_volume_s.dat:
 * out[0..6] = K_pol, K_tor, K, <T^2>, M_pol, M_tor, M  (total temperature) */
int calo_energies(cal_oracle *o, double out[7]);
/* the seven energies by degree l, order |m| and l - |m|: out_x[q (L+1) + g] */
int calo_energy_spectra(cal_oracle *o, double *out_l, double *out_m, double *out_lm);
/* copy one field slot (nr*jmax doubles) out / in */
int calo_get_field(const cal_oracle *o, int slot, double *buf);
int calo_set_field(cal_oracle *o, int slot, const double *buf);
/* recompute derived fields (gradients, vorticity, current, diffusion terms)
 * and the first nonlinear terms after fields were set: set_sph_field_to_start
 * + nonlinear of SPH_initialize_MHD */
int calo_start(cal_oracle *o);

/* tables: Gauss colatitudes and weights (nth), radius (nr) */
int calo_get_gauss(const cal_oracle *o, double *colat, double *weight);
int calo_get_radius(const cal_oracle *o, double *r);
/* Schmidt P_l^m(theta_i) and dP/dtheta for one (l, m>=0) over all nth */
int calo_get_plm(const cal_oracle *o, int l, int m, double *p, double *dp);
/* Coriolis Gaunt/Elsasser coefficients of j: gi(2), ei(1) */
int calo_get_gaunt(const cal_oracle *o, int j, double *gi, double *ei);
double calo_leadki(int l1, int m1, int l2, int m2, int l3, int m3);
double calo_leadli(int l1, int m1, int l2, int m2, int l3, int m3);

/* Isolated spherical transforms (legendre_b_trans_*_org + FFT):
 * spec: (3*nvec + nscal) fields of nr*jmax, order vec0(S,dS,T), vec1.., scal0..
 * grid: (3*nvec + nscal) components of nr*nth*nph, vector = (r, theta, phi) */
int calo_sht_backward(cal_oracle *o, int nvec, int nscal,
                      const double *spec, double *grid);
int calo_sht_forward(cal_oracle *o, int nvec, int nscal,
                     const double *grid, double *spec);
/* Legendre-only and FFT-only halves of the transforms: Fourier arrays
 * four[c][k][i][m + L] (m < 0: the sin(|m| phi) coefficient), grids
 * grid[c][k][i][p]; spectra as for calo_sht_* */
int calo_leg_backward(cal_oracle *o, int nvec, int nscal, const double *spec, double *four);
int calo_leg_forward(cal_oracle *o, int nvec, int nscal, const double *four, double *spec);
int calo_fft_backward(cal_oracle *o, int ncomp, const double *four, double *grid);
int calo_fft_forward(cal_oracle *o, int ncomp, const double *grid, double *four);

#ifdef __cplusplus
}
#endif
#endif
