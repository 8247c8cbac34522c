/*
 * oracle_sht.c -- spherical transforms and grid products of the CPU oracle
 * (test infrastructure, see calypso_oracle.h).
 *
 * Legendre transforms follow the definition of the reference's original loop
 * (F/PARALLEL_src/SPH_SHELL_src/legendre_bwd_trans_org.f90:45-209,
 *  legendre_fwd_trans_org.f90:45-169) evaluated with the north/south
 * symmetry of P_l^m that the reference's SYMMETRIC_MATMUL variant uses
 * (cal_vr_rtm_by_matmul.f90, cal_sp_rlm_by_matmul.f90).  The phi transform
 * follows the normalisation of t_MHD_multi_FFTW.F90:220-355:
 *   f(phi) = a_0 + sum_{m=1..L} (a_m cos m phi + b_m sin m phi),
 *   a_0 = (1/N) sum f, a_m = (2/N) sum f cos, b_m = (2/N) sum f sin.
 * Slot m + L of a Fourier array holds a_m for m >= 0 and b_|m| for m < 0.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

typedef struct { double re, im; } cpx;

typedef struct {
  int n, nfac, fac[32];
  cpx *tw;   /* exp(-2 pi i k / n) */
} fftplan;

void *calo_fft_plan(int n) {
  fftplan *p = calloc(1, sizeof(fftplan));
  p->n = n;
  int m = n;
  const int rad[] = {4, 2, 3, 5};
  for (int r = 0; r < 4 && m > 1; r++)
    while (m % rad[r] == 0) { p->fac[p->nfac++] = rad[r]; m /= rad[r]; }
  for (int f = 7; m > 1; f += 2)
    while (m % f == 0) { p->fac[p->nfac++] = f; m /= f; }
  p->tw = malloc(n * sizeof(cpx));
  double pi = 4.0 * atan(1.0);
  for (int k = 0; k < n; k++) {
    p->tw[k].re = cos(2.0 * pi * k / n);
    p->tw[k].im = -sin(2.0 * pi * k / n);
  }
  return p;
}

void calo_fft_free(void *plan) {
  fftplan *p = plan;
  if (!p) return;
  free(p->tw);
  free(p);
}

/* out[0..n) = sum_t in[t*stride] w^(t k); w = exp(sign 2 pi i / n) */
static void fft_rec(const fftplan *pl, const cpx *in, cpx *out, int n,
                    int stride, int fi, int sign) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = pl->fac[fi], m = n / p;
  for (int q = 0; q < p; q++)
    fft_rec(pl, in + q * stride, out + q * m, m, stride * p, fi + 1, sign);
  int N = pl->n, step = N / n;
  cpx t[64];
  for (int k = 0; k < m; k++) {
    for (int q = 0; q < p; q++) {
      int e = (q * k * step) % N;
      cpx w = pl->tw[e];
      if (sign > 0) w.im = -w.im;
      cpx a = out[k + q * m];
      t[q].re = a.re * w.re - a.im * w.im;
      t[q].im = a.re * w.im + a.im * w.re;
    }
    for (int s = 0; s < p; s++) {
      cpx acc = {0.0, 0.0};
      for (int q = 0; q < p; q++) {
        int e = ((q * s) % p) * (N / p);
        cpx w = pl->tw[e];
        if (sign > 0) w.im = -w.im;
        acc.re += t[q].re * w.re - t[q].im * w.im;
        acc.im += t[q].re * w.im + t[q].im * w.re;
      }
      out[k + s * m] = acc;
    }
  }
}

void calo_fourier_to_grid2(const void *plan, int n, int L,
                           const double *a0, const double *b0,
                           const double *a1, const double *b1,
                           double *x0, double *x1) {
  const fftplan *pl = plan;
  cpx *Z = calloc(2 * n, sizeof(cpx)), *z = Z + n;
  /* X_m = (a_m - i b_m)/2, X_0 = a_0; Z = X + i Y */
  Z[0].re = a0[0];
  Z[0].im = a1[0];
  for (int m = 1; m <= L && m < (n + 1) / 2; m++) {
    double xr = 0.5 * a0[m], xi = -0.5 * b0[m];
    double yr = 0.5 * a1[m], yi = -0.5 * b1[m];
    Z[m].re = xr - yi;      Z[m].im = xi + yr;
    Z[n - m].re = xr + yi;  Z[n - m].im = -xi + yr;
  }
  fft_rec(pl, Z, z, n, 1, 0, +1);
  for (int p = 0; p < n; p++) { x0[p] = z[p].re; x1[p] = z[p].im; }
  free(Z);
}

void calo_grid_to_fourier2(const void *plan, int n, int L,
                           const double *x0, const double *x1,
                           double *a0, double *b0, double *a1, double *b1) {
  const fftplan *pl = plan;
  cpx *z = calloc(2 * n, sizeof(cpx)), *Z = z + n;
  for (int p = 0; p < n; p++) { z[p].re = x0[p]; z[p].im = x1[p]; }
  fft_rec(pl, z, Z, n, 1, 0, -1);
  double an = 1.0 / (double)n;
  a0[0] = an * Z[0].re;  b0[0] = 0.0;
  a1[0] = an * Z[0].im;  b1[0] = 0.0;
  for (int m = 1; m <= L; m++) {
    cpx zk = Z[m % n], zn = Z[(n - m) % n];
    /* X = (Z_k + conj Z_{n-k})/2, Y = (Z_k - conj Z_{n-k})/(2i) */
    double xr = 0.5 * (zk.re + zn.re), xi = 0.5 * (zk.im - zn.im);
    double yr = 0.5 * (zk.im + zn.im), yi = -0.5 * (zk.re - zn.re);
    a0[m] = 2.0 * an * xr;  b0[m] = -2.0 * an * xi;
    a1[m] = 2.0 * an * yr;  b1[m] = -2.0 * an * yi;
  }
  free(z);
}

/* ---------------------------------------------------------------------- */
/* Backward Legendre transform at one radius.
 * sp[c][j]: nvec vectors (S, dS/dr, T) then nscal scalars, raw rj values.
 * four[c][i][m+L]: components (v_r, v_theta, v_phi) per vector, then scalars.
 * (legendre_bwd_trans_org.f90:45-209: S/r^2 g3 P -> v_r, dS/r dP -> v_theta,
 *  -T/r dP -> v_phi, mirror order -m with -m P/sin(theta)) */
static void leg_bwd_k(const cal_oracle *o, int k, int nvec, int nscal,
                      const double *const *sp, double *four) {
  int L = o->L, nth = o->nth, ns = 2 * L + 1, nh = nth / 2;
  int ncomp = 3 * nvec + nscal;
  double a1 = o->ar1[k], a2 = a1 * a1;
  size_t cs = (size_t)nth * ns;
  memset(four, 0, (size_t)ncomp * cs * sizeof(double));
  double *buf = malloc((size_t)(3 * nvec + nscal) * 2 * (L + 1) * sizeof(double));
  for (int m = 0; m <= L; m++) {
    int nl = L + 1 - m;
    const double *P = o->pm[m], *dP = o->dpm[m];
    /* gathered, pre-scaled coefficients: [c][sign][l-m] */
    for (int v = 0; v < nvec; v++) {
      for (int s = 0; s < 2; s++) {
        int mm = s ? -m : m;
        double *bS = buf + ((3 * v + 0) * 2 + s) * (L + 1);
        double *bD = buf + ((3 * v + 1) * 2 + s) * (L + 1);
        double *bT = buf + ((3 * v + 2) * 2 + s) * (L + 1);
        for (int l = m; l <= L; l++) {
          int j = calo_j(l, mm);
          bS[l - m] = sp[3 * v + 0][(size_t)k * o->jmax + j] * a2 * o->g3rlm[j];
          bD[l - m] = sp[3 * v + 1][(size_t)k * o->jmax + j] * a1;
          bT[l - m] = sp[3 * v + 2][(size_t)k * o->jmax + j] * a1;
        }
      }
    }
    for (int c = 0; c < nscal; c++)
      for (int s = 0; s < 2; s++) {
        int mm = s ? -m : m;
        double *b = buf + ((3 * nvec + c) * 2 + s) * (L + 1);
        for (int l = m; l <= L; l++)
          b[l - m] = sp[3 * nvec + c][(size_t)k * o->jmax + calo_j(l, mm)];
      }
    int nsg = (m == 0) ? 1 : 2;
    for (int i = 0; i < nh + (nth & 1); i++) {
      int ii = nth - 1 - i;           /* mirror node */
      int mid = (ii == i);
      const double *Pi = P + (size_t)i * nl, *dPi = dP + (size_t)i * nl;
      double am = (double)m * o->asin_t[i];
      for (int v = 0; v < nvec; v++) {
        for (int s = 0; s < nsg; s++) {
          /* s = 0: order +m, s = 1: order -m */
          const double *bS = buf + ((3 * v + 0) * 2 + s) * (L + 1);
          const double *bD = buf + ((3 * v + 1) * 2 + s) * (L + 1);
          const double *bT = buf + ((3 * v + 2) * 2 + s) * (L + 1);
          const double *bDo = buf + ((3 * v + 1) * 2 + (1 - s)) * (L + 1);
          const double *bTo = buf + ((3 * v + 2) * 2 + (1 - s)) * (L + 1);
          double re[2] = {0, 0}, te[2] = {0, 0}, pe[2] = {0, 0};
          double tm[2] = {0, 0}, pm_[2] = {0, 0};
          for (int t = 0; t < nl; t++) {
            int par = t & 1;
            re[par] += bS[t] * Pi[t];
            te[par] += bD[t] * dPi[t];
            pe[par] += bT[t] * dPi[t];
            if (m > 0) {
              tm[par] += bTo[t] * Pi[t];
              pm_[par] += bDo[t] * Pi[t];
            }
          }
          /* sign of the mirror term: order +m gets +m P/sin from -m data,
           * order -m gets -m P/sin from +m data */
          double sg = (s == 0) ? am : -am;
          int slot = (s == 0 ? m : -m) + L;
          double *fr = four + (size_t)(3 * v + 0) * cs;
          double *ft = four + (size_t)(3 * v + 1) * cs;
          double *fp = four + (size_t)(3 * v + 2) * cs;
          fr[(size_t)i * ns + slot] = re[0] + re[1];
          ft[(size_t)i * ns + slot] = (te[0] + te[1]) + sg * (tm[0] + tm[1]);
          fp[(size_t)i * ns + slot] = -(pe[0] + pe[1]) + sg * (pm_[0] + pm_[1]);
          if (!mid) {
            fr[(size_t)ii * ns + slot] = re[0] - re[1];
            ft[(size_t)ii * ns + slot] = (-te[0] + te[1]) + sg * (tm[0] - tm[1]);
            fp[(size_t)ii * ns + slot] = -(-pe[0] + pe[1]) + sg * (pm_[0] - pm_[1]);
          }
        }
      }
      for (int c = 0; c < nscal; c++)
        for (int s = 0; s < nsg; s++) {
          const double *b = buf + ((3 * nvec + c) * 2 + s) * (L + 1);
          double e[2] = {0, 0};
          for (int t = 0; t < nl; t++) e[t & 1] += b[t] * Pi[t];
          int slot = (s == 0 ? m : -m) + L;
          double *f = four + (size_t)(3 * nvec + c) * cs;
          f[(size_t)i * ns + slot] = e[0] + e[1];
          if (!mid) f[(size_t)ii * ns + slot] = e[0] - e[1];
        }
    }
  }
  free(buf);
}

/* Forward Legendre transform at one radius
 * (legendre_fwd_trans_org.f90:45-169); output sp[c][k*jmax + j]. */
static void leg_fwd_k(const cal_oracle *o, int k, int nvec, int nscal,
                      const double *four, double *const *sp) {
  int L = o->L, nth = o->nth, ns = 2 * L + 1, nh = nth / 2;
  int ncomp = 3 * nvec + nscal;
  size_t cs = (size_t)nth * ns;
  double r = o->r[k], r2 = r * r;
  int nhm = nh + (nth & 1);
  /* weighted symmetric / antisymmetric halves: [c][slot][i][2] */
  double *h = malloc((size_t)ncomp * ns * nhm * 2 * sizeof(double));
  for (int c = 0; c < ncomp; c++)
    for (int sl = 0; sl < ns; sl++)
      for (int i = 0; i < nhm; i++) {
        int ii = nth - 1 - i;
        double w = o->wgt[i];
        double fa = four[(size_t)c * cs + (size_t)i * ns + sl] * w;
        double *hh = h + (((size_t)c * ns + sl) * nhm + i) * 2;
        if (ii == i) { hh[0] = fa; hh[1] = fa; continue; }
        double fb = four[(size_t)c * cs + (size_t)ii * ns + sl] * o->wgt[ii];
        hh[0] = fa + fb;   /* pairs with even-parity functions */
        hh[1] = fa - fb;   /* pairs with odd-parity functions  */
      }
  for (int m = 0; m <= L; m++) {
    int nl = L + 1 - m;
    const double *P = o->pm[m], *dP = o->dpm[m];
    int nsg = (m == 0) ? 1 : 2;
    for (int t = 0; t < nl; t++) {
      int l = m + t, par = t & 1;
      for (int s = 0; s < nsg; s++) {
        int mm = s ? -m : m;
        int j = calo_j(l, mm);
        int ip = mm + L, in = -mm + L;
        double g7 = o->g7[j], g6 = o->g6[j];
        for (int v = 0; v < nvec; v++) {
          const double *hr = h + ((size_t)(3 * v + 0) * ns + ip) * nhm * 2;
          const double *htp = h + ((size_t)(3 * v + 1) * ns + ip) * nhm * 2;
          const double *htn = h + ((size_t)(3 * v + 1) * ns + in) * nhm * 2;
          const double *hpp = h + ((size_t)(3 * v + 2) * ns + ip) * nhm * 2;
          const double *hpn = h + ((size_t)(3 * v + 2) * ns + in) * nhm * 2;
          double s1 = 0, s2 = 0, s3 = 0;
          for (int i = 0; i < nhm; i++) {
            double p = P[(size_t)i * nl + t], dp = dP[(size_t)i * nl + t];
            double pg = p * (double)mm * o->asin_t[i];
            /* P(pi-theta) = (-1)^(l-m) P, dP(pi-theta) = -(-1)^(l-m) dP */
            s1 += hr[2 * i + par] * p;
            s2 += htp[2 * i + (1 - par)] * dp - hpn[2 * i + par] * pg;
            s3 -= htn[2 * i + par] * pg + hpp[2 * i + (1 - par)] * dp;
          }
          size_t a = (size_t)k * o->jmax + j;
          sp[3 * v + 0][a] = s1 * g7 * r2;
          sp[3 * v + 1][a] = s2 * g7 * r;
          sp[3 * v + 2][a] = s3 * g7 * r;
        }
        for (int c = 0; c < nscal; c++) {
          const double *hs = h + ((size_t)(3 * nvec + c) * ns + ip) * nhm * 2;
          double s1 = 0;
          for (int i = 0; i < nhm; i++) s1 += hs[2 * i + par] * P[(size_t)i * nl + t];
          sp[3 * nvec + c][(size_t)k * o->jmax + j] = s1 * g6;
        }
      }
    }
  }
  free(h);
}

/* Fourier array (ncomp x nth x (2L+1)) <-> grid rows (ncomp x nth x nph) */
static void four_to_grid_rows(const cal_oracle *o, int ncomp, const double *four,
                              double *grid, double *wa, double *wb) {
  int L = o->L, nth = o->nth, ns = 2 * L + 1, n = o->nph;
  double *a0 = wa, *b0 = wa + (L + 1), *a1 = wb, *b1 = wb + (L + 1);
  double *dummy = malloc(n * sizeof(double));
  for (int c = 0; c < ncomp; c += 2) {
    for (int i = 0; i < nth; i++) {
      const double *f0 = four + ((size_t)c * nth + i) * ns;
      const double *f1 = (c + 1 < ncomp) ? four + ((size_t)(c + 1) * nth + i) * ns : NULL;
      for (int m = 0; m <= L; m++) {
        a0[m] = f0[m + L]; b0[m] = (m > 0) ? f0[-m + L] : 0.0;
        a1[m] = f1 ? f1[m + L] : 0.0;
        b1[m] = (f1 && m > 0) ? f1[-m + L] : 0.0;
      }
      double *x0 = grid + ((size_t)c * nth + i) * n;
      double *x1 = f1 ? grid + ((size_t)(c + 1) * nth + i) * n : dummy;
      calo_fourier_to_grid2(o->fft_plan, n, L, a0, b0, a1, b1, x0, x1);
    }
  }
  free(dummy);
}

static void grid_to_four_rows(const cal_oracle *o, int ncomp, const double *grid,
                              double *four, double *wa, double *wb) {
  int L = o->L, nth = o->nth, ns = 2 * L + 1, n = o->nph;
  double *a0 = wa, *b0 = wa + (L + 1), *a1 = wb, *b1 = wb + (L + 1);
  double *zero = calloc(n, sizeof(double));
  for (int c = 0; c < ncomp; c += 2) {
    for (int i = 0; i < nth; i++) {
      const double *x0 = grid + ((size_t)c * nth + i) * n;
      const double *x1 = (c + 1 < ncomp) ? grid + ((size_t)(c + 1) * nth + i) * n : zero;
      calo_grid_to_fourier2(o->fft_plan, n, L, x0, x1, a0, b0, a1, b1);
      double *f0 = four + ((size_t)c * nth + i) * ns;
      for (int m = 0; m <= L; m++) {
        f0[m + L] = a0[m];
        if (m > 0) f0[-m + L] = b0[m];
      }
      if (c + 1 < ncomp) {
        double *f1 = four + ((size_t)(c + 1) * nth + i) * ns;
        for (int m = 0; m <= L; m++) {
          f1[m + L] = a1[m];
          if (m > 0) f1[-m + L] = b1[m];
        }
      }
    }
  }
  free(zero);
}

int calo_sht_backward(cal_oracle *o, int nvec, int nscal,
                      const double *spec, double *grid) {
  int ncomp = 3 * nvec + nscal, nth = o->nth, nph = o->nph, L = o->L;
  size_t fs = (size_t)o->nr * o->jmax;
  const double **sp = malloc(ncomp * sizeof(double *));
  for (int c = 0; c < ncomp; c++) sp[c] = spec + c * fs;
#pragma omp parallel
  {
    double *four = malloc((size_t)ncomp * nth * (2 * L + 1) * sizeof(double));
    double *g = malloc((size_t)ncomp * nth * nph * sizeof(double));
    double *wa = malloc(2 * (L + 1) * sizeof(double)), *wb = malloc(2 * (L + 1) * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < o->nr; k++) {
      leg_bwd_k(o, k, nvec, nscal, sp, four);
      four_to_grid_rows(o, ncomp, four, g, wa, wb);
      for (int c = 0; c < ncomp; c++)
        memcpy(grid + ((size_t)c * o->nr + k) * nth * nph, g + (size_t)c * nth * nph,
               (size_t)nth * nph * sizeof(double));
    }
    free(four); free(g); free(wa); free(wb);
  }
  free(sp);
  return 0;
}

int calo_sht_forward(cal_oracle *o, int nvec, int nscal,
                     const double *grid, double *spec) {
  int ncomp = 3 * nvec + nscal, nth = o->nth, nph = o->nph, L = o->L;
  size_t fs = (size_t)o->nr * o->jmax;
  double **sp = malloc(ncomp * sizeof(double *));
  for (int c = 0; c < ncomp; c++) {
    sp[c] = spec + c * fs;
    memset(sp[c], 0, fs * sizeof(double));
  }
#pragma omp parallel
  {
    double *four = malloc((size_t)ncomp * nth * (2 * L + 1) * sizeof(double));
    double *g = malloc((size_t)ncomp * nth * nph * sizeof(double));
    double *wa = malloc(2 * (L + 1) * sizeof(double)), *wb = malloc(2 * (L + 1) * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < o->nr; k++) {
      for (int c = 0; c < ncomp; c++)
        memcpy(g + (size_t)c * nth * nph, grid + ((size_t)c * o->nr + k) * nth * nph,
               (size_t)nth * nph * sizeof(double));
      grid_to_four_rows(o, ncomp, g, four, wa, wb);
      leg_fwd_k(o, k, nvec, nscal, four, sp);
    }
    free(four); free(g); free(wa); free(wb);
  }
  free(sp);
  return 0;
}

/* The two halves of calo_sht_backward / calo_sht_forward on their own, for
 * the Legendre-only and FFT-only entry points (legendre_transform_select.f90:
 * 309-439, MHD_FFT_selector.F90:185-249).  Fourier arrays are
 * four[c][k][i][m + L], m = -L..L (m < 0: the sin(|m| phi) coefficient);
 * grids grid[c][k][i][p]. */
int calo_leg_backward(cal_oracle *o, int nvec, int nscal, const double *spec, double *four) {
  int ncomp = 3 * nvec + nscal, nth = o->nth, L = o->L, nr = o->nr;
  size_t fs = (size_t)nr * o->jmax, cs = (size_t)nth * (2 * L + 1);
  const double **sp = malloc(ncomp * sizeof(double *));
  for (int c = 0; c < ncomp; c++) sp[c] = spec + c * fs;
#pragma omp parallel
  {
    double *f = malloc((size_t)ncomp * cs * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < nr; k++) {
      leg_bwd_k(o, k, nvec, nscal, sp, f);
      for (int c = 0; c < ncomp; c++)
        memcpy(four + ((size_t)c * nr + k) * cs, f + (size_t)c * cs, cs * sizeof(double));
    }
    free(f);
  }
  free(sp);
  return 0;
}

int calo_leg_forward(cal_oracle *o, int nvec, int nscal, const double *four, double *spec) {
  int ncomp = 3 * nvec + nscal, nth = o->nth, L = o->L, nr = o->nr;
  size_t fs = (size_t)nr * o->jmax, cs = (size_t)nth * (2 * L + 1);
  double **sp = malloc(ncomp * sizeof(double *));
  for (int c = 0; c < ncomp; c++) {
    sp[c] = spec + c * fs;
    memset(sp[c], 0, fs * sizeof(double));
  }
#pragma omp parallel
  {
    double *f = malloc((size_t)ncomp * cs * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < nr; k++) {
      for (int c = 0; c < ncomp; c++)
        memcpy(f + (size_t)c * cs, four + ((size_t)c * nr + k) * cs, cs * sizeof(double));
      leg_fwd_k(o, k, nvec, nscal, f, sp);
    }
    free(f);
  }
  free(sp);
  return 0;
}

int calo_fft_backward(cal_oracle *o, int ncomp, const double *four, double *grid) {
  int nth = o->nth, nph = o->nph, L = o->L, nr = o->nr;
  size_t cs = (size_t)nth * (2 * L + 1), gs = (size_t)nth * nph;
#pragma omp parallel
  {
    double *f = malloc((size_t)ncomp * cs * sizeof(double));
    double *g = malloc((size_t)ncomp * gs * sizeof(double));
    double *wa = malloc(2 * (L + 1) * sizeof(double)), *wb = malloc(2 * (L + 1) * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < nr; k++) {
      for (int c = 0; c < ncomp; c++)
        memcpy(f + (size_t)c * cs, four + ((size_t)c * nr + k) * cs, cs * sizeof(double));
      four_to_grid_rows(o, ncomp, f, g, wa, wb);
      for (int c = 0; c < ncomp; c++)
        memcpy(grid + ((size_t)c * nr + k) * gs, g + (size_t)c * gs, gs * sizeof(double));
    }
    free(f); free(g); free(wa); free(wb);
  }
  return 0;
}

int calo_fft_forward(cal_oracle *o, int ncomp, const double *grid, double *four) {
  int nth = o->nth, nph = o->nph, L = o->L, nr = o->nr;
  size_t cs = (size_t)nth * (2 * L + 1), gs = (size_t)nth * nph;
#pragma omp parallel
  {
    double *f = malloc((size_t)ncomp * cs * sizeof(double));
    double *g = malloc((size_t)ncomp * gs * sizeof(double));
    double *wa = malloc(2 * (L + 1) * sizeof(double)), *wb = malloc(2 * (L + 1) * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < nr; k++) {
      for (int c = 0; c < ncomp; c++)
        memcpy(g + (size_t)c * gs, grid + ((size_t)c * nr + k) * gs, gs * sizeof(double));
      grid_to_four_rows(o, ncomp, g, f, wa, wb);
      for (int c = 0; c < ncomp; c++)
        memcpy(four + ((size_t)c * nr + k) * cs, f + (size_t)c * cs, cs * sizeof(double));
    }
    free(f); free(g); free(wa); free(wb);
  }
  return 0;
}

/* Nonlinear terms by the pseudo-spectral method (F/MHD_src/sph_MHD/
 * cal_nonlinear.f90 nonlinear_by_pseudo_sph, sph_transforms_4_MHD.f90,
 * cal_nonlinear_sph_MHD.f90:35-84, F/SERIAL_src/BASE/cal_products_smp.f90):
 *   backward: u, w, B, J (vectors), T (scalar)
 *   products: m_advect = c_v (w x u), lorentz = c_L (J x B),
 *             vp_induct = c_i (u x B), h_flux = c_T u T
 *   forward:  the four product vectors into rj. */
int calo_nonlinear_transforms(cal_oracle *o) {
  int L = o->L, nth = o->nth, nph = o->nph, ns = 2 * L + 1;
  const double *sp[13];
  for (int c = 0; c < 3; c++) {
    sp[c] = o->f[CALO_VELO + c];
    sp[3 + c] = o->f[CALO_VORT + c];
    sp[6 + c] = o->f[CALO_MAGNE + c];
    sp[9 + c] = o->f[CALO_CURRENT + c];
  }
  sp[12] = o->f[CALO_TEMP];
  double *out[12];
  for (int c = 0; c < 3; c++) {
    out[c] = o->f[CALO_MADV + c];
    out[3 + c] = o->f[CALO_LOR + c];
    out[6 + c] = o->f[CALO_VPIND + c];
    out[9 + c] = o->f[CALO_HFLUX + c];
  }
  double cv = o->p.coef_velo, cl = o->p.coef_lor, ci = o->p.coef_induct;
  double ct = o->p.coef_temp;
#pragma omp parallel
  {
    double *fin = malloc((size_t)13 * nth * ns * sizeof(double));
    double *fout = malloc((size_t)12 * nth * ns * sizeof(double));
    double *g = malloc((size_t)13 * nph * sizeof(double));
    double *q = malloc((size_t)12 * nph * sizeof(double));
    double *wa = malloc(2 * (L + 1) * sizeof(double)), *wb = malloc(2 * (L + 1) * sizeof(double));
    double *wc = malloc(2 * (L + 1) * sizeof(double)), *wd = malloc(2 * (L + 1) * sizeof(double));
#pragma omp for schedule(dynamic)
    for (int k = 0; k < o->nr; k++) {
      leg_bwd_k(o, k, 4, 1, sp, fin);
      for (int i = 0; i < nth; i++) {
        /* Fourier -> grid for the 13 components of this (k, theta) row */
        for (int c = 0; c < 13; c += 2) {
          const double *f0 = fin + ((size_t)c * nth + i) * ns;
          const double *f1 = (c + 1 < 13) ? fin + ((size_t)(c + 1) * nth + i) * ns : NULL;
          for (int m = 0; m <= L; m++) {
            wa[m] = f0[m + L]; wa[L + 1 + m] = (m > 0) ? f0[-m + L] : 0.0;
            wb[m] = f1 ? f1[m + L] : 0.0;
            wb[L + 1 + m] = (f1 && m > 0) ? f1[-m + L] : 0.0;
          }
          calo_fourier_to_grid2(o->fft_plan, nph, L, wa, wa + L + 1, wb, wb + L + 1,
                                g + (size_t)c * nph, (c + 1 < 13) ? g + (size_t)(c + 1) * nph : q);
        }
        const double *ur = g, *ut = g + nph, *up = g + 2 * nph;
        const double *wr = g + 3 * nph, *wt = g + 4 * nph, *wp = g + 5 * nph;
        const double *br = g + 6 * nph, *bt = g + 7 * nph, *bp = g + 8 * nph;
        const double *jr = g + 9 * nph, *jt = g + 10 * nph, *jp = g + 11 * nph;
        const double *tt = g + 12 * nph;
        for (int p = 0; p < nph; p++) {
          q[0 * nph + p] = (wt[p] * up[p] - wp[p] * ut[p]) * cv;
          q[1 * nph + p] = (wp[p] * ur[p] - wr[p] * up[p]) * cv;
          q[2 * nph + p] = (wr[p] * ut[p] - wt[p] * ur[p]) * cv;
          q[3 * nph + p] = (jt[p] * bp[p] - jp[p] * bt[p]) * cl;
          q[4 * nph + p] = (jp[p] * br[p] - jr[p] * bp[p]) * cl;
          q[5 * nph + p] = (jr[p] * bt[p] - jt[p] * br[p]) * cl;
          q[6 * nph + p] = (ut[p] * bp[p] - up[p] * bt[p]) * ci;
          q[7 * nph + p] = (up[p] * br[p] - ur[p] * bp[p]) * ci;
          q[8 * nph + p] = (ur[p] * bt[p] - ut[p] * br[p]) * ci;
          q[9 * nph + p] = ur[p] * tt[p] * ct;
          q[10 * nph + p] = ut[p] * tt[p] * ct;
          q[11 * nph + p] = up[p] * tt[p] * ct;
        }
        for (int c = 0; c < 12; c += 2) {
          calo_grid_to_fourier2(o->fft_plan, nph, L, q + (size_t)c * nph,
                                q + (size_t)(c + 1) * nph, wa, wa + L + 1, wb, wb + L + 1);
          double *f0 = fout + ((size_t)c * nth + i) * ns;
          double *f1 = fout + ((size_t)(c + 1) * nth + i) * ns;
          for (int m = 0; m <= L; m++) {
            f0[m + L] = wa[m]; f1[m + L] = wb[m];
            if (m > 0) { f0[-m + L] = wa[L + 1 + m]; f1[-m + L] = wb[L + 1 + m]; }
          }
        }
      }
      leg_fwd_k(o, k, 4, 0, fout, out);
    }
    free(fin); free(fout); free(g); free(q); free(wa); free(wb); free(wc); free(wd);
  }
  return 0;
}
