/*
 * oracle_gaunt.c -- Gaunt and Elsasser integrals of Schmidt harmonics and the
 * Coriolis coupling coefficients of the CPU oracle (test infrastructure).
 *
 * The reference evaluates the Adams-Gaunt sum exactly through prime
 * factorisations (F/SERIAL_src/spherical_harmonics/normgi_by_primes.f90
 * gs_prime).  Here the same sum is evaluated with factorials in 80-bit
 * long double, which holds 514! without overflow and keeps ~19 digits.
 */
#include <math.h>
#include <stdlib.h>

#include "oracle_internal.h"

static long double fact(int n) {
  long double f = 1.0L;
  for (int i = 2; i <= n; i++) f *= (long double)i;
  return f;
}

/* gs(m1,l1,m2,l2,m3,l3), m1 = m2 + m3 >= 0
 * (F/SERIAL_src/spherical_harmonics/normgi_by_primes.f90:70-190) */
static double gs(int m1, int l1, int m2, int l2, int m3, int l3) {
  int is = (l1 + l2 + l3) / 2;
  int itmax = l1 - m1;
  if (l3 - m3 < itmax) itmax = l3 - m3;
  if (l2 + l3 - m1 < itmax) itmax = l2 + l3 - m1;
  int itmin = l2 - l3 + m1;
  if (l1 + m1 < itmin) itmin = l1 + m1;
  if (0 < itmin) itmin = 0;
  itmin = -itmin;
  long double gi = fact(2 * is - 2 * l3) * fact(is)
                 / (fact(is - l1) * fact(is - l2) * fact(is - l3) * fact(2 * is + 1));
  long double gsi = fact(l1 - m1) * fact(l2 + m2) * fact(l3 + m3) * fact(l3 - m3)
                  / (fact(l1 + m1) * fact(l2 - m2));
  long double sq = sqrtl(gsi);
  long double tsum = 0.0L;
  for (int t = itmin; t <= itmax; t++) {
    long double ti = fact(l1 + m1 + t) * fact(l2 + l3 - m1 - t)
                   / (fact(l1 - m1 - t) * fact(l2 - l3 + m1 + t)
                      * fact(l3 - m3 - t) * fact(t));
    long double term = gi * ti * sq;
    tsum += (t % 2 == 0) ? term : -term;
  }
  int e = is - l2 - m3;
  long double g = ((e % 2 == 0) ? 1.0L : -1.0L) * 2.0L * tsum;
  if (m1 != 0) g *= sqrtl(2.0L);
  if (m2 != 0) g *= sqrtl(2.0L);
  if (m3 != 0) g *= sqrtl(2.0L);
  return (double)g;
}

/* (F/SERIAL_src/spherical_harmonics/cal_gaunt_itgs.f90:107-130) */
static double normki(double gi, int m1, int m2, int m3) {
  if (m1 * m2 * m3 > 0) {
    if (m2 < 0 && m3 < 0) return -gi * 0.5;
    return gi * 0.5;
  } else if (m2 == 0 && m1 * m3 > 0) {
    return gi;
  } else if (m3 == 0 && m2 * m1 > 0) {
    return gi;
  } else if (m3 == 0 && m2 == 0 && m1 == 0) {
    return 2.0 * gi;
  }
  return 0.0;
}

/* (F/SERIAL_src/spherical_harmonics/cal_gaunt_itgs.f90:134-155) */
static double normli(double ei, int m1, int m2, int m3, int mm1) {
  if (m1 * m2 * m3 < 0) {
    if (m3 > 0 && m2 > 0) return ei * 0.5;
    return -ei * 0.5;
  } else if (m2 == 0 && m1 * m3 < 0) {
    return -(double)(m1 / mm1) * ei;
  } else if (m3 == 0 && m2 * m1 < 0) {
    return -(double)(m1 / mm1) * ei;
  }
  return 0.0;
}

/* (F/SERIAL_src/spherical_harmonics/normei.f90 leades) */
static double leades(int m2, int l2, int m3, int l3, const double gg[4]) {
  double a1 = (double)((l2 + m2) * (l3 - m3));
  double a2 = (double)((l3 + m3) * (l2 - m2));
  double a3 = (double)((l2 + m2 - 1) * (l3 + m3 + 1));
  double a4 = (double)((l3 + m3 - 1) * (l2 + m2 + 1));
  double a5 = (double)((l2 - m2) * (l3 - m3));
  if (m2 - 1 == 0) a3 = a3 * 2.0;
  if (m3 == 0) { a3 = a3 * 0.5; a4 = a4 * 0.5; }
  if (m2 == 0) { a3 = a3 * 0.5; a4 = a4 * 0.5; }
  if (m3 - 1 == 0) a4 = a4 * 2.0;
  return -(sqrt(a1) * (sqrt(a3) * gg[0] + sqrt(a5) * gg[1])
           - sqrt(a2) * (sqrt(a4) * gg[2] + sqrt(a5) * gg[3])) * 0.5;
}

/* Elsasser integral through Gaunt integrals (F/SERIAL_src/spherical_harmonics/normei.f90 setei) */
static double setei(int l1, int m1, int l2, int m2, int l3, int m3) {
  double gg[4];
  if (l2 == l3 && m2 == m3) return 0.0;
  if ((m3 + 1) > l3 || abs(m2 - 1) > (l2 - 1)) gg[0] = 0.0;
  else if (m2 == 0) gg[0] = -gs(m3 + 1, l3, 1, l2 - 1, m1, l1);
  else gg[0] = gs(m1, l1, m2 - 1, l2 - 1, m3 + 1, l3);
  if (m2 > (l2 - 1)) gg[1] = 0.0;
  else gg[1] = gs(m1, l1, m2, l2 - 1, m3, l3);
  if ((m2 + 1) > l2 || abs(m3 - 1) > (l3 - 1)) gg[2] = 0.0;
  else if (m3 == 0) gg[2] = -gs(m2 + 1, l2, 1, l3 - 1, m1, l1);
  else gg[2] = gs(m1, l1, m2 + 1, l2, m3 - 1, l3 - 1);
  if (m3 > (l3 - 1)) gg[3] = 0.0;
  else gg[3] = gs(m1, l1, m2, l2, m3, l3 - 1);
  return leades(m2, l2, m3, l3, gg);
}

/* Gaunt integral K (F/SERIAL_src/spherical_harmonics/cal_gaunt_itgs.f90:50-79) */
double calo_leadki(int l1, int m1, int l2, int m2, int l3, int m3) {
  if (!(l1 + l2 >= l3 && l2 + l3 >= l1 && l3 + l1 >= l2)) return 0.0;
  if ((l1 + l2 + l3) % 2 != 0) return 0.0;
  if (!((m1 + m2 + m3) == 0 || (m1 + m2 - m3) == 0 || (m1 - m2 + m3) == 0
        || (-m1 + m2 + m3) == 0)) return 0.0;
  int mm1 = abs(m1), mm2 = abs(m2), mm3 = abs(m3);
  if (mm1 == mm2 + mm3) return normki(gs(mm1, l1, mm2, l2, mm3, l3), m1, m2, m3);
  if (mm2 == mm1 + mm3) return normki(gs(mm2, l2, mm1, l1, mm3, l3), m2, m1, m3);
  if (mm3 == mm2 + mm1) return normki(gs(mm3, l3, mm2, l2, mm1, l1), m3, m2, m1);
  return 0.0;
}

/* Elsasser integral L (F/SERIAL_src/spherical_harmonics/cal_gaunt_itgs.f90:81-104) */
double calo_leadli(int l1, int m1, int l2, int m2, int l3, int m3) {
  if (!(l1 + l2 >= l3 && l2 + l3 >= l1 && l3 + l1 >= l2)) return 0.0;
  if ((l1 + l2 + l3) % 2 != 1) return 0.0;
  if (!((m1 + m2 + m3) == 0 || (m1 + m2 - m3) == 0 || (m1 - m2 + m3) == 0
        || (-m1 + m2 + m3) == 0)) return 0.0;
  int mm1 = abs(m1), mm2 = abs(m2), mm3 = abs(m3);
  if (mm1 == mm2 + mm3)
    return normli(setei(l1, mm1, l2, mm2, l3, mm3), m1, m2, m3, mm1);
  if (mm2 == mm1 + mm3)
    return -normli(setei(l2, mm2, l1, mm1, l3, mm3), m2, m1, m3, mm2);
  if (mm3 == mm2 + mm1)
    return -normli(setei(l3, mm3, l2, mm2, l1, mm1), m3, m2, m1, mm3);
  return 0.0;
}

/* Coriolis couplings (F/MHD_src/sph_MHD/interact_coriolis_rlm.f90:35-178) */
int calo_setup_coriolis(cal_oracle *o) {
  int jmax = o->jmax, L = o->L;
  o->jgi1 = malloc(jmax * sizeof(int));
  o->jgi2 = malloc(jmax * sizeof(int));
  o->jei1 = malloc(jmax * sizeof(int));
  o->gi1 = calloc(jmax, sizeof(double));
  o->gi2 = calloc(jmax, sizeof(double));
  o->ei1 = calloc(jmax, sizeof(double));
  for (int i = 0; i < 6; i++) o->sw[i] = calloc(jmax, sizeof(double));
  for (int i = 0; i < 8; i++) o->tw[i] = calloc(jmax, sizeof(double));
#pragma omp parallel for schedule(dynamic, 16)
  for (int j = 0; j < jmax; j++) {
    int l3 = o->jl[j], m3 = o->jm[j];
    int lk1, mk1, lk2, mk2, ll1 = l3, ml1 = m3;
    int l2 = l3 - 1;
    if (l2 >= 1 && l2 <= L && abs(m3) <= l2) {
      o->gi1[j] = calo_leadki(1, 0, l2, m3, l3, m3);
      lk1 = l2; mk1 = m3;
    } else {
      o->gi1[j] = 0.0;
      lk1 = l3; mk1 = m3;
    }
    l2 = l3 + 1;
    if (l2 >= 1 && l2 <= L && abs(m3) <= l2) {
      o->gi2[j] = calo_leadki(1, 0, l2, m3, l3, m3);
      lk2 = l2; mk2 = m3;
    } else {
      o->gi2[j] = 0.0;
      lk2 = l3; mk2 = m3;
    }
    if (l3 >= 1) {
      o->ei1[j] = calo_leadli(1, 0, l3, -m3, l3, m3);
      ll1 = l3; ml1 = -m3;
    }
    if (j == 0) {
      lk1 = mk1 = lk2 = mk2 = ll1 = ml1 = 0;
      o->gi2[j] = 0.0;
      o->ei1[j] = 0.0;
    }
    o->jgi1[j] = calo_j(lk1, mk1);
    o->jgi2[j] = calo_j(lk2, mk2);
    o->jei1[j] = calo_j(ll1, ml1);
  }
  for (int j = 0; j < jmax; j++) {
    int l = o->jl[j];
    double g3 = o->g3rlm[j], g4 = (double)((l - 1) * l), g5 = (double)((l + 1) * (l + 2));
    double g17 = o->g17[j], gi1 = o->gi1[j], gi2 = o->gi2[j], ei1 = o->ei1[j];
    o->sw[0][j] = (2.0 - g4 - g3) * gi1 * g17;                    /* sw11 */
    o->sw[1][j] = (2.0 - g5 - g3) * gi2 * g17;                    /* sw21 */
    o->sw[2][j] = g4 * (2.0 - g4 + g3) * gi1 * g17 * 0.5;         /* sw12 */
    o->sw[3][j] = g5 * (2.0 - g5 + g3) * gi2 * g17 * 0.5;         /* sw22 */
    o->sw[4][j] = 2.0 * ei1 * g17;                                /* sw13 */
    o->sw[5][j] = 0.0;                                            /* sw23 */
    o->tw[4][j] = -(g3 * (2.0 + g4 - g3) + 2.0 * (-2.0 + g4 + g3)) * gi1 * g17 * 0.5; /* tw13 */
    o->tw[5][j] = -(g3 * (2.0 + g5 - g3) + 2.0 * (-2.0 + g5 + g3)) * gi2 * g17 * 0.5; /* tw23 */
    o->tw[6][j] = -(-2.0 + g4 + g3) * gi1 * g17;                  /* tw14 */
    o->tw[7][j] = -(-2.0 + g5 + g3) * gi2 * g17;                  /* tw24 */
    o->tw[0][j] = -2.0 * ei1 * g17;                               /* tw11 */
    o->tw[1][j] = 0.0;                                            /* tw21 */
    o->tw[2][j] = -g3 * ei1 * g17;                                /* tw12 */
    o->tw[3][j] = 0.0;                                            /* tw22 */
  }
  return 0;
}
