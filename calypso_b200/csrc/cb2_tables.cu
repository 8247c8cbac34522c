// cb2_tables.cu -- set-up of the shell: radial grid, finite-difference and
// boundary weights, harmonic normalisations, Gauss nodes, Coriolis couplings
// (host, float64 / 80-bit), and the Schmidt P_l^m tables (GPU, float64).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "cb2_internal.cuh"

namespace cb2 {

// ---------------------------------------------------------------------------
// 3x3 inverse by cofactors (reference: SERIAL_src/BASE/cal_inverse_small_matrix.f90:176)
static void inv33(const double a[3][3], double ainv[3][3]) {
  double det = a[0][0] * (a[1][1] * a[2][2] - a[2][1] * a[1][2])
             - a[0][1] * (a[1][0] * a[2][2] - a[2][0] * a[1][2])
             + a[0][2] * (a[1][0] * a[2][1] - a[2][0] * a[1][1]);
  double adet = 1.0 / det;
  for (int kj = 0; kj < 3; kj++)
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
      ainv[kj][ki] = (((ki + kj) % 2 == 0) ? 1.0 : -1.0) * d * adet;
    }
}

// Gaunt integral by the Adams sum with factorials in 80-bit floating point
// (reference: SERIAL_src/spherical_harmonics/normgi_by_primes.f90 gs_prime,
//  which evaluates the same sum exactly through prime factorisations).
static long double factl(int n) {
  long double f = 1.0L;
  for (int i = 2; i <= n; i++) f *= (long double)i;
  return f;
}

static double gaunt_gs(int m1, int l1, int m2, int l2, int m3, int l3) {
  int is = (l1 + l2 + l3) / 2;
  int itmax = std::min(std::min(l1 - m1, l3 - m3), l2 + l3 - m1);
  int itmin = -std::min(std::min(l2 - l3 + m1, l1 + m1), 0);
  long double gi = factl(2 * is - 2 * l3) * factl(is)
                 / (factl(is - l1) * factl(is - l2) * factl(is - l3) * factl(2 * is + 1));
  long double sq = sqrtl(factl(l1 - m1) * factl(l2 + m2) * factl(l3 + m3) * factl(l3 - m3)
                         / (factl(l1 + m1) * factl(l2 - m2)));
  long double s = 0.0L;
  for (int t = itmin; t <= itmax; t++) {
    long double ti = factl(l1 + m1 + t) * factl(l2 + l3 - m1 - t)
                   / (factl(l1 - m1 - t) * factl(l2 - l3 + m1 + t) * factl(l3 - m3 - t) * factl(t));
    long double term = gi * ti * sq;
    s += (t % 2 == 0) ? term : -term;
  }
  int e = is - l2 - m3;
  long double g = ((e % 2 == 0) ? 2.0L : -2.0L) * s;
  if (m1 != 0) g *= sqrtl(2.0L);
  if (m2 != 0) g *= sqrtl(2.0L);
  if (m3 != 0) g *= sqrtl(2.0L);
  return (double)g;
}

// normalisation of the real-harmonic Gaunt / Elsasser integrals
// (reference: SERIAL_src/spherical_harmonics/cal_gaunt_itgs.f90 normki/normli)
static double norm_k(double gi, int m1, int m2, int m3) {
  if (m1 * m2 * m3 > 0) return (m2 < 0 && m3 < 0) ? -0.5 * gi : 0.5 * gi;
  if (m2 == 0 && m1 * m3 > 0) return gi;
  if (m3 == 0 && m2 * m1 > 0) return gi;
  if (m1 == 0 && m2 == 0 && m3 == 0) return 2.0 * gi;
  return 0.0;
}

static double norm_l(double ei, int m1, int m2, int m3, int mm1) {
  if (m1 * m2 * m3 < 0) return (m3 > 0 && m2 > 0) ? 0.5 * ei : -0.5 * ei;
  if (m2 == 0 && m1 * m3 < 0) return -(double)(m1 / mm1) * ei;
  if (m3 == 0 && m2 * m1 < 0) return -(double)(m1 / mm1) * ei;
  return 0.0;
}

// Elsasser integral from four Gaunt integrals
// (reference: SERIAL_src/spherical_harmonics/normei.f90 setei/leades)
static double elsasser(int l1, int m1, int l2, int m2, int l3, int m3) {
  if (l2 == l3 && m2 == m3) return 0.0;
  double g[4];
  if (m3 + 1 > l3 || std::abs(m2 - 1) > l2 - 1) g[0] = 0.0;
  else if (m2 == 0) g[0] = -gaunt_gs(m3 + 1, l3, 1, l2 - 1, m1, l1);
  else g[0] = gaunt_gs(m1, l1, m2 - 1, l2 - 1, m3 + 1, l3);
  g[1] = (m2 > l2 - 1) ? 0.0 : gaunt_gs(m1, l1, m2, l2 - 1, m3, l3);
  if (m2 + 1 > l2 || std::abs(m3 - 1) > l3 - 1) g[2] = 0.0;
  else if (m3 == 0) g[2] = -gaunt_gs(m2 + 1, l2, 1, l3 - 1, m1, l1);
  else g[2] = gaunt_gs(m1, l1, m2 + 1, l2, m3 - 1, l3 - 1);
  g[3] = (m3 > l3 - 1) ? 0.0 : gaunt_gs(m1, l1, m2, l2, m3, l3 - 1);
  double a1 = (double)((l2 + m2) * (l3 - m3)), a2 = (double)((l3 + m3) * (l2 - m2));
  double a3 = (double)((l2 + m2 - 1) * (l3 + m3 + 1)), a4 = (double)((l3 + m3 - 1) * (l2 + m2 + 1));
  double a5 = (double)((l2 - m2) * (l3 - m3));
  if (m2 == 1) a3 *= 2.0;
  if (m3 == 0) { a3 *= 0.5; a4 *= 0.5; }
  if (m2 == 0) { a3 *= 0.5; a4 *= 0.5; }
  if (m3 == 1) a4 *= 2.0;
  return -(sqrt(a1) * (sqrt(a3) * g[0] + sqrt(a5) * g[1])
           - sqrt(a2) * (sqrt(a4) * g[2] + sqrt(a5) * g[3])) * 0.5;
}

// K(1,0; l2,m; l,m) and L(1,0; l,-m; l,m): the only couplings the Coriolis
// term needs (reference: MHD_src/sph_MHD/interact_coriolis_rlm.f90:35-104
// with cal_gaunt_itgs.f90 leadki/leadli)
static double coriolis_k(int l2, int m, int l3) {
  int am = std::abs(m);
  if (!(1 + l2 >= l3 && l2 + l3 >= 1 && l3 + 1 >= l2) || (1 + l2 + l3) % 2 != 0) return 0.0;
  if (am == 0) return norm_k(gaunt_gs(0, 1, 0, l2, 0, l3), 0, 0, 0);
  return norm_k(gaunt_gs(am, l2, 0, 1, am, l3), m, 0, m);
}

static double coriolis_l(int l3, int m3) {
  int am = std::abs(m3);
  if (l3 < 1) return 0.0;
  if (am == 0) return 0.0;
  return -norm_l(elsasser(l3, am, 1, 0, l3, am), -m3, 0, m3, am);
}

// ---------------------------------------------------------------------------
// Schmidt quasi-normalised P_l^m and dP/dtheta at one colatitude (device)
// (reference: SERIAL_src/spherical_harmonics/schmidt_fix_m.f90:62-175)
__device__ static void d_schmidt_m(int ltr, int m, double th, double *p, double *df) {
  double ct = cos(th), st = sin(th);
  if (m < 0) {
    for (int l = 0; l <= ltr; l++) p[l] = 0.0;
  } else if (m == 0) {
    p[0] = 1.0;
    if (ltr >= 1) p[1] = ct;
    for (int l = 2; l <= ltr; l++)
      p[l] = p[l - 1] * (double)(2 * l - 1) / (double)l * ct - p[l - 2] * (double)(l - 1) / (double)l;
  } else {
    df[m] = 1.0;
    for (int k = 1; k <= m; k++) df[m] = df[m] * (double)(2 * k - 1) / (double)(2 * k);
    df[m + 1] = sqrt(2.0 * df[m] * (double)(2 * m + 1)) * ct;
    df[m] = sqrt(2.0 * df[m]);
    if (m < ltr - 1)
      for (int l = m + 2; l <= ltr; l++)
        df[l] = (ct * (double)(2 * l - 1) * df[l - 1]
                 - sqrt((double)((l - 1) * (l - 1) - m * m)) * df[l - 2])
                / sqrt((double)(l * l - m * m));
    for (int l = m; l <= ltr; l++) {
      double v = df[l];
      for (int m1 = 1; m1 <= m; m1++) v = v * st;
      p[l] = v;
    }
  }
}

// one thread per (m, node i < nh); scratch rows in global memory
__global__ void k_plm(int L, int nh, const double *colat, const size_t *poff,
                      double *scratch, double *Plt, double *dPlt, double *Ptl, double *dPtl) {
  int m = blockIdx.y;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L || i >= nh) return;
  size_t row = (size_t)(m * nh + i) * (4 * (L + 4));
  double *p = scratch + row, *pn = p + (L + 4), *pp = pn + (L + 4), *df = pp + (L + 4);
  double th = colat[i];
  d_schmidt_m(L, m - 1, th, pn, df);
  d_schmidt_m(L, m + 1, th, pp, df);
  d_schmidt_m(L, m, th, p, df);
  int nl = L + 1 - m;
  size_t o = poff[m];
  for (int l = m; l <= L; l++) {
    double dp;
    if (m == 0) {
      dp = (l == 0) ? 0.0 : -sqrt((double)(l * (l + 1) / 2)) * pp[l];
    } else if (m == 1) {
      dp = (l == 1) ? pn[1]
                    : 0.5 * (sqrt((double)(2 * l * (l + 1))) * pn[l]
                             - sqrt((double)((l - 1) * (l + 2))) * pp[l]);
    } else {
      dp = (l == m) ? 0.5 * sqrt((double)(2 * m)) * pn[m]
                    : 0.5 * (sqrt((double)((l + m) * (l - m + 1))) * pn[l]
                             - sqrt((double)((l - m) * (l + m + 1))) * pp[l]);
    }
    Plt[o + (size_t)(l - m) * nh + i] = p[l];
    dPlt[o + (size_t)(l - m) * nh + i] = dp;
    Ptl[o + (size_t)i * nl + (l - m)] = p[l];
    dPtl[o + (size_t)i * nl + (l - m)] = dp;
  }
}

template <typename T>
static int upload(T **dst, const std::vector<T> &v) {
  CB2_CUDA(cudaMalloc(dst, v.size() * sizeof(T)));
  CB2_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

#define UP(dst, v) \
  do { int _r = upload(&(dst), (v)); if (_r) return _r; } while (0)

int setup_tables(Ctx &c) {
  const cb2_params &p = c.p;
  int L = c.L, nr = c.nr, nth = c.nth;
  // index tables, m-major jj ordering
  c.h_moff.assign(L + 2, 0);
  int off = 0;
  for (int m = 0; m <= L; m++) {
    c.h_moff[m] = off;
    off += (m == 0) ? (L + 1) : 2 * (L + 1 - m);
  }
  c.h_moff[L + 1] = off;
  if (off != c.jmax) { set_error("index table size mismatch"); return CB2_ERR_ARG; }
  c.h_jl.assign(c.jmax, 0);
  c.h_jm.assign(c.jmax, 0);
  c.h_perm.assign(c.jmax, 0);
  for (int m = 0; m <= L; m++)
    for (int s = 0; s < (m == 0 ? 1 : 2); s++)
      for (int l = m; l <= L; l++) {
        int jj = c.h_moff[m] + s * (L + 1 - m) + (l - m);
        int mm = s ? -m : m;
        c.h_jl[jj] = l;
        c.h_jm[jj] = mm;
        c.h_perm[jj] = l * (l + 1) + mm;
      }
  // normalisations (reference: SERIAL_src/spherical_harmonics/spherical_harmonics.f90:92-141)
  std::vector<double> g3(c.jmax), g3rlm(c.jmax), gl(c.jmax), g6(c.jmax), g7(c.jmax), g11(c.jmax),
      g12(c.jmax), g17(c.jmax);
  for (int jj = 0; jj < c.jmax; jj++) {
    int l = c.h_jl[jj], m = c.h_jm[jj];
    gl[jj] = l;
    g3[jj] = (double)(l * (l + 1));
    g11[jj] = 1.0 / (double)(2 * l + 1);
    g12[jj] = (double)(l * (l + 1)) / (double)(2 * l + 1);
    if (l == 0) {
      g6[jj] = 0.5; g7[jj] = 1.0; g17[jj] = 0.0; g3rlm[jj] = 0.5;
    } else {
      g17[jj] = (double)(2 * l + 1) / (double)(4 * l * (l + 1));
      g6[jj] = (m == 0) ? (double)(2 * l + 1) / 2.0 : (double)(2 * l + 1) / 4.0;
      g7[jj] = (m == 0) ? (double)(2 * l + 1) / (double)(2 * l * (l + 1))
                        : (double)(2 * l + 1) / (double)(4 * l * (l + 1));
      g3rlm[jj] = g3[jj];
    }
  }
  // radial grid (reference: SERIAL_src/SPH_SPECTR_src/set_radial_grid_sph_shell.f90:40-111)
  std::vector<double> r(nr), ar1(nr), ar2(nr);
  double pi = 4.0 * atan(1.0), shell = p.r_cmb - p.r_icb;
  for (int k = 0; k < nr; k++) {
    r[k] = (p.radial_grid_type == 1)
               ? p.r_icb + 0.5 * shell * (1.0 - cos(pi * (double)k / (double)(nr - 1)))
               : p.r_icb + (p.r_cmb - p.r_icb) * (double)k / (double)(nr - 1);
    ar1[k] = 1.0 / r[k];
    ar2[k] = ar1[k] * ar1[k];
  }
  c.h_r = r;
  // interior FDM (reference: SERIAL_src/SPH_SPECTR_src/set_radius_func_noequi.f90)
  std::vector<double> d1(3 * nr), d2(3 * nr), dr(nr);
  for (int k = 1; k < nr - 1; k++) dr[k] = r[k + 1] - r[k];
  dr[nr - 1] = r[nr - 1] - r[nr - 2];
  dr[0] = r[1] - r[0];
  for (int k = 0; k < nr; k++) {
    double dp = dr[k], dn = (k == 0 || k == nr - 1) ? dr[k] : dr[k - 1];
    double a[3][3] = {{1, 0, 0}, {1, dp, 0.5 * dp * dp}, {1, -dn, 0.5 * dn * dn}}, mi[3][3];
    inv33(a, mi);
    d1[0 * nr + k] = mi[1][2]; d1[1 * nr + k] = mi[1][0]; d1[2 * nr + k] = mi[1][1];
    d2[0 * nr + k] = mi[2][2]; d2[1 * nr + k] = mi[2][0]; d2[2 * nr + k] = mi[2][1];
  }
  // boundary weights (reference: MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90)
  {
    BCW &b = c.bc;
    memset(&b, 0, sizeof(b));
    int ki = c.kin, ko = c.kout;
    double mi[3][3];
    double e1 = r[ki + 1] - r[ki], e2 = r[ki + 2] - r[ki];
    double a1[3][3] = {{1, 0, 0}, {1, e1, e1 * e1 / 2.0}, {1, e2, e2 * e2 / 2.0}};
    inv33(a1, mi);
    for (int q = 0; q < 3; q++) for (int i = 0; i < 3; i++) b.fix_fld_icb[i][q + 1] = mi[q][i];
    double a2[3][3] = {{1, 0, 0}, {0, 1, 0}, {e1, 1, e1 * e1 / 2.0}};
    inv33(a2, mi);
    for (int q = 0; q < 3; q++) for (int i = 0; i < 3; i++) b.fix_dr_icb[i][q + 1] = mi[q][i];
    double f1 = r[ko] - r[ko - 1], f2 = r[ko] - r[ko - 2];
    double a3[3][3] = {{1, 0, 0}, {1, -f1, f1 * f1 / 2.0}, {1, -f2, f2 * f2 / 2.0}};
    inv33(a3, mi);
    for (int q = 0; q < 3; q++) for (int i = 0; i < 3; i++) b.fix_fld_cmb[i][q + 1] = mi[q][i];
    double a4[3][3] = {{1, 0, 0}, {0, 1, 0}, {1, -f1, f1 * f1 / 2.0}};
    inv33(a4, mi);
    for (int q = 0; q < 3; q++) {
      b.fix_dr_cmb[0][q + 1] = mi[q][2];
      b.fix_dr_cmb[1][q + 1] = mi[q][0];
      b.fix_dr_cmb[2][q + 1] = mi[q][1];
    }
    b.r_icb[0] = r[ki]; b.r_icb[1] = ar1[ki]; b.r_icb[2] = ar2[ki];
    b.r_cmb[0] = r[ko]; b.r_cmb[1] = ar1[ko]; b.r_cmb[2] = ar2[ko];
  }
  // reference temperature and rotation (set_reference_sph_mhd.f90, m_poloidal_rotation.f90)
  std::vector<double> reft0(nr, 0.0), reft1(nr, 0.0), om(3 * nr);
  for (int k = 0; k < nr; k++) {
    if (p.use_ref_temp) {
      double dh = p.depth_high_t, dl = p.depth_low_t, ht = p.high_temp, lt = p.low_temp;
      reft0[k] = (dh * dl * ar1[k] * (ht - lt) - dh * ht + dl * lt) / (dl - dh);
      reft1[k] = -dh * dl * ar2[k] * (ht - lt) / (dl - dh);
    }
    om[0 * nr + k] = 0.5 * r[k] * r[k];
    om[1 * nr + k] = r[k];
    om[2 * nr + k] = 1.0;
  }
  c.temp_icb_fld = p.temp_icb - (p.use_ref_temp ? reft0[c.kin] : 0.0);
  c.temp_cmb_fld = p.temp_cmb - (p.use_ref_temp ? reft0[c.kout] : 0.0);
  c.cev = 1.0 - p.coef_imp_v;
  c.cet = 1.0 - p.coef_imp_t;
  c.ceb = 1.0 - p.coef_imp_b;
  // Gauss-Legendre nodes (reference: SERIAL_src/gauss_integration/m_gauss_points.f90:117-210)
  std::vector<double> colat(nth), wgt(nth), asn(nth), x(nth), w(nth);
  for (int i = 1; i <= (nth + 1 - (nth + 1) % 2) / 2; i++) {
    double z = cos(pi * ((double)i - 0.25) / ((double)nth + 0.5)), pp, z1;
    for (;;) {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= nth; j++) {
        p3 = p2; p2 = p1;
        p1 = ((2.0 * (double)j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
      }
      pp = (double)nth * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (fabs(z - z1) < 3.0e-12) break;
    }
    x[i - 1] = 0.5 - 0.5 * z;
    x[nth - i] = 0.5 + 0.5 * z;
    w[i - 1] = 1.0 / ((1.0 - z * z) * pp * pp);
    w[nth - i] = w[i - 1];
  }
  for (int i = 0; i < nth; i++) {
    wgt[i] = w[i] * 2.0;
    colat[i] = acos(x[i] * 2.0 - 1.0);
    asn[i] = 1.0 / sin(colat[i]);
  }
  c.h_colat = colat;
  c.h_wgt = wgt;
  // Coriolis couplings in jj indexing
  std::vector<int> jgi1(c.jmax), jgi2(c.jmax), jei1(c.jmax);
  std::vector<double> sw(6 * (size_t)c.jmax), tw(8 * (size_t)c.jmax);
  auto jj_of = [&](int l, int m) {
    int am = std::abs(m);
    return c.h_moff[am] + ((m < 0) ? (L + 1 - am) : 0) + (l - am);
  };
#pragma omp parallel for schedule(dynamic, 16)
  for (int jj = 0; jj < c.jmax; jj++) {
    int l3 = c.h_jl[jj], m3 = c.h_jm[jj];
    double gi1 = 0.0, gi2 = 0.0, ei1 = 0.0;
    int lk1 = l3, lk2 = l3, ll1 = l3, ml1 = m3;
    if (l3 - 1 >= 1 && std::abs(m3) <= l3 - 1) { gi1 = coriolis_k(l3 - 1, m3, l3); lk1 = l3 - 1; }
    if (l3 + 1 <= L) { gi2 = coriolis_k(l3 + 1, m3, l3); lk2 = l3 + 1; }
    if (l3 >= 1) { ei1 = coriolis_l(l3, m3); ml1 = -m3; }
    if (l3 == 0) { lk1 = lk2 = ll1 = 0; ml1 = 0; gi2 = 0.0; ei1 = 0.0; }
    jgi1[jj] = jj_of(lk1, m3);
    jgi2[jj] = jj_of(lk2, m3);
    jei1[jj] = jj_of(ll1, ml1);
    double G3 = g3rlm[jj], G4 = (double)((l3 - 1) * l3), G5 = (double)((l3 + 1) * (l3 + 2));
    double G17 = g17[jj];
    size_t n = c.jmax;
    sw[0 * n + jj] = (2.0 - G4 - G3) * gi1 * G17;
    sw[1 * n + jj] = (2.0 - G5 - G3) * gi2 * G17;
    sw[2 * n + jj] = G4 * (2.0 - G4 + G3) * gi1 * G17 * 0.5;
    sw[3 * n + jj] = G5 * (2.0 - G5 + G3) * gi2 * G17 * 0.5;
    sw[4 * n + jj] = 2.0 * ei1 * G17;
    sw[5 * n + jj] = 0.0;
    tw[4 * n + jj] = -(G3 * (2.0 + G4 - G3) + 2.0 * (-2.0 + G4 + G3)) * gi1 * G17 * 0.5;
    tw[5 * n + jj] = -(G3 * (2.0 + G5 - G3) + 2.0 * (-2.0 + G5 + G3)) * gi2 * G17 * 0.5;
    tw[6 * n + jj] = -(-2.0 + G4 + G3) * gi1 * G17;
    tw[7 * n + jj] = -(-2.0 + G5 + G3) * gi2 * G17;
    tw[0 * n + jj] = -2.0 * ei1 * G17;
    tw[1 * n + jj] = 0.0;
    tw[2 * n + jj] = -G3 * ei1 * G17;
    tw[3 * n + jj] = 0.0;
  }
  // P table offsets per order
  c.h_poff.assign(L + 2, 0);
  size_t po = 0;
  for (int m = 0; m <= L; m++) {
    c.h_poff[m] = po;
    po += (size_t)(L + 1 - m) * c.nh;
  }
  c.h_poff[L + 1] = po;
  UP(c.d_jl, c.h_jl); UP(c.d_jm, c.h_jm); UP(c.d_perm, c.h_perm); UP(c.d_moff, c.h_moff);
  UP(c.d_g3, g3); UP(c.d_g3rlm, g3rlm); UP(c.d_gl, gl); UP(c.d_g6, g6); UP(c.d_g7, g7);
  UP(c.d_g11, g11); UP(c.d_g12, g12);
  UP(c.d_r, r); UP(c.d_ar1, ar1); UP(c.d_ar2, ar2); UP(c.d_d1, d1); UP(c.d_d2, d2);
  UP(c.d_reft0, reft0); UP(c.d_reft1, reft1); UP(c.d_om, om);
  UP(c.d_colat, colat); UP(c.d_wgt, wgt); UP(c.d_asin, asn);
  UP(c.d_poff, c.h_poff);
  UP(c.d_jgi1, jgi1); UP(c.d_jgi2, jgi2); UP(c.d_jei1, jei1); UP(c.d_sw, sw); UP(c.d_tw, tw);
  // Schmidt tables on the device
  CB2_CUDA(cudaMalloc(&c.d_Plt, po * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_dPlt, po * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_Ptl, po * sizeof(double)));
  CB2_CUDA(cudaMalloc(&c.d_dPtl, po * sizeof(double)));
  size_t sbytes = (size_t)(L + 1) * c.nh * 4 * (L + 4) * sizeof(double);
  double *scratch = nullptr;
  CB2_CUDA(cudaMalloc(&scratch, sbytes));
  dim3 grid(cdiv(c.nh, 64), L + 1);
  k_plm<<<grid, 64, 0, c.stream>>>(L, c.nh, c.d_colat, c.d_poff, scratch, c.d_Plt, c.d_dPlt,
                                   c.d_Ptl, c.d_dPtl);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  CB2_CUDA(cudaFree(scratch));
  return 0;
}

void free_tables(Ctx &c) {
  void *ptrs[] = {c.d_jl, c.d_jm, c.d_perm, c.d_moff, c.d_g3, c.d_g3rlm, c.d_gl, c.d_g6, c.d_g7,
                  c.d_g11, c.d_g12, c.d_r, c.d_ar1, c.d_ar2, c.d_d1, c.d_d2, c.d_reft0, c.d_reft1,
                  c.d_om, c.d_colat, c.d_wgt, c.d_asin, c.d_poff, c.d_Plt, c.d_dPlt, c.d_Ptl,
                  c.d_dPtl, c.d_jgi1, c.d_jgi2, c.d_jei1, c.d_sw, c.d_tw};
  for (void *q : ptrs)
    if (q) cudaFree(q);
}

}  // namespace cb2
