// cb2_cn.cu -- the Crank-Nicolson part of the time step in one pass per
// radial column, float64.
//
// cb2_rj.cu runs it as four passes over the rj fields: the explicit update
// (k_explicit: cal_explicit_sph_adams / cal_first_prev_step_adams of
// MHD_src/sph_MHD/cal_explicit_terms.f90), the banded solves (k_implicit:
// cal_sol_sph_fluid_crank.f90 over lubksb_357band.f90), and the radial
// derivatives of the new state (k_derived_a / k_derived_b:
// const_grad_vp_and_vorticity, const_grad_bp_and_current,
// cal_rot_buoyancy_sph_MHD, const_sph_vorticirty_diffusion,
// const_sph_scalar_diffusion, const_sph_mag_diffuse_by_j).  Every value
// those passes produce at (l, m) depends only on the same (l, m) column of
// one field, so here one thread per (field, column) does all of it:
//
//   forward sweep, rows ascending: the explicit right-hand side b(k) (the
//     expressions of k_explicit, which also store the previous-step forces),
//     then L y = b, y stored in the field's solution slot;
//   backward sweep, rows descending: U x = y, and from the last three rows
//     held in registers the derived fields of the column, one row behind
//     the solve (two rows for the diffusion of the toroidal vorticity, a
//     second derivative of a second derivative).
//
// The solves run the back substitution of lubksb_357band.f90 over the
// pivoted banded LU of m_ludcmp_3band.f90 / m_ludcmp_band.f90, streamed:
//   y(i) = x'(i) - L(i,i-NL) y(i-NL) - ... - L(i,i-1) y(i-1)
//   x(i) = (y(i) - U(i,i+1) x(i+1) - ... - U(i,i+NU) x(i+NU)) / U(i,i)
// where x' is the right-hand side after the row interchanges.  The
// interchange of row i reaches at most row i + 2 (i + 1 for the 3-band
// operators), so the forward sweep applies it to a window of the next
// right-hand-side values held in registers.  Operators whose factorisation
// made no interchange have exactly zero outer bands, and their factors are
// kept in a narrow form (NL = NU = 2, or 1): the same products and sums, in
// the same order, less the products with exact zeros.
#include <algorithm>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

constexpr int CN_THREADS = 256;   // a block: 8 warps, each 32 consecutive degrees of one (m, sign)
constexpr int CN_RING = 4;        // rows each thread keeps in flight (cp.async ring)
constexpr int CN_RV = 4;          // values per ring slot (forward: X, D, F, P; backward: y)

// Forms of one field's factors.  Per row i: NL multipliers L(i,i-1) ..
// L(i,i-NL), NL superdiagonals U(i,i+1) .. U(i,i+NL), then 1 / U(i,i);
// forms with row interchanges also keep, per row, the offset d of the row
// i + d that the factorisation swapped with row i (0 <= d <= PD).
enum CnForm { CN_N5 = 0, CN_W5 = 1, CN_N3 = 2, CN_W3 = 3 };
__host__ __device__ constexpr int cn_nl(int f) { return f == CN_N5 ? 2 : f == CN_W5 ? 4 : f == CN_N3 ? 1 : 2; }
__host__ __device__ constexpr int cn_pd(int f) { return f == CN_W5 ? 2 : f == CN_W3 ? 1 : 0; }
__host__ __device__ constexpr int cn_entries(int f) { return 2 * cn_nl(f) + 1; }

// shared memory of a block: the radial coefficients, then the per-thread rings
__host__ __device__ inline size_t cn_ring_offset(int n) { return 9 * (size_t)n * sizeof(double); }
static size_t cn_smem(int n) {
  return cn_ring_offset(n) + (size_t)CN_RING * CN_RV * CN_THREADS * sizeof(double);
}

struct LuSet {
  const double *lu[5];   // degree-interleaved pivoted band factors (width 9, then 5)
  const int *pv[5];      // degree-interleaved pivots (1-based rows)
};

// the step's view of the factors: per field [row][entry][degree] doubles
// and (forms with interchanges) [row][degree] offsets
struct CnPack {
  const double *fac[5];
  const unsigned char *piv[5];
  int form[5];
};

// entry b (1-based) of band column c (1-based) of one degree's factors
struct BandCol {
  const double *lu;
  int W, nl;
  __device__ double operator()(int b, int c) const { return lu[(size_t)((c - 1) * W + (b - 1)) * nl]; }
};

// one thread per (field, degree).  ok bit 0: no row interchange and the
// outer bands zero (the narrow form holds the factors); bit 1: every
// interchange within the reach of the form with interchanges
__global__ void k_cn_check(int n, int nl, LuSet set, int *ok) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 5 * nl) return;
  const int fld = e / nl, l = e - fld * nl;
  const int W = (fld == 0) ? 9 : 5, H = (W - 1) / 2;
  const BandCol E{set.lu[fld] + l, W, nl};
  const int *pv = set.pv[fld] + l;
  int narrow = 1, wide = 1;
  for (int i = 1; i <= n; i++) {
    const int d = pv[(size_t)(i - 1) * nl] - i;
    if (d != 0) narrow = 0;
    if (d < 0 || d > H / 2) wide = 0;
    // U(., i) beyond the narrow reach: entries 1 .. H - H/2; L(., i) beyond
    // it: entries H + 2 + H/2 .. W
    for (int b = 1; b <= H - H / 2; b++)
      if (E(b, i) != 0.0) narrow = 0;
    for (int b = H + 2 + H / 2; b <= W; b++)
      if (E(b, i) != 0.0) narrow = 0;
  }
  ok[e] = narrow | (wide << 1);
}

// one thread per (field, degree): the factors in the form chosen for the field
__global__ void k_cn_pack(int n, int nl, LuSet set, CnPack pk) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 5 * nl) return;
  const int fld = e / nl, l = e - fld * nl;
  const int W = (fld == 0) ? 9 : 5, H = (W - 1) / 2;
  const int form = pk.form[fld], NL = cn_nl(form), NE = cn_entries(form);
  const BandCol E{set.lu[fld] + l, W, nl};
  const int *pv = set.pv[fld] + l;
  double *o = const_cast<double *>(pk.fac[fld]) + l;
  for (int i = 1; i <= n; i++) {
    double *r = o + (size_t)(i - 1) * NE * nl;
    for (int t = 1; t <= NL; t++) {
      r[(size_t)(t - 1) * nl] = (i - t >= 1) ? E(H + 1 + t, i - t) : 0.0;        // L(i, i-t)
      r[(size_t)(NL + t - 1) * nl] = (i + t <= n) ? E(H + 1 - t, i + t) : 0.0;   // U(i, i+t)
    }
    r[(size_t)2 * NL * nl] = 1.0 / E(H + 1, i);
    if (cn_pd(form))
      const_cast<unsigned char *>(pk.piv[fld])[(size_t)(i - 1) * nl + l] =
          (unsigned char)(pv[(size_t)(i - 1) * nl] - i);
  }
}

// radial coefficients staged in shared memory: d1[3][n], d2[3][n], ar1, ar2, r
struct RadCo {
  const double *c;
  int n;
  __device__ double ar1(int k) const { return c[6 * n + k]; }
  __device__ double ar2(int k) const { return c[7 * n + k]; }
  __device__ double r(int k) const { return c[8 * n + k]; }
  // the three-point first / second derivative at row k (D1 / D2 of cb2_rj.cu)
  __device__ double D1(int k, double f0, double f1, double f2) const {
    return c[k] * f0 + c[n + k] * f1 + c[2 * n + k] * f2;
  }
  __device__ double D2(int k, double f0, double f1, double f2) const {
    return c[3 * n + k] * f0 + c[4 * n + k] * f1 + c[5 * n + k] * f2;
  }
};

// one column of one slot: element k at p[k * st] (k * st < 2^31).  stcs:
// written once (evict-first); stkeep: the forward sweep's y, read back by
// the backward sweep, held in L2 with an evict-last policy
struct Col {
  double *p;
  __device__ void stcs(int k, unsigned s, double v) const { __stcs(p + (unsigned)k * s, v); }
  __device__ void stkeep(int k, unsigned st, double v, uint64_t pol) const {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p + (unsigned)k * st), "d"(v), "l"(pol)
                 : "memory");
  }
};
// 8-byte asynchronous copy global -> shared, and its group bookkeeping
__device__ __forceinline__ void cp8(double *dst, const double *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// this thread's ring: slot s, value v at base[(s * CN_RV + v) * CN_THREADS]
struct Ring {
  double *base;
  __device__ double *at(int s, int v) const { return base + (s * CN_RV + v) * CN_THREADS; }
};

__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// the last three values pushed, in descending rows: v0 = row k, v1 = k + 1, v2 = k + 2
struct Win3 {
  double v0 = 0.0, v1 = 0.0, v2 = 0.0;
  __device__ void push(double v) { v2 = v1; v1 = v0; v0 = v; }
};

// everything a column thread reads besides its slots
struct CnCtx {
  const RJArgs &a;
  RadCo co;
  int n;
  unsigned st;
  int jj;
  double g3, gl;
};

// one degree's factors in global memory (degree-interleaved, so the 32
// lanes of a warp read 32 consecutive values; the block's 8 warps share
// them through L1): entry e of row i at p[(i * NE + e) * nl], the
// interchange offset of row i at pv[i * nl]
struct FacCol {
  const double *p;
  const unsigned char *pv;
  int nl;
  __device__ double at(int i, int ne, int e) const { return __ldg(p + (i * ne + e) * nl); }
  __device__ int piv(int i) const { return __ldg(pv + i * nl); }
};

// ---------------------------------------------------------------------------
// forward sweep: explicit right-hand side and L y = P b.  X, D, F, P: the
// field before the step, its diffusion term, its force and the force of the
// step before (P receives this step's force); S: the solution slot.
// FLD: 0 poloidal velocity (from the toroidal vorticity), 1 toroidal
// velocity (from the poloidal vorticity), 2 temperature, 3 poloidal and
// 4 toroidal magnetic field.  fac: the column's factors.  The
// inputs of row k + CN_RING are copied into the thread's ring while row k
// is computed, so a thread keeps CN_RING rows of loads in flight.
template <int FLD, int FORM>
__device__ __forceinline__ void cn_forward(const CnCtx &q, FacCol fac, Ring ring,
                                           Col X, Col D, Col F, Col P, Col S, int euler) {
  constexpr int NL = cn_nl(FORM), PD = cn_pd(FORM), NE = cn_entries(FORM);
  const RJArgs &a = q.a;
  const int n = q.n;
  const unsigned st = q.st;
  const double adam_0 = 3.0 / 2.0, adam_1 = -1.0 / 2.0, dt = a.dt;
  const double ce = (FLD <= 1) ? a.cev : (FLD == 2) ? a.cet : a.ceb;
  const double fbi = (q.jj == 0) ? a.temp_icb_fld : 0.0, fbo = (q.jj == 0) ? a.temp_cmb_fld : 0.0;
  const uint64_t keep = l2_evict_last();
  auto fetch = [&](int sl, int k) {   // inputs of row k into slot sl (none past the last row)
    if (k < n) {
      const unsigned o = (unsigned)k * st;
      cp8(ring.at(sl, 0), X.p + o);
      cp8(ring.at(sl, 1), D.p + o);
      cp8(ring.at(sl, 2), F.p + o);
      if (!euler) cp8(ring.at(sl, 3), P.p + o);
    }
    cp_commit();
  };
#pragma unroll
  for (int r = 0; r < CN_RING; r++) fetch(r, r);
  double yh[NL];       // y(i - 1 - t)
  double pend[PD + 1]; // right-hand side of rows i .. i + PD, interchanges of rows < i applied
#pragma unroll
  for (int t = 0; t < NL; t++) yh[t] = 0.0;
#pragma unroll
  for (int t = 0; t <= PD; t++) pend[t] = 0.0;
  int sl = 0;
  for (int k = 0; k < n + PD; k++) {
    double b = 0.0;
    if (k < n) {
      cp_wait<CN_RING - 1>();   // row k has landed
      const double xv = *ring.at(sl, 0), dv = *ring.at(sl, 1), fv = *ring.at(sl, 2);
      const double pw = euler ? 0.0 : *ring.at(sl, 3);
      // the temperature's force is minus the heat advection (pH = -H)
      const double f = (FLD == 2) ? -fv : fv;
      const double rhs = euler ? xv + dt * (ce * dv + f) : xv + dt * (ce * dv + adam_0 * f + adam_1 * pw);
      P.stcs(k, st, f);
      const bool wall = (k == 0 || k == n - 1);
      if (FLD == 0 || FLD == 1 || FLD == 4) b = (q.jj != 0 && !wall) ? rhs : 0.0;
      else if (FLD == 2) b = (k == 0) ? fbi : (k == n - 1) ? fbo : rhs;
      else b = (q.jj != 0) ? rhs : 0.0;
    }
    pend[PD] = b;
    const int i = k - PD;
    if (i >= 0 && i < n) {
      if constexpr (PD >= 1) {
        const int d = fac.piv(i);
        if (d == 1) { const double t = pend[0]; pend[0] = pend[1]; pend[1] = t; }
        if constexpr (PD >= 2)
          if (d == 2) { const double t = pend[0]; pend[0] = pend[2]; pend[2] = t; }
      }
      double y = pend[0];
#pragma unroll
      for (int t = NL - 1; t >= 0; t--) y = y - fac.at(i, NE, t) * yh[t];
      S.stkeep(i, st, y, keep);
#pragma unroll
      for (int t = NL - 1; t > 0; t--) yh[t] = yh[t - 1];
      yh[0] = y;
    }
#pragma unroll
    for (int t = 0; t < PD; t++) pend[t] = pend[t + 1];
    if (k < n) {
      // refill the slot just read (its values are used above)
      fetch(sl, k + CN_RING);
      sl = (sl + 1 == CN_RING) ? 0 : sl + 1;
    }
  }
  cp_wait<0>();   // the ring is free for the backward sweep
}

// backward sweep: U x = y, rows n-1 .. 0, handing each x to the emitter:
// em.point(k, x) for the row itself, then em.top() once rows n-1 .. n-3
// are known, em.interior(r) for rows r = n-2 .. 1 as soon as row r - 1 is
// known, and em.bottom() at the end.  y of row k - CN_RING is copied into
// the ring while row k is computed.
template <int FORM, class Em>
__device__ __forceinline__ void cn_backward(const CnCtx &q, FacCol fac, Ring ring, Col S, Em &em) {
  constexpr int NL = cn_nl(FORM), NE = cn_entries(FORM);
  const int n = q.n;
  const unsigned st = q.st;
  auto fetch = [&](int sl, int k) {
    if (k >= 0) cp8(ring.at(sl, 0), S.p + (unsigned)k * st);
    cp_commit();
  };
#pragma unroll
  for (int r = 0; r < CN_RING; r++) fetch(r, n - 1 - r);
  double xh[NL];   // x(k + 1 + t)
#pragma unroll
  for (int t = 0; t < NL; t++) xh[t] = 0.0;
  int sl = 0;
  for (int k = n - 1; k >= 0; k--) {
    cp_wait<CN_RING - 1>();
    double v = *ring.at(sl, 0);
#pragma unroll
    for (int t = 0; t < NL; t++) v = v - fac.at(k, NE, NL + t) * xh[t];
    const double x = v * fac.at(k, NE, 2 * NL);
#pragma unroll
    for (int t = NL - 1; t > 0; t--) xh[t] = xh[t - 1];
    xh[0] = x;
    em.point(k, x);
    // refill the slot just read (its value is stored above, through x)
    fetch(sl, k - CN_RING);
    sl = (sl + 1 == CN_RING) ? 0 : sl + 1;
    if (k == n - 3) {
      em.top();
      em.interior(n - 2);
    } else if (k < n - 3) {
      em.interior(k + 1);
    }
  }
  em.bottom();
  cp_wait<0>();
}

// ---------------------------------------------------------------------------
// emitters: the derived fields of one column (the expressions of
// k_derived_a / k_derived_b at the same rows; walls k = 0 and k = n - 1)

// field 0: poloidal velocity uS (zero at the walls), d uS / dr, toroidal
// vorticity wT and its diffusion
struct EmVelPol {
  const CnCtx &q;
  Col uS, udS, wT, dwT;
  Win3 s, w;   // uS and wT windows
  __device__ void wpush(int r, double v) {
    const BCW &b = q.a.bc;
    const int n = q.n;
    const double cv = q.a.coef_d_velo;
    wT.stcs(r, q.st, v);
    w.push(v);
    if (r == n - 3)
      dwT.stcs(n - 1, q.st, cv * ((b.fix_fld_cmb[2][3] * w.v0 + b.fix_fld_cmb[1][3] * w.v1
                                   + b.fix_fld_cmb[0][3] * w.v2) - q.g3 * b.r_cmb[2] * w.v2));
    if (r <= n - 3) {
      const int k = r + 1;
      dwT.stcs(k, q.st, cv * (q.co.D2(k, w.v0, w.v1, w.v2) - q.g3 * q.co.ar2(k) * w.v1));
    }
  }
  __device__ void point(int k, double x) {
    const double v = (k == 0 || k == q.n - 1) ? 0.0 : x;
    uS.stcs(k, q.st, v);
    s.push(v);
  }
  __device__ void top() {
    udS.stcs(q.n - 1, q.st, 0.0);
    const double d2s = q.a.bc.fix_dr_cmb[0][3] * s.v1;
    wpush(q.n - 1, -d2s);
  }
  __device__ void interior(int k) {
    udS.stcs(k, q.st, q.co.D1(k, s.v0, s.v1, s.v2));
    wpush(k, -q.co.D2(k, s.v0, s.v1, s.v2) + q.g3 * q.co.ar2(k) * s.v1);
  }
  __device__ void bottom() {
    const BCW &b = q.a.bc;
    udS.stcs(0, q.st, 0.0);
    const double d2s = b.fix_dr_icb[1][3] * s.v0 + b.fix_dr_icb[2][3] * s.v1;
    wpush(0, -(d2s - q.g3 * b.r_icb[2] * s.v0));
    dwT.stcs(0, q.st, q.a.coef_d_velo * ((b.fix_fld_icb[0][3] * w.v0 + b.fix_fld_icb[1][3] * w.v1
                                          + b.fix_fld_icb[2][3] * w.v2) - q.g3 * b.r_icb[2] * w.v0));
  }
};

// field 1: toroidal velocity uT (zero at the walls) = poloidal vorticity wS,
// d wS / dr and the diffusion of wS
struct EmVelTor {
  const CnCtx &q;
  Col uT, wS, wdS, dwS;
  Win3 t;
  __device__ void point(int k, double x) {
    const double v = (k == 0 || k == q.n - 1) ? 0.0 : x;
    uT.stcs(k, q.st, v);
    wS.stcs(k, q.st, v);
    t.push(v);
  }
  __device__ void top() {
    const BCW &b = q.a.bc;
    const int k = q.n - 1;
    wdS.stcs(k, q.st, b.fix_fld_cmb[2][2] * t.v0 + b.fix_fld_cmb[1][2] * t.v1 + b.fix_fld_cmb[0][2] * t.v2);
    const double d2s = b.fix_fld_cmb[2][3] * t.v0 + b.fix_fld_cmb[1][3] * t.v1 + b.fix_fld_cmb[0][3] * t.v2;
    dwS.stcs(k, q.st, q.a.coef_d_velo * (d2s - q.g3 * b.r_cmb[2] * t.v2));
  }
  __device__ void interior(int k) {
    wdS.stcs(k, q.st, q.co.D1(k, t.v0, t.v1, t.v2));
    dwS.stcs(k, q.st, q.a.coef_d_velo * (q.co.D2(k, t.v0, t.v1, t.v2) - q.g3 * q.co.ar2(k) * t.v1));
  }
  __device__ void bottom() {
    const BCW &b = q.a.bc;
    wdS.stcs(0, q.st, b.fix_fld_icb[0][2] * t.v0 + b.fix_fld_icb[1][2] * t.v1 + b.fix_fld_icb[2][2] * t.v2);
    const double d2s = b.fix_fld_icb[0][3] * t.v0 + b.fix_fld_icb[1][3] * t.v1 + b.fix_fld_icb[2][3] * t.v2;
    dwS.stcs(0, q.st, q.a.coef_d_velo * (d2s - q.g3 * b.r_icb[2] * t.v0));
  }
};

// field 2: temperature (the fixed values at the walls), buoyancy (from the
// solved values) and the diffusion of T
struct EmTemp {
  const CnCtx &q;
  Col T, buo, dT;
  double fbi, fbo;
  Win3 t;
  __device__ void point(int k, double x) {
    buo.stcs(k, q.st, q.a.coef_buo * x * q.co.r(k));
    const double v = (k == 0) ? fbi : (k == q.n - 1) ? fbo : x;
    T.stcs(k, q.st, v);
    t.push(v);
  }
  __device__ void top() {
    const BCW &b = q.a.bc;
    const double d1t = b.fix_fld_cmb[2][2] * t.v0 + b.fix_fld_cmb[1][2] * t.v1 + b.fix_fld_cmb[0][2] * fbo;
    const double d2t = b.fix_fld_cmb[2][3] * t.v0 + b.fix_fld_cmb[1][3] * t.v1 + b.fix_fld_cmb[0][3] * fbo;
    dT.stcs(q.n - 1, q.st,
            q.a.coef_d_temp * (d2t + 2.0 * b.r_cmb[1] * d1t - q.g3 * b.r_cmb[2] * fbo));
  }
  __device__ void interior(int k) {
    dT.stcs(k, q.st, q.a.coef_d_temp * (q.co.D2(k, t.v0, t.v1, t.v2)
                                        + 2.0 * q.co.ar1(k) * q.co.D1(k, t.v0, t.v1, t.v2)
                                        - q.g3 * q.co.ar2(k) * t.v1));
  }
  __device__ void bottom() {
    const BCW &b = q.a.bc;
    const double d1t = b.fix_fld_icb[0][2] * fbi + b.fix_fld_icb[1][2] * t.v1 + b.fix_fld_icb[2][2] * t.v2;
    const double d2t = b.fix_fld_icb[0][3] * fbi + b.fix_fld_icb[1][3] * t.v1 + b.fix_fld_icb[2][3] * t.v2;
    dT.stcs(0, q.st, q.a.coef_d_temp * (d2t + 2.0 * b.r_icb[1] * d1t - q.g3 * b.r_icb[2] * fbi));
  }
};

// field 3: poloidal magnetic field bS, d bS / dr, toroidal current cT and
// the magnetic diffusion of bS
struct EmMagPol {
  const CnCtx &q;
  Col bS, bdS, cT, dbS;
  Win3 s;
  __device__ void point(int k, double x) {
    bS.stcs(k, q.st, x);
    s.push(x);
  }
  __device__ void top() {
    const BCW &b = q.a.bc;
    const int k = q.n - 1;
    const double B0 = s.v2, Bm = s.v1, cb = q.a.coef_d_magne;
    bdS.stcs(k, q.st, -q.gl * b.r_cmb[1] * B0);
    const double d2b = b.fix_dr_cmb[0][3] * Bm + (b.fix_dr_cmb[1][3] - q.gl * b.r_cmb[1] * b.fix_dr_cmb[2][3]) * B0;
    cT.stcs(k, q.st, -(d2b - q.g3 * b.r_cmb[2] * B0));
    dbS.stcs(k, q.st, cb * (d2b - q.g3 * b.r_cmb[2] * B0));
  }
  __device__ void interior(int k) {
    bdS.stcs(k, q.st, q.co.D1(k, s.v0, s.v1, s.v2));
    const double c = -q.co.D2(k, s.v0, s.v1, s.v2) + q.g3 * q.co.ar2(k) * s.v1;
    cT.stcs(k, q.st, c);
    dbS.stcs(k, q.st, -q.a.coef_d_magne * c);
  }
  __device__ void bottom() {
    const BCW &b = q.a.bc;
    const double B0 = s.v0, B1 = s.v1, cb = q.a.coef_d_magne;
    bdS.stcs(0, q.st, (q.gl + 1.0) * b.r_icb[1] * B0);
    const double d2b = ((q.gl + 1.0) * b.r_icb[1] * b.fix_dr_icb[0][3] + b.fix_dr_icb[1][3]) * B0
                     + b.fix_dr_icb[2][3] * B1;
    cT.stcs(0, q.st, -(d2b - q.g3 * b.r_icb[2] * B0));
    dbS.stcs(0, q.st, cb * (d2b - q.g3 * b.r_icb[2] * B0));
  }
};

// field 4: toroidal magnetic field bT (zero at the walls) = poloidal current
// cS, d cS / dr and the magnetic diffusion of bT
struct EmMagTor {
  const CnCtx &q;
  Col bT, cS, cdS, dbT;
  Win3 t;
  __device__ void point(int k, double x) {
    const double v = (k == 0 || k == q.n - 1) ? 0.0 : x;
    bT.stcs(k, q.st, v);
    cS.stcs(k, q.st, v);
    t.push(v);
  }
  __device__ void top() {
    const BCW &b = q.a.bc;
    const int k = q.n - 1;
    cdS.stcs(k, q.st, b.fix_fld_cmb[2][2] * t.v0 + b.fix_fld_cmb[1][2] * t.v1);
    const double d2 = b.fix_fld_cmb[2][3] * t.v0 + b.fix_fld_cmb[1][3] * t.v1 + b.fix_fld_cmb[0][3] * t.v2;
    dbT.stcs(k, q.st, q.a.coef_d_magne * (d2 - q.g3 * b.r_cmb[2] * t.v2));
  }
  __device__ void interior(int k) {
    cdS.stcs(k, q.st, q.co.D1(k, t.v0, t.v1, t.v2));
    dbT.stcs(k, q.st, q.a.coef_d_magne * (q.co.D2(k, t.v0, t.v1, t.v2) - q.g3 * q.co.ar2(k) * t.v1));
  }
  __device__ void bottom() {
    const BCW &b = q.a.bc;
    cdS.stcs(0, q.st, b.fix_fld_icb[1][2] * t.v1 + b.fix_fld_icb[2][2] * t.v2);
    const double d2 = b.fix_fld_icb[0][3] * t.v0 + b.fix_fld_icb[1][3] * t.v1 + b.fix_fld_icb[2][3] * t.v2;
    dbT.stcs(0, q.st, q.a.coef_d_magne * (d2 - q.g3 * b.r_icb[2] * t.v0));
  }
};

// ---------------------------------------------------------------------------
// one (field, column) thread: the sweeps with the field's slots and emitter
template <int FLD, int FORM>
__device__ __forceinline__ void cn_column(const CnCtx &q, double *col, size_t fs, FacCol fac, Ring ring,
                                          int euler) {
  auto C = [&](int slot) { return Col{col + (size_t)slot * fs}; };
  if constexpr (FLD == 0) {
    cn_forward<0, FORM>(q, fac, ring, C(VORT + 2), C(WDIFF + 2), C(FORCES + 2), C(PREMOM + 2), C(VELO), euler);
    EmVelPol em{q, C(VELO), C(VELO + 1), C(VORT + 2), C(WDIFF + 2)};
    cn_backward<FORM>(q, fac, ring, C(VELO), em);
  } else if constexpr (FLD == 1) {
    cn_forward<1, FORM>(q, fac, ring, C(VORT), C(WDIFF), C(FORCES), C(PREMOM), C(VELO + 2), euler);
    EmVelTor em{q, C(VELO + 2), C(VORT), C(VORT + 1), C(WDIFF)};
    cn_backward<FORM>(q, fac, ring, C(VELO + 2), em);
  } else if constexpr (FLD == 2) {
    cn_forward<2, FORM>(q, fac, ring, C(TEMP), C(TDIFF), C(HADV), C(PREHEAT), C(TEMP), euler);
    EmTemp em{q, C(TEMP), C(ROTBUO + 2), C(TDIFF), (q.jj == 0) ? q.a.temp_icb_fld : 0.0,
              (q.jj == 0) ? q.a.temp_cmb_fld : 0.0};
    cn_backward<FORM>(q, fac, ring, C(TEMP), em);
  } else if constexpr (FLD == 3) {
    cn_forward<3, FORM>(q, fac, ring, C(MAGNE), C(BDIFF), C(INDUCT), C(PREUXB), C(MAGNE), euler);
    EmMagPol em{q, C(MAGNE), C(MAGNE + 1), C(CURRENT + 2), C(BDIFF)};
    cn_backward<FORM>(q, fac, ring, C(MAGNE), em);
  } else {
    cn_forward<4, FORM>(q, fac, ring, C(MAGNE + 2), C(BDIFF + 2), C(INDUCT + 2), C(PREUXB + 2), C(MAGNE + 2),
                        euler);
    EmMagTor em{q, C(MAGNE + 2), C(CURRENT), C(CURRENT + 1), C(BDIFF + 2)};
    cn_backward<FORM>(q, fac, ring, C(MAGNE + 2), em);
  }
}

// one field's entries of the pack (a switch: indexing the parameter arrays
// with a run-time index would copy them to local memory)
struct CnField {
  const double *fac;
  const unsigned char *piv;
  int form;
};
__device__ __forceinline__ CnField cn_field(const CnPack &pk, int fld) {
  switch (fld) {
    case 0: return {pk.fac[0], pk.piv[0], pk.form[0]};
    case 1: return {pk.fac[1], pk.piv[1], pk.form[1]};
    case 2: return {pk.fac[2], pk.piv[2], pk.form[2]};
    case 3: return {pk.fac[3], pk.piv[3], pk.form[3]};
    default: return {pk.fac[4], pk.piv[4], pk.form[4]};
  }
}

// One block: 8 warps of one field (the tile's x); warp w takes the (m, sign)
// pair p0 + w (pair 0: m = 0; pair 2m - 1: (m, +); pair 2m: (m, -)), lane
// the degree l0 + lane, so every access of a warp to a slot row is 32
// consecutive doubles.  The block stages the radial coefficients in shared
// memory; each thread then runs its column.
__global__ void __launch_bounds__(CN_THREADS, 4)
k_cn_step(RJArgs a, double *f, size_t fs, CnPack pk, const int *moff, const int4 *tiles, int euler) {
  extern __shared__ double cn_sm[];
  const int n = a.nr, nl = a.L + 1, tid = threadIdx.x;
  const int4 tl = tiles[blockIdx.x];   // (field, p0, l0, -)
  const int fld = tl.x;
  const CnField fd = cn_field(pk, fld);
  const int form = fd.form;
  double *sco = cn_sm;                 // [9][n]
  for (int e = tid; e < 3 * n; e += CN_THREADS) {
    sco[e] = __ldg(a.d1 + e);
    sco[3 * n + e] = __ldg(a.d2 + e);
  }
  for (int e = tid; e < n; e += CN_THREADS) {
    sco[6 * n + e] = __ldg(a.ar1 + e);
    sco[7 * n + e] = __ldg(a.ar2 + e);
    sco[8 * n + e] = __ldg(a.r + e);
  }
  __syncthreads();
  const int p = tl.y + tid / 32, l = tl.z + tid % 32;
  const int m = (p + 1) >> 1, sgn = (p > 0 && (p & 1) == 0) ? 1 : 0;
  if (l >= nl || m > l) return;
  const int jj = moff[m] + sgn * (nl - m) + (l - m);
  const CnCtx q{a, RadCo{sco, n}, n, (unsigned)a.jmax, jj, __ldg(a.g3 + jj), __ldg(a.gl + jj)};
  double *col = f + jj;
  const FacCol fac{fd.fac + l, fd.piv ? fd.piv + l : nullptr, nl};
  const Ring ring{reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(cn_sm) + cn_ring_offset(n)) + tid};
  switch (fld * 4 + form) {
    case 0 * 4 + CN_N5: cn_column<0, CN_N5>(q, col, fs, fac, ring, euler); break;
    case 0 * 4 + CN_W5: cn_column<0, CN_W5>(q, col, fs, fac, ring, euler); break;
    case 1 * 4 + CN_N3: cn_column<1, CN_N3>(q, col, fs, fac, ring, euler); break;
    case 1 * 4 + CN_W3: cn_column<1, CN_W3>(q, col, fs, fac, ring, euler); break;
    case 2 * 4 + CN_N3: cn_column<2, CN_N3>(q, col, fs, fac, ring, euler); break;
    case 2 * 4 + CN_W3: cn_column<2, CN_W3>(q, col, fs, fac, ring, euler); break;
    case 3 * 4 + CN_N3: cn_column<3, CN_N3>(q, col, fs, fac, ring, euler); break;
    case 3 * 4 + CN_W3: cn_column<3, CN_W3>(q, col, fs, fac, ring, euler); break;
    case 4 * 4 + CN_N3: cn_column<4, CN_N3>(q, col, fs, fac, ring, euler); break;
    case 4 * 4 + CN_W3: cn_column<4, CN_W3>(q, col, fs, fac, ring, euler); break;
    default: break;
  }
}

// ---------------------------------------------------------------------------
int cn_setup(Ctx &c) {
  c.cn_ready = false;
  c.cn_off_reason = "";
  const int n = c.nr, nl = c.L + 1;
  if (n < 6 || c.kin != 0 || c.kout != n - 1 || (size_t)n * c.jmax >= ((size_t)1 << 31)) {
    c.tune[TUNE_CN] = -1;
    c.cn_off_reason = n < 6 ? "fewer than 6 radial points" : "the fluid shell is not the whole radial grid, or "
                                                             "the shell has 2^31 values or more per field";
    return 0;
  }
  int *d_ok = nullptr;
  CB2_CUDA(cudaMalloc(&d_ok, (size_t)5 * nl * sizeof(int)));
  const LuSet set{{c.d_lu_vp, c.d_lu_vt, c.d_lu_t, c.d_lu_bs, c.d_lu_bt},
                  {c.d_pv_vp, c.d_pv_vt, c.d_pv_t, c.d_pv_bs, c.d_pv_bt}};
  k_cn_check<<<cdiv(5 * nl, 128), 128, 0, c.stream>>>(n, nl, set, d_ok);
  std::vector<int> ok((size_t)5 * nl);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(ok.data(), d_ok, ok.size() * sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFree(d_ok);
  if (e != cudaSuccess) return cuda_fail(e, "cn_setup: factor check");
  // per field: the narrow form if every degree allows it, else the form
  // with interchanges if every degree fits it, else no fused step
  CnPack pk{};
  size_t dbl = 0, byt = 0, smem = 0;
  for (int q = 0; q < 5; q++) {
    int all = 3;
    for (int l = 0; l < nl; l++) all &= ok[(size_t)q * nl + l];
    if (!all) {
      c.tune[TUNE_CN] = -1;   // an interchange beyond the form's reach
      c.cn_off_reason = "a radial LU factor has a row interchange more than two rows away";
      return 0;
    }
    pk.form[q] = (all & 1) ? (q == 0 ? CN_N5 : CN_N3) : (q == 0 ? CN_W5 : CN_W3);
    dbl += (size_t)n * cn_entries(pk.form[q]) * nl;
    if (cn_pd(pk.form[q])) byt += (size_t)n * nl;
  }
  smem = cn_smem(n);
  if (smem > 227 * 1024) {
    c.tune[TUNE_CN] = -1;
    c.cn_off_reason = "the per-thread input rings need more than 227 KB of shared memory";
    return 0;
  }
  CB2_CUDA(cudaMalloc(&c.d_cn_lu, dbl * sizeof(double) + byt));
  size_t od = 0, ob = dbl * sizeof(double);
  for (int q = 0; q < 5; q++) {
    pk.fac[q] = c.d_cn_lu + od;
    od += (size_t)n * cn_entries(pk.form[q]) * nl;
    if (cn_pd(pk.form[q])) {
      pk.piv[q] = reinterpret_cast<const unsigned char *>(c.d_cn_lu) + ob;
      ob += (size_t)n * nl;
    }
  }
  k_cn_pack<<<cdiv(5 * nl, 128), 128, 0, c.stream>>>(n, nl, set, pk);
  CB2_CUDA(cudaGetLastError());
  // blocks: (field, p0, l0) tiles of 8 (m, sign) pairs x 32 degrees
  std::vector<int4> tl;
  for (int q = 0; q < 5; q++) {
    for (int l0 = 0; l0 <= c.L; l0 += 32) {
      const int npair = 2 * std::min(l0 + 31, c.L) + 1;
      for (int p0 = 0; p0 < npair; p0 += 8) tl.push_back(int4{q, p0, l0, 0});
    }
  }
  c.cn_tiles = (int)tl.size();
  CB2_CUDA(cudaMalloc(&c.d_cn_tiles, tl.size() * sizeof(int4)));
  CB2_CUDA(cudaMemcpyAsync(c.d_cn_tiles, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice, c.stream));
  CB2_CUDA(raise_smem_limit(k_cn_step, smem));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  c.cn_pack = new CnPack(pk);
  c.cn_smem = smem;
  c.cn_ready = true;
  return 0;
}

void cn_free(Ctx &c) {
  delete static_cast<CnPack *>(c.cn_pack);
  c.cn_pack = nullptr;
}

void cn_stage(Ctx &c, bool euler) {
  if (c.cn_ready && c.tune[TUNE_CN] == 1) {
    cn_step(c, euler);
  } else {
    rj_explicit(c, euler);
    rj_implicit(c);
  }
}

// one launch for the five fields (the 5-band field's blocks first)
void cn_step(Ctx &c, bool euler) {
  k_cn_step<<<c.cn_tiles, CN_THREADS, c.cn_smem, c.stream>>>(c.rj_args(), c.d_f, c.fsize(),
                                                              *static_cast<const CnPack *>(c.cn_pack), c.d_moff,
                                                              c.d_cn_tiles, euler ? 1 : 0);
}

}  // namespace cb2
