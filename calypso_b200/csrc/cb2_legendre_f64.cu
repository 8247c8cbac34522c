// cb2_legendre_f64.cu -- float64 Legendre transforms (the plain path).
//
// Definition: PARALLEL_src/SPH_SHELL_src/legendre_bwd_trans_org.f90:45-209 and
// legendre_fwd_trans_org.f90:45-169 of the reference, evaluated with the
// equatorial symmetry that its SYMMETRIC_MATMUL variant uses
// (cal_vr_rtm_by_matmul.f90, cal_sp_rlm_by_matmul.f90):
//   P_l^m(pi - theta) = (-1)^(l-m) P_l^m(theta),
//   dP_l^m/dtheta (pi - theta) = -(-1)^(l-m) dP_l^m/dtheta (theta).
// Each term is accumulated by its reflection parity sigma, so the south node
// i gets acc[0] + acc[1] and the mirror node nth-1-i gets acc[0] - acc[1].
//
// Backward: one block per (order m, radial tile, colatitude tile); one warp
// per field group (a vector: S, dS/dr, T of orders +m and -m; or a scalar),
// one lane per Gauss node of the south half.  The spectral coefficients of a
// chunk of degrees are staged in shared memory, pre-scaled by l(l+1)/r^2,
// 1/r and 1/r as legendre_b_trans_vector_org does.
// Forward: one block per (order m, radial tile); one lane per degree l, the
// Gauss-weighted symmetric / antisymmetric grid values staged in shared
// memory.
#include <algorithm>
#include <type_traits>

#include "cb2_internal.cuh"

namespace cb2 {

constexpr int BWD_LC = 16;  // degrees per staged chunk
constexpr int FWD_TC = 8;   // Gauss node pairs per staged chunk
// radial levels per block (BWD_KT backward, FWD_KT forward) are template
// parameters; the autotuner picks them per shell shape (cb2_autotune)
constexpr int MAXG = 6;     // field groups (vectors + scalars) per launch

// 8-byte asynchronous copy global -> shared; n = 0 fills the 8 bytes with
// zeros and reads nothing
__device__ inline void cp_async8(double *dst, const double *src, int n) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(n)
               : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// every group but the newest has landed
__device__ inline void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

struct LegArgs {
  int L, nr, nth, nh, jmax, NS, nvec, nscal, ncomp, cbase;
  int slot[MAXG];           // first rj slot of each group of this launch
  const int *moff;
  const size_t *poff;
  const double *Plt, *dPlt, *Ptl, *dPtl, *asin_t, *wgt;
  const double *g3rlm, *g6, *g7, *r, *ar1;
  double *f;                // rj fields
  size_t fs;                // slot stride
};

__device__ inline int jj_of(const LegArgs &a, int l, int m, int s) {
  return a.moff[m] + s * (a.L + 1 - m) + (l - m);
}

// F[theta][k][c][slot], slot 2m = order +m, 2m+1 = order -m
__device__ inline size_t four_at(const LegArgs &a, int th, int k, int c) {
  return (((size_t)th * a.nr + k) * a.ncomp + c) * a.NS;
}

// Each lane handles two Gauss nodes of the south half, i and i + 32, so the
// spectral coefficients it reads from shared memory (three 16-byte loads
// per radial level and degree) feed twice the FMAs.
template <int BWD_KT>
__global__ void __launch_bounds__(32 * MAXG)
k_leg_bwd_f64(LegArgs a, double *four) {
  const int m = blockIdx.z, k0 = blockIdx.y * BWD_KT, i0 = blockIdx.x * 64;
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int ngrp = a.nvec + a.nscal;
  const int nl = a.L + 1 - m;
  const int ia = i0 + lane, ib = i0 + 32 + lane;
  const bool act = g < ngrp && ia < a.nh;
  const bool isvec = g < a.nvec;
  // two shared-memory buffers, each [group][degree][radial level][S+ S- D+
  // D- T+ T-] and P_l^m, dP_l^m of the chunk's degrees at the block's 64
  // nodes: the copies of the next chunk (cp.async) are in flight while the
  // FMAs of this one run
  constexpr int SCN = MAXG * BWD_LC * BWD_KT * 6, PN = BWD_LC * 64, BUF = SCN + 2 * PN;
  extern __shared__ __align__(16) double smb[];
  double acc[2][BWD_KT][6][2];
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int q = 0; q < BWD_KT; q++)
#pragma unroll
      for (int c = 0; c < 6; c++) acc[h][q][c][0] = acc[h][q][c][1] = 0.0;
  // node b may lie beyond the half grid: it reads node a's tables and is
  // not stored
  const int ibr = (ib < a.nh) ? ib : ia;
  const double ama = (ia < a.nh) ? (double)m * a.asin_t[ia] : 0.0;
  const double amb = (ia < a.nh) ? (double)m * a.asin_t[ibr] : 0.0;
  const size_t po = a.poff[m];
  const int tot = ngrp * BWD_LC * 6 * BWD_KT;
  // element e of a chunk: degree lc (fastest, coalesced), component v, level q, group gg
  auto decomp = [&](int e, int &lc, int &v, int &q, int &gg) {
    lc = e % BWD_LC;
    int t = e / BWD_LC;
    v = t % 6; t /= 6;
    q = t % BWD_KT; gg = t / BWD_KT;
  };
  auto issue = [&](int lc0, int b) {
    double *sc = smb + (size_t)b * BUF, *ps = sc + SCN, *dps = ps + PN;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      int lc, v, q, gg;
      decomp(e, lc, v, q, gg);
      const int l = m + lc0 + lc, k = k0 + q, s = v & 1, comp = v >> 1;  // v: 0 S+ 1 S- 2 D+ 3 D- 4 T+ 5 T-
      const double *src = nullptr;
      if (l <= a.L && k < a.nr && !(m == 0 && s == 1) && (gg < a.nvec || comp == 0))
        src = a.f + (size_t)(a.slot[gg] + (gg < a.nvec ? comp : 0)) * a.fs + (size_t)k * a.jmax + jj_of(a, l, m, s);
      cp_async8(sc + ((gg * BWD_LC + lc) * BWD_KT + q) * 6 + v, src ? src : a.f, src ? 8 : 0);
    }
    for (int e = threadIdx.x; e < PN; e += blockDim.x) {
      const int lc = e >> 6, ii = i0 + (e & 63), t = lc0 + lc;
      const bool in = t < nl && ii < a.nh;
      const size_t at = in ? po + (size_t)t * a.nh + ii : 0;
      cp_async8(ps + e, a.Plt + at, in ? 8 : 0);
      cp_async8(dps + e, a.dPlt + at, in ? 8 : 0);
    }
    cp_async_commit();
  };
  // the radial and degree factors of the vector spectra, applied by the
  // thread that copied each value once its copies have landed
  auto convert = [&](int lc0, int b) {
    double *sc = smb + (size_t)b * BUF;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      int lc, v, q, gg;
      decomp(e, lc, v, q, gg);
      const int l = m + lc0 + lc, k = k0 + q;
      if (gg < a.nvec && l <= a.L && k < a.nr) {
        const double ar = a.ar1[k], l3 = (l == 0) ? 0.5 : (double)l * (double)(l + 1);
        double &x = sc[((gg * BWD_LC + lc) * BWD_KT + q) * 6 + v];
        x *= ((v >> 1) == 0) ? ar * ar * l3 : ar;
      }
    }
  };
  const int nch = (nl + BWD_LC - 1) / BWD_LC;
  issue(0, 0);
  for (int ch = 0; ch < nch; ch++) {
    const int lc0 = ch * BWD_LC, b = ch & 1;
    if (ch + 1 < nch) issue(lc0 + BWD_LC, b ^ 1);
    else cp_async_commit();
    cp_async_wait1();
    convert(lc0, b);
    __syncthreads();
    const double(*sc)[BWD_LC][BWD_KT][6] =
        reinterpret_cast<const double(*)[BWD_LC][BWD_KT][6]>(smb + (size_t)b * BUF);
    const double(*Ps)[64] = reinterpret_cast<const double(*)[64]>(smb + (size_t)b * BUF + SCN);
    const double(*dPs)[64] = reinterpret_cast<const double(*)[64]>(smb + (size_t)b * BUF + SCN + PN);
    if (act) {
      int lcn = min(BWD_LC, nl - lc0);
      // lc0 is even, so degree t = lc0 + lc has parity lc & 1: unrolling by
      // two keeps the parity index a compile-time constant (registers)
      auto body = [&](int lc, auto SPc) {
        constexpr int sp = decltype(SPc)::value, sd = sp ^ 1;
        const double Pa = Ps[lc][lane], dPa = dPs[lc][lane], Pb = Ps[lc][32 + lane], dPb = dPs[lc][32 + lane];
        const double mPa = Pa * ama, mPb = Pb * amb;
#pragma unroll
        for (int q = 0; q < BWD_KT; q++) {
          const double2 *row = reinterpret_cast<const double2 *>(&sc[g][lc][q][0]);
          const double2 S = row[0];
          if (isvec) {
            const double2 D = row[1], T = row[2];
            // S = (S+, S-), D = (D+, D-), T = (T+, T-)
            acc[0][q][0][sp] += S.x * Pa;          acc[1][q][0][sp] += S.x * Pb;   // v_r(+m)
            acc[0][q][1][sp] += S.y * Pa;          acc[1][q][1][sp] += S.y * Pb;   // v_r(-m)
            acc[0][q][2][sd] += D.x * dPa;         acc[1][q][2][sd] += D.x * dPb;  // v_theta(+m)
            acc[0][q][2][sp] += T.y * mPa;         acc[1][q][2][sp] += T.y * mPb;
            acc[0][q][3][sd] += D.y * dPa;         acc[1][q][3][sd] += D.y * dPb;  // v_theta(-m)
            acc[0][q][3][sp] -= T.x * mPa;         acc[1][q][3][sp] -= T.x * mPb;
            acc[0][q][4][sd] -= T.x * dPa;         acc[1][q][4][sd] -= T.x * dPb;  // v_phi(+m)
            acc[0][q][4][sp] += D.y * mPa;         acc[1][q][4][sp] += D.y * mPb;
            acc[0][q][5][sd] -= T.y * dPa;         acc[1][q][5][sd] -= T.y * dPb;  // v_phi(-m)
            acc[0][q][5][sp] -= D.x * mPa;         acc[1][q][5][sp] -= D.x * mPb;
          } else {
            acc[0][q][0][sp] += S.x * Pa;          acc[1][q][0][sp] += S.x * Pb;
            acc[0][q][1][sp] += S.y * Pa;          acc[1][q][1][sp] += S.y * Pb;
          }
        }
      };
      int lc = 0;
      for (; lc + 1 < lcn; lc += 2) {
        body(lc, std::integral_constant<int, 0>());
        body(lc + 1, std::integral_constant<int, 1>());
      }
      if (lc < lcn) body(lc, std::integral_constant<int, 0>());
    }
    __syncthreads();   // buffer b is refilled by the next iteration's copies
  }
  if (!act) return;
  const int ncw = isvec ? 3 : 1;
  const int c0 = a.cbase + (isvec ? 3 * g : 3 * a.nvec + (g - a.nvec));
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int i = h ? ib : ia;
    if (i >= a.nh) break;
    const int ii = a.nth - 1 - i;
#pragma unroll
    for (int q = 0; q < BWD_KT; q++) {
      int k = k0 + q;
      if (k >= a.nr) break;
      for (int c = 0; c < ncw; c++) {
        double e0 = acc[h][q][2 * c][0], o0 = acc[h][q][2 * c][1];
        double e1 = acc[h][q][2 * c + 1][0], o1 = acc[h][q][2 * c + 1][1];
        double2 south = make_double2(e0 + o0, m == 0 ? 0.0 : e1 + o1);
        double2 north = make_double2(e0 - o0, m == 0 ? 0.0 : e1 - o1);
        *reinterpret_cast<double2 *>(four + four_at(a, i, k, c0 + c) + 2 * m) = south;
        if (ii != i)
          *reinterpret_cast<double2 *>(four + four_at(a, ii, k, c0 + c) + 2 * m) = north;
      }
    }
  }
}

// forward: block = (order m, radial tile); thread = two consecutive
// degrees l - m = t (even) and t + 1, one of each reflection parity, so the
// symmetric and antisymmetric sums of a grid value, adjacent in shared
// memory, are read as one 16-byte pair and both used.  NV vectors and NSC
// scalars starting at component c0 of the Fourier buffer (which holds
// a.ncomp components) and at group g0 of a.slot.
template <int NV, int NSC, int FWD_KT>
__global__ void __launch_bounds__(256)
k_leg_fwd_f64(LegArgs a, const double *four, int c0, int g0) {
  const int m = blockIdx.z, k0 = blockIdx.y * FWD_KT;
  const int nl = a.L + 1 - m;
  constexpr int C = 3 * NV + NSC;
  // two buffers, each [pair][k][c][s][sym/anti] and P_l^m, dP_l^m
  // [pair][degree] of one chunk of node pairs: the copies (cp.async) of the
  // next chunk are in flight while the FMAs of this one run
  extern __shared__ __align__(16) double hs0[];
  const size_t HN = (size_t)FWD_TC * FWD_KT * C * 4, BUF = HN + 2 * (size_t)FWD_TC * nl;
  double *hs = hs0;
  auto H2 = [&](int ip, int q, int c, int s) -> double2 {   // (sym, anti) of (c, s)
    return *reinterpret_cast<const double2 *>(&hs[((((size_t)ip * FWD_KT + q) * C + c) * 2 + s) * 2]);
  };
  const size_t po = a.poff[m];
  const double *PT = nullptr, *dPT = nullptr;
  // the raw values of pair (ip, q, c, s): this node and its mirror, into
  // the (sym, anti) slots that convert() fills
  auto issue = [&](int ib, int b) {
    double *h = hs0 + b * BUF, *pt = h + HN, *dpt = pt + (size_t)FWD_TC * nl;
    const int npair = min(FWD_TC, a.nh - ib), tot = npair * FWD_KT * C * 2;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      int s = e & 1, tt = e >> 1;
      int c = tt % C; tt /= C;
      int q = tt % FWD_KT, ip = tt / FWD_KT;
      int k = k0 + q, i = ib + ip, ii = a.nth - 1 - i;
      const bool in = k < a.nr && !(m == 0 && s == 1);
      double *d = h + ((((size_t)ip * FWD_KT + q) * C + c) * 2 + s) * 2;
      cp_async8(d, in ? four + four_at(a, i, k, c0 + c) + 2 * m + s : four, in ? 8 : 0);
      cp_async8(d + 1, in ? four + four_at(a, ii, k, c0 + c) + 2 * m + s : four, in ? 8 : 0);
    }
    for (int e = threadIdx.x; e < npair * nl; e += blockDim.x) {
      const int ip = e / nl, tt = e - ip * nl;
      cp_async8(pt + ip * nl + tt, a.Ptl + po + (size_t)(ib + ip) * nl + tt, 8);
      cp_async8(dpt + ip * nl + tt, a.dPtl + po + (size_t)(ib + ip) * nl + tt, 8);
    }
    cp_async_commit();
  };
  auto convert = [&](int ib, int b) {
    double *h = hs0 + b * BUF;
    const int npair = min(FWD_TC, a.nh - ib), tot = npair * FWD_KT * C * 2;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      int tt = e >> 1;
      tt /= C;
      const int ip = tt / FWD_KT, i = ib + ip, ii = a.nth - 1 - i;
      double *d = h + (size_t)e * 2;
      const double fa = d[0] * a.wgt[i], fb = d[1] * a.wgt[ii];
      d[0] = fa + fb;
      d[1] = fa - fb;
    }
  };
  for (int lt0 = 0; lt0 < nl; lt0 += 2 * blockDim.x) {
    const int t = lt0 + 2 * threadIdx.x;   // even: parity 0; t + 1: parity 1
    const bool act0 = t < nl, act1 = t + 1 < nl;
    double accv[2][NV > 0 ? NV : 1][FWD_KT][6];
    double accs[2][NSC > 0 ? NSC : 1][FWD_KT][2];
#pragma unroll
    for (int d = 0; d < 2; d++)
#pragma unroll
      for (int q = 0; q < FWD_KT; q++) {
#pragma unroll
        for (int v = 0; v < (NV > 0 ? NV : 1); v++)
#pragma unroll
          for (int c = 0; c < 6; c++) accv[d][v][q][c] = 0.0;
#pragma unroll
        for (int v = 0; v < (NSC > 0 ? NSC : 1); v++) accs[d][v][q][0] = accs[d][v][q][1] = 0.0;
      }
    __syncthreads();   // the buffers of the previous degree block are free
    issue(0, 0);
    for (int ib = 0, b = 0; ib < a.nh; ib += FWD_TC, b ^= 1) {
      const int npair = min(FWD_TC, a.nh - ib);
      if (ib + FWD_TC < a.nh) issue(ib + FWD_TC, b ^ 1);
      else cp_async_commit();
      cp_async_wait1();
      convert(ib, b);
      __syncthreads();
      hs = hs0 + b * BUF;
      PT = hs + HN;
      dPT = PT + (size_t)FWD_TC * nl;
      if (act0) {
        const int t1 = act1 ? t + 1 : t;   // a missing odd degree reads the even one's table, not stored
        for (int ip = 0; ip < npair; ip++) {
          const int i = ib + ip;
          const double *Pr = PT + ip * nl, *dPr = dPT + ip * nl;
          const double P0 = Pr[t], dP0 = dPr[t], P1 = Pr[t1], dP1 = dPr[t1];
          const double am = (double)m * a.asin_t[i];
          const double pg0 = P0 * am, pg1 = P1 * am;   // P m / sin(theta), order +m
#pragma unroll
          for (int v = 0; v < NV; v++) {
#pragma unroll
            for (int q = 0; q < FWD_KT; q++) {
              const double2 R0 = H2(ip, q, 3 * v, 0), R1 = H2(ip, q, 3 * v, 1);
              const double2 T0 = H2(ip, q, 3 * v + 1, 0), T1 = H2(ip, q, 3 * v + 1, 1);
              const double2 F0 = H2(ip, q, 3 * v + 2, 0), F1 = H2(ip, q, 3 * v + 2, 1);
              // parity 0 (degree t): r, tn, pn from the symmetric sums,
              // tp, pp from the antisymmetric ones; parity 1 the converse.
              // Order +m: s slot 0, order -m: s slot 1.
              accv[0][v][q][0] += R0.x * P0;
              accv[0][v][q][1] += R1.x * P0;
              accv[0][v][q][2] += T0.y * dP0 - F1.x * pg0;
              accv[0][v][q][3] += T1.y * dP0 + F0.x * pg0;
              accv[0][v][q][4] -= T1.x * pg0 + F0.y * dP0;
              accv[0][v][q][5] -= -T0.x * pg0 + F1.y * dP0;
              accv[1][v][q][0] += R0.y * P1;
              accv[1][v][q][1] += R1.y * P1;
              accv[1][v][q][2] += T0.x * dP1 - F1.y * pg1;
              accv[1][v][q][3] += T1.x * dP1 + F0.y * pg1;
              accv[1][v][q][4] -= T1.y * pg1 + F0.x * dP1;
              accv[1][v][q][5] -= -T0.y * pg1 + F1.x * dP1;
            }
          }
#pragma unroll
          for (int sc = 0; sc < NSC; sc++) {
#pragma unroll
            for (int q = 0; q < FWD_KT; q++) {
              const double2 S0 = H2(ip, q, 3 * NV + sc, 0), S1 = H2(ip, q, 3 * NV + sc, 1);
              accs[0][sc][q][0] += S0.x * P0;
              accs[0][sc][q][1] += S1.x * P0;
              accs[1][sc][q][0] += S0.y * P1;
              accs[1][sc][q][1] += S1.y * P1;
            }
          }
        }
      }
      __syncthreads();   // buffer b is refilled by the next chunk's copies
    }
#pragma unroll
    for (int d = 0; d < 2; d++) {
      if (!(d ? act1 : act0)) continue;
      int l = m + t + d;
      for (int s = 0; s < (m == 0 ? 1 : 2); s++) {
        int jj = jj_of(a, l, m, s);
        double g7 = a.g7[jj], g6 = a.g6[jj];
#pragma unroll
        for (int q = 0; q < FWD_KT; q++) {
          int k = k0 + q;
          if (k >= a.nr) break;
          double r = a.r[k];
          size_t at = (size_t)k * a.jmax + jj;
#pragma unroll
          for (int v = 0; v < NV; v++) {
            double *f0 = a.f + (size_t)a.slot[g0 + v] * a.fs;
            f0[at] = accv[d][v][q][0 + s] * g7 * r * r;
            f0[a.fs + at] = accv[d][v][q][2 + s] * g7 * r;
            f0[2 * a.fs + at] = accv[d][v][q][4 + s] * g7 * r;
          }
#pragma unroll
          for (int sc = 0; sc < NSC; sc++)
            a.f[(size_t)a.slot[g0 + NV + sc] * a.fs + at] = accs[d][sc][q][s] * g6;
        }
      }
    }
  }
}

static LegArgs leg_args(Ctx &c, int nvec, int nscal, const int *slots) {
  LegArgs a;
  a.L = c.L; a.nr = c.nr; a.nth = c.nth; a.nh = c.nh; a.jmax = c.jmax; a.NS = c.NS;
  a.nvec = nvec; a.nscal = nscal; a.ncomp = 3 * nvec + nscal; a.cbase = 0;
  for (int g = 0; g < MAXG; g++) a.slot[g] = 0;
  a.moff = c.d_moff; a.poff = c.d_poff;
  a.Plt = c.d_Plt; a.dPlt = c.d_dPlt; a.Ptl = c.d_Ptl; a.dPtl = c.d_dPtl;
  a.asin_t = c.d_asin; a.wgt = c.d_wgt;
  a.g3rlm = c.d_g3rlm; a.g6 = c.d_g6; a.g7 = c.d_g7; a.r = c.d_r; a.ar1 = c.d_ar1;
  a.f = c.d_f; a.fs = c.fsize();
  return a;
}

template <int KT>
static void launch_bwd(Ctx &c, const LegArgs &b, double *four, int nb) {
  const size_t sm = 2 * ((size_t)MAXG * BWD_LC * KT * 6 + 2 * BWD_LC * 64) * sizeof(double);
  static bool attr = false;   // the kernel's dynamic shared-memory limit, raised once
  if (!attr) {
    cudaFuncSetAttribute(k_leg_bwd_f64<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  dim3 grid(cdiv(c.nh, 64), cdiv(c.nr, KT), c.L + 1);
  k_leg_bwd_f64<KT><<<grid, 32 * nb, sm, c.stream>>>(b, four);
}

void leg_bwd_f64(Ctx &c, int nvec, int nscal, const int *slots, double *four) {
  LegArgs a = leg_args(c, nvec, nscal, slots);
  // launches of at most MAXG groups: vectors first, then scalars
  int g = 0, comp = 0, ngrp = nvec + nscal;
  while (g < ngrp) {
    int nb = std::min(MAXG, ngrp - g);
    LegArgs b = a;
    b.nvec = std::max(0, std::min(nvec - g, nb));
    b.nscal = nb - b.nvec;
    b.cbase = comp;
    for (int q = 0; q < nb; q++) b.slot[q] = slots[g + q];
    // tuning value 2: two radial levels per block, 4: four
    if (c.tune[TUNE_BWD_KT] == 2) launch_bwd<2>(c, b, four, nb);
    else launch_bwd<4>(c, b, four, nb);
    comp += 3 * b.nvec + b.nscal;
    g += nb;
  }
}

template <int NV, int NSC, int KT>
static void launch_fwd_kt(Ctx &c, const LegArgs &a, const double *four, int c0) {
  int nthr = 32 * cdiv(cdiv(std::min(c.L + 1, 512), 2), 32);   // two degrees per thread
  size_t sm = 2 * ((size_t)FWD_TC * KT * (3 * NV + NSC) * 2 * 2 + 2 * (size_t)FWD_TC * (c.L + 1)) * sizeof(double);
  static size_t attr = 0;   // the kernel's dynamic shared-memory limit, raised once per size
  if (sm > 48 * 1024 && sm > attr) {
    cudaFuncSetAttribute(k_leg_fwd_f64<NV, NSC, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = sm;
  }
  dim3 grid(1, cdiv(c.nr, KT), c.L + 1);
  k_leg_fwd_f64<NV, NSC, KT><<<grid, nthr, sm, c.stream>>>(a, four, c0, 0);
}

template <int NV, int NSC>
static void launch_fwd(Ctx &c, LegArgs a, const double *four, int c0, const int *slots) {
  for (int q = 0; q < NV + NSC; q++) a.slot[q] = slots[q];
  switch (c.tune[TUNE_FWD_KT]) {
    case 1: launch_fwd_kt<NV, NSC, 1>(c, a, four, c0); break;
    default: launch_fwd_kt<NV, NSC, 2>(c, a, four, c0); break;
  }
}

void leg_fwd_f64(Ctx &c, int nvec, int nscal, const double *four, const int *slots) {
  LegArgs a = leg_args(c, nvec, nscal, slots);
  int g = 0, comp = 0;
  // vectors in batches of up to 4, scalars in batches of up to 4
  while (g < nvec) {
    int nb = std::min(4, nvec - g);
    if (nb == 4) launch_fwd<4, 0>(c, a, four, comp, slots + g);
    else if (nb == 3) launch_fwd<3, 0>(c, a, four, comp, slots + g);
    else if (nb == 2) launch_fwd<2, 0>(c, a, four, comp, slots + g);
    else launch_fwd<1, 0>(c, a, four, comp, slots + g);
    g += nb;
    comp += 3 * nb;
  }
  int s = 0;
  while (s < nscal) {
    int nb = std::min(4, nscal - s);
    if (nb == 4) launch_fwd<0, 4>(c, a, four, comp, slots + g);
    else if (nb == 3) launch_fwd<0, 3>(c, a, four, comp, slots + g);
    else if (nb == 2) launch_fwd<0, 2>(c, a, four, comp, slots + g);
    else launch_fwd<0, 1>(c, a, four, comp, slots + g);
    g += nb;
    s += nb;
    comp += nb;
  }
}

}  // namespace cb2
