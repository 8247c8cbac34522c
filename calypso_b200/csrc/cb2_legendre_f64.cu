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
// 16-byte form (both addresses 16-byte aligned); n = 0 fills zeros
__device__ inline void cp_async16(double *dst, const double *src, int n) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
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

// ---------------------------------------------------------------------------
// Backward on the float64 tensor cores (mma.sync m16n8k4, f64 in and out).
//
// For one order m and the degrees l of one parity p = (l - m) & 1 the sums
// of k_leg_bwd_f64 are three products whose terms land in the
// reflection-parity accumulators (south node = sigma 0 + sigma 1, mirror
// node = sigma 0 - sigma 1):
//   R  (A = P_l^m):        columns (k, group, s) of X_s, X = S l(l+1)/r^2
//                          (vector) or the scalar          -> sigma = p
//   TP (A = dP_l^m):       columns (k, vector, q) of
//                          [D+, D-, -T+, -T-] (D = dS/dr / r, T = T / r)
//                                                          -> sigma = 1 - p
//   TM (A = m P_l^m / sin): the same columns of [T-, -T+, D-, -D+]
//                                                          -> sigma = p
// with q = 0 v_theta(+m), 1 v_theta(-m), 2 v_phi(+m), 3 v_phi(-m).
// A block takes 64 south nodes (four row tiles of 16) and TKT radial
// levels; per node row tile, TW warps share the column tiles (8 columns
// each; R and TP/TM tiles round-robin).  A chunk of 16 degrees (8 of each
// parity) is staged by cp.async (P, dP by parity [j][node]; the spectra as
// copied), converted into the three B matrices [parity][j][column], and
// consumed by two k4 steps per parity; the next chunk's copies are in flight
// meanwhile.
constexpr int TKT = 2;                      // radial levels per block
constexpr int TW = 2;                       // warps per 16-node row tile
constexpr int TLC = 16;                     // degrees per chunk
constexpr int TMAXG = 6;                    // groups per launch
constexpr int TAP = 68;                     // A row pitch (nodes, 68 = 4 mod 16: no bank conflicts)
constexpr int TRP = ((2 * TMAXG * TKT + 15) / 16) * 16 + 4;   // 36: R pitch, 4 mod 16
constexpr int TTP = ((4 * TMAXG * TKT + 15) / 16) * 16 + 4;   // 52: TP / TM pitch, 4 mod 16
constexpr int TRAW = TKT * TMAXG * 6;       // raw spectral columns of a chunk
constexpr int TMAXT = ((2 * TMAXG * TKT + 7) / 8 + (4 * TMAXG * TKT) / 8 + TW - 1) / TW;   // tiles per warp
constexpr int TBUF = 2 * 2 * (TLC / 2) * TAP + TLC * TRAW;   // one stage: P, dP by parity + raw spectra
constexpr int TBM = 2 * (TLC / 2) * (TRP + 2 * TTP);          // the built B matrices
constexpr int TBST = 2;                                       // staging buffers (cp.async pipeline depth)
// + the column tables (raw offsets, R and T factors, R and T descriptors)
constexpr size_t tc_bwd_smem() {
  return (TBST * (size_t)TBUF + TBM) * sizeof(double) + TRAW * 8 + 6 * TMAXG * TKT * 8 + 6 * TMAXG * TKT * 4;
}

__device__ __forceinline__ void dmma16n8k4(double (&d)[4], double a0, double a1, double b0) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(4 * TW * 32, 2)
k_leg_bwd_f64tc(LegArgs a, double *four) {
  const int m = blockIdx.z, k0 = blockIdx.y * TKT, i0 = blockIdx.x * 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rt = warp / TW, wc = warp - rt * TW;        // row tile (16 nodes), column warp
  const int gq = lane >> 2, tq = lane & 3;              // fragment row / k index
  const int G = a.nvec + a.nscal, nl = a.L + 1 - m;
  const int ncr = 2 * G * TKT, nct = 4 * a.nvec * TKT;  // R and TP/TM columns
  const int nraw = 6 * G * TKT;                         // raw columns ((kq G + g) 3 + comp) 2 + s
  const int ntr = (ncr + 7) / 8, ntt = nct / 8, ntiles = ntr + ntt;
  extern __shared__ __align__(16) double smt[];
  double *BR = smt + TBST * TBUF, *BTP = BR + 2 * (TLC / 2) * TRP, *BTM = BTP + 2 * (TLC / 2) * TTP;
  // per-block column tables, so the staging of a chunk does no index
  // division: raw column -> offset of its degree-m spectral value (-1: a
  // zero column); R column -> raw column (+ 1 << 16 for a vector) and its
  // radial factor; T column -> raw column of its vector's S+ and 1 / r
  long long *rawsrc = reinterpret_cast<long long *>(BTM + 2 * (TLC / 2) * TTP);
  double *rsc = reinterpret_cast<double *>(rawsrc + TRAW), *tsc = rsc + 2 * TMAXG * TKT;
  int *rdesc = reinterpret_cast<int *>(tsc + 4 * TMAXG * TKT), *tdesc = rdesc + 2 * TMAXG * TKT;
  for (int col = tid; col < nraw; col += blockDim.x) {
    const int s = col & 1, comp = (col >> 1) % 3, kg = col / 6, g = kg % G, kq = kg / G, k = k0 + kq;
    long long off = -1;
    if (k < a.nr && !(m == 0 && s == 1) && (g < a.nvec || comp == 0))
      off = (long long)(a.slot[g] + (g < a.nvec ? comp : 0)) * (long long)a.fs + (long long)k * a.jmax +
            a.moff[m] + s * nl;
    rawsrc[col] = off;
  }
  for (int c = tid; c < ncr; c += blockDim.x) {
    const int kg = c >> 1, g = kg % G, k = k0 + kg / G;
    const bool vec = g < a.nvec && k < a.nr;
    const double ar = vec ? a.ar1[k] : 1.0;
    rdesc[c] = kg * 6 + (c & 1) + (vec ? (1 << 16) : 0);
    rsc[c] = ar * ar;
  }
  for (int c = tid; c < nct; c += blockDim.x) {
    const int kv = c >> 2, v = kv % a.nvec, kq = kv / a.nvec, k = k0 + kq;
    tdesc[c] = (kq * G + v) * 6;
    tsc[c] = (k < a.nr) ? a.ar1[k] : 0.0;
  }
  __syncthreads();
  const size_t po = a.poff[m];
  const bool pair16 = (a.nh & 1) == 0;
  // staging of chunk lc0 into stage b: P and dP of the block's 64 nodes by
  // parity [p][j][node], and the raw spectra [raw column][lc]
  auto issue = [&](int lc0, int b) {
    double *st = smt + (size_t)b * TBUF;
    double *Ps = st, *dPs = st + 2 * (TLC / 2) * TAP, *raw = st + 4 * (TLC / 2) * TAP;
    if (pair16) {
      // two nodes per 16-byte copy (nh even: every row starts 16-byte aligned)
      for (int e = tid; e < TLC * 32; e += blockDim.x) {
        const int lc = e >> 5, nd = (e & 31) * 2, ii = i0 + nd, t = lc0 + lc;
        const bool in = t < nl && ii < a.nh;
        const size_t at = in ? po + (size_t)t * a.nh + ii : 0;
        const int o = ((lc & 1) * (TLC / 2) + (lc >> 1)) * TAP + nd;
        cp_async16(Ps + o, a.Plt + at, in ? 16 : 0);
        cp_async16(dPs + o, a.dPlt + at, in ? 16 : 0);
      }
    } else {
      for (int e = tid; e < TLC * 64; e += blockDim.x) {
        const int lc = e >> 6, nd = e & 63, ii = i0 + nd, t = lc0 + lc;
        const bool in = t < nl && ii < a.nh;
        const size_t at = in ? po + (size_t)t * a.nh + ii : 0;
        const int o = ((lc & 1) * (TLC / 2) + (lc >> 1)) * TAP + nd;
        cp_async8(Ps + o, a.Plt + at, in ? 8 : 0);
        cp_async8(dPs + o, a.dPlt + at, in ? 8 : 0);
      }
    }
    for (int e = tid; e < TLC * nraw; e += blockDim.x) {
      const int lc = e & (TLC - 1), col = e >> 4;
      const long long so = rawsrc[col];
      const bool in = so >= 0 && lc0 + lc < nl;
      cp_async8(raw + col * TLC + lc, in ? a.f + so + lc0 + lc : a.f, in ? 8 : 0);
    }
    cp_async_commit();
  };
  // raw spectra of stage b -> B matrices (radial and degree factors, signs)
  auto build = [&](int lc0, int b) {
    const double *raw = smt + (size_t)b * TBUF + 4 * (TLC / 2) * TAP;
    // lanes along the degrees of a column: consecutive raw addresses
    for (int e = tid; e < TLC * 32; e += blockDim.x) {
      const int c = e >> 4, lc = e & (TLC - 1);
      if (c >= ncr) continue;
      const int rd = rdesc[c], l = m + lc0 + lc;
      double x = raw[(rd & 0xffff) * TLC + lc];
      if (rd >> 16) x *= rsc[c] * ((l == 0) ? 0.5 : (double)l * (double)(l + 1));
      BR[((lc & 1) * (TLC / 2) + (lc >> 1)) * TRP + c] = x;
    }
    for (int e = tid; e < TLC * 64; e += blockDim.x) {
      const int c = e >> 4, lc = e & (TLC - 1);
      if (c >= nct) continue;
      const int q = c & 3;
      const double ar = tsc[c];
      const double *rw = raw + tdesc[c] * TLC + lc;   // S+ S- D+ D- T+ T-, TLC apart
      const double Dp = rw[2 * TLC] * ar, Dm = rw[3 * TLC] * ar, Tp = rw[4 * TLC] * ar, Tm = rw[5 * TLC] * ar;
      const int o = ((lc & 1) * (TLC / 2) + (lc >> 1));
      BTP[o * TTP + c] = (q == 0) ? Dp : (q == 1) ? Dm : (q == 2) ? -Tp : -Tm;
      BTM[o * TTP + c] = (q == 0) ? Tm : (q == 1) ? -Tp : (q == 2) ? Dm : -Dp;
    }
    // padding columns of the last R tile stay zero
    for (int e = tid; e < TLC * 8; e += blockDim.x) {
      const int lc = e >> 3, c = ncr + (e & 7);
      if (c < ntr * 8) BR[((lc & 1) * (TLC / 2) + (lc >> 1)) * TRP + c] = 0.0;
    }
  };
  double acc[TMAXT][2][4];
#pragma unroll
  for (int i = 0; i < TMAXT; i++)
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int u = 0; u < 4; u++) acc[i][p][u] = 0.0;
  // m / sin(theta) of this thread's two fragment rows
  const int na = i0 + 16 * rt + gq, nb = na + 8;
  const double ama = (na < a.nh) ? (double)m * a.asin_t[na] : 0.0;
  const double amb = (nb < a.nh) ? (double)m * a.asin_t[nb] : 0.0;
  const int nch = (nl + TLC - 1) / TLC;
  issue(0, 0);
  for (int ch = 0; ch < nch; ch++) {
    const int lc0 = ch * TLC, b = ch & 1;
    if (ch + 1 < nch) issue(lc0 + TLC, b ^ 1);
    else cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    build(lc0, b);
    __syncthreads();
    const double *Ps = smt + (size_t)b * TBUF, *dPs = Ps + 2 * (TLC / 2) * TAP;
#pragma unroll
    for (int p = 0; p < 2; p++) {
#pragma unroll
      for (int ks = 0; ks < TLC / 8; ks++) {
        const int j = ks * 4 + tq, o = (p * (TLC / 2) + j);
        const double pa = Ps[o * TAP + 16 * rt + gq], pb = Ps[o * TAP + 16 * rt + gq + 8];
        const double da = dPs[o * TAP + 16 * rt + gq], db = dPs[o * TAP + 16 * rt + gq + 8];
        const double ma = pa * ama, mb = pb * amb;
#pragma unroll
        for (int i = 0; i < TMAXT; i++) {
          const int jt = wc + TW * i;
          if (jt < ntt) {
            const double btp = BTP[o * TTP + 8 * jt + gq], btm = BTM[o * TTP + 8 * jt + gq];
            dmma16n8k4(acc[i][p ^ 1], da, db, btp);
            dmma16n8k4(acc[i][p], ma, mb, btm);
          } else if (jt < ntiles) {
            const double br = BR[o * TRP + 8 * (jt - ntt) + gq];
            dmma16n8k4(acc[i][p], pa, pb, br);
          }
        }
      }
    }
    __syncthreads();   // stage b and the B matrices are refilled next
  }
  // south / mirror values of each fragment: rows na, nb; columns 2 tq, 2 tq + 1
  // are the orders +m and -m of one component
#pragma unroll
  for (int i = 0; i < TMAXT; i++) {
    const int jt = wc + TW * i;
    if (jt >= ntiles) continue;
    int kq, c;
    if (jt < ntt) {
      const int cc = 8 * jt + 2 * tq, kv = cc >> 2, v = kv % a.nvec;
      kq = kv / a.nvec;
      c = a.cbase + 3 * v + 1 + ((cc & 3) >> 1);
    } else {
      const int cc = 8 * (jt - ntt) + 2 * tq;
      if (cc >= ncr) continue;
      const int kg = cc >> 1, g = kg % G;
      kq = kg / G;
      c = a.cbase + (g < a.nvec ? 3 * g : 3 * a.nvec + (g - a.nvec));
    }
    const int k = k0 + kq;
    if (k >= a.nr) continue;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int n = h ? nb : na;
      if (n >= a.nh) continue;
      const double e0 = acc[i][0][2 * h], e1 = acc[i][0][2 * h + 1];
      const double o0 = acc[i][1][2 * h], o1 = acc[i][1][2 * h + 1];
      const double2 south = make_double2(e0 + o0, m == 0 ? 0.0 : e1 + o1);
      const double2 north = make_double2(e0 - o0, m == 0 ? 0.0 : e1 - o1);
      *reinterpret_cast<double2 *>(four + four_at(a, n, k, c) + 2 * m) = south;
      *reinterpret_cast<double2 *>(four + four_at(a, a.nth - 1 - n, k, c) + 2 * m) = north;
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

// ---------------------------------------------------------------------------
// Forward on the float64 tensor cores (mma.sync m16n8k4).  For one order m
// and the degrees of one parity p the sums of k_leg_fwd_f64 are products
// over the south nodes i (K) of the tables (rows: degrees) with the
// Gauss-weighted symmetric / antisymmetric grid sums H (same = the sums of
// the parity of P, other = the converse):
//   R  (A = P):   columns (k, group, s): R_same(s) or the scalar's S_same(s)
//   TP (A = dP):  columns (k, vector, q): [T_other(+), T_other(-),
//                 -F_other(+), -F_other(-)]
//   TM (A = P, rows of B times m / sin theta_i): the same columns of
//                 [-F_same(-), F_same(+), -T_same(-), T_same(+)]
// with q = 0, 1 the dS/dr coefficient of orders +m, -m and q = 2, 3 the
// toroidal one.  A block takes 64 degrees (two 16-row tiles of each parity)
// and TKT radial levels and walks the nodes in chunks of 16 (four k4
// steps): the P and dP rows of its degrees and the raw grid values of the
// chunk's nodes and mirrors by cp.async (the next chunk in flight), then
// the weighted sums built into the B matrices of both parities.
constexpr int TFC = 16;                     // nodes per chunk
constexpr int TFAP = TFC + 4;               // A row pitch (20 = 4 mod 16)
constexpr int TFRAW = TKT * (3 * TMAXG) * 2 * 2;   // raw values of a node: (k, comp, s, node / mirror)
constexpr int TFBUF = 2 * 64 * TFAP + TFC * TFRAW; // one stage: P, dP rows, raw values
constexpr int TFBM = 2 * TFC * (TRP + 2 * TTP);   // the B matrices of both parities
// + the column tables (raw offsets, R and T descriptors)
constexpr size_t tc_fwd_smem() {
  return (2 * (size_t)TFBUF + TFBM) * sizeof(double) + (TFRAW / 2) * 8 + 6 * TMAXG * TKT * 4;
}

__global__ void __launch_bounds__(4 * TW * 32, 2)
k_leg_fwd_f64tc(LegArgs a, const double *four) {
  const int m = blockIdx.z, k0 = blockIdx.y * TKT, t0 = blockIdx.x * 64;   // degree offset l - m
  const int nl = a.L + 1 - m;
  if (t0 >= nl) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rt = warp / TW, wc = warp - rt * TW;         // row tile: parity rt & 1, half rt >> 1
  const int gq = lane >> 2, tq = lane & 3;
  const int G = a.nvec + a.nscal, C = 3 * a.nvec + a.nscal;
  const int ncr = 2 * G * TKT, nct = 4 * a.nvec * TKT, nrw = 4 * C * TKT;
  const int ntr = (ncr + 7) / 8, ntt = nct / 8, ntiles = ntr + ntt;
  extern __shared__ __align__(16) double smf[];
  double *BR = smf + 2 * TFBUF, *BTP = BR + 2 * TFC * TRP, *BTM = BTP + 2 * TFC * TTP;
  // per-block column tables, so the staging of a chunk does no index
  // division: raw value x = ((kq C + c) 2 + s) 2 + h -> offset of its
  // (k, component, order) in a Fourier row (-1: a zero value); R column ->
  // raw value of its node (h = 0); T column -> raw value of its vector's
  // theta component (s = 0, h = 0)
  long long *rawsrc = reinterpret_cast<long long *>(BTM + 2 * TFC * TTP);
  int *rdesc = reinterpret_cast<int *>(rawsrc + TFRAW / 2), *tdesc = rdesc + 2 * TMAXG * TKT;
  for (int x2 = tid; x2 < nrw / 2; x2 += blockDim.x) {   // x2 = (kq C + c) 2 + s
    const int s = x2 & 1, kc = x2 >> 1, c = kc % C, k = k0 + kc / C;
    rawsrc[x2] = (k < a.nr && !(m == 0 && s == 1))
                     ? (long long)(((size_t)k * a.ncomp + a.cbase + c) * a.NS + 2 * m + s) : -1;
  }
  for (int cc = tid; cc < ncr; cc += blockDim.x) {   // cc = (kq G + g) 2 + s
    const int s = cc & 1, kg = cc >> 1, g = kg % G, kq = kg / G;
    const int c = (g < a.nvec) ? 3 * g : 3 * a.nvec + (g - a.nvec);
    rdesc[cc] = ((kq * C + c) * 2 + s) * 2;
  }
  for (int cc = tid; cc < nct; cc += blockDim.x) {   // cc = (kq nvec + v) 4 + q
    const int kv = cc >> 2, v = kv % a.nvec, kq = kv / a.nvec;
    tdesc[cc] = ((kq * C + 3 * v + 1) * 2) * 2;
  }
  __syncthreads();
  const size_t po = a.poff[m];
  const bool pair16 = (a.nh & 1) == 0;
  const size_t rowst = (size_t)a.nr * a.ncomp * a.NS;   // one colatitude of the Fourier buffer
  // stage b: P, dP of the block's degrees (row r = 32 p + j, degree
  // t0 + 2 j + p) at the chunk's nodes [r][node]; raw grid values
  // [node][x], h = 0 the node, 1 its mirror
  auto issue = [&](int ib, int b) {
    double *st = smf + (size_t)b * TFBUF, *Ps = st, *dPs = st + 64 * TFAP, *raw = st + 2 * 64 * TFAP;
    if (pair16) {
      // two nodes per 16-byte copy (nh even: every row starts 16-byte aligned)
      for (int e = tid; e < 64 * TFC / 2; e += blockDim.x) {
        const int r = e >> 3, nd = (e & 7) * 2, t = t0 + 2 * (r & 31) + (r >> 5), i = ib + nd;
        const bool in = t < nl && i < a.nh;
        const size_t at = in ? po + (size_t)t * a.nh + i : 0;
        cp_async16(Ps + r * TFAP + nd, a.Plt + at, in ? 16 : 0);
        cp_async16(dPs + r * TFAP + nd, a.dPlt + at, in ? 16 : 0);
      }
    } else {
      for (int e = tid; e < 64 * TFC; e += blockDim.x) {
        const int r = e >> 4, nd = e & (TFC - 1), t = t0 + 2 * (r & 31) + (r >> 5), i = ib + nd;
        const bool in = t < nl && i < a.nh;
        const size_t at = in ? po + (size_t)t * a.nh + i : 0;
        cp_async8(Ps + r * TFAP + nd, a.Plt + at, in ? 8 : 0);
        cp_async8(dPs + r * TFAP + nd, a.dPlt + at, in ? 8 : 0);
      }
    }
    for (int e = tid; e < TFC * 128; e += blockDim.x) {
      const int nd = e >> 7, x = e & 127, i = ib + nd;
      if (x >= nrw) continue;
      const long long so = rawsrc[x >> 1];
      const bool in = so >= 0 && i < a.nh;
      const size_t th = (x & 1) ? (size_t)(a.nth - 1 - i) : (size_t)i;
      cp_async8(raw + nd * TFRAW + x, in ? four + th * rowst + so : four, in ? 8 : 0);
    }
    cp_async_commit();
  };
  // weighted sums of stage b -> B matrices of both parities [p][node][col]
  auto build = [&](int ib, int b) {
    const double *raw = smf + (size_t)b * TFBUF + 2 * 64 * TFAP;
    for (int e = tid; e < TFC * 32; e += blockDim.x) {
      const int nd = e >> 5, cc = e & 31, i = ib + nd;
      if (cc >= ncr) continue;
      double sym = 0.0, anti = 0.0;
      if (i < a.nh) {
        const double *rv = raw + nd * TFRAW + rdesc[cc];
        const double fa = rv[0] * a.wgt[i], fb = rv[1] * a.wgt[a.nth - 1 - i];
        sym = fa + fb; anti = fa - fb;
      }
      BR[(0 * TFC + nd) * TRP + cc] = sym;
      BR[(1 * TFC + nd) * TRP + cc] = anti;
    }
    for (int e = tid; e < TFC * 64; e += blockDim.x) {
      const int nd = e >> 6, cc = e & 63, i = ib + nd;
      if (cc >= nct) continue;
      const int q = cc & 3;
      double Ts[2] = {0, 0}, Ta[2] = {0, 0}, Fs[2] = {0, 0}, Fa[2] = {0, 0}, ams = 0.0;
      if (i < a.nh) {
        const double wa = a.wgt[i], wb = a.wgt[a.nth - 1 - i];
        const double *rt_ = raw + nd * TFRAW + tdesc[cc];   // theta (s 0, 1; node, mirror)
        const double *rf_ = rt_ + 4;                          // phi
        for (int s = 0; s < 2; s++) {
          const double ta = rt_[2 * s] * wa, tb = rt_[2 * s + 1] * wb;
          const double fa = rf_[2 * s] * wa, fb = rf_[2 * s + 1] * wb;
          Ts[s] = ta + tb; Ta[s] = ta - tb; Fs[s] = fa + fb; Fa[s] = fa - fb;
        }
        ams = (double)m * a.asin_t[i];
      }
      // parity 0: same = symmetric, other = antisymmetric; parity 1 the converse
      for (int p = 0; p < 2; p++) {
        const double *Tsm = p ? Ta : Ts, *Tot = p ? Ts : Ta, *Fsm = p ? Fa : Fs, *Fot = p ? Fs : Fa;
        const double tp = (q == 0) ? Tot[0] : (q == 1) ? Tot[1] : (q == 2) ? -Fot[0] : -Fot[1];
        const double tm = (q == 0) ? -Fsm[1] : (q == 1) ? Fsm[0] : (q == 2) ? -Tsm[1] : Tsm[0];
        BTP[(p * TFC + nd) * TTP + cc] = tp;
        BTM[(p * TFC + nd) * TTP + cc] = tm * ams;
      }
    }
    for (int e = tid; e < TFC * 8; e += blockDim.x) {
      const int nd = e >> 3, cc = ncr + (e & 7);
      if (cc < ntr * 8) {
        BR[nd * TRP + cc] = 0.0;
        BR[(TFC + nd) * TRP + cc] = 0.0;
      }
    }
  };
  double acc[TMAXT][4];
#pragma unroll
  for (int i = 0; i < TMAXT; i++)
#pragma unroll
    for (int u = 0; u < 4; u++) acc[i][u] = 0.0;
  const int p = rt & 1, ar0 = 32 * p + 16 * (rt >> 1);   // this warp's A rows
  const int nchk = (a.nh + TFC - 1) / TFC;
  issue(0, 0);
  for (int ch = 0; ch < nchk; ch++) {
    const int ib = ch * TFC, b = ch & 1;
    if (ch + 1 < nchk) issue(ib + TFC, b ^ 1);
    else cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    build(ib, b);
    __syncthreads();
    const double *Ps = smf + (size_t)b * TFBUF, *dPs = Ps + 64 * TFAP;
#pragma unroll
    for (int ks = 0; ks < TFC / 4; ks++) {
      const int kk = 4 * ks + tq;
      const double pa = Ps[(ar0 + gq) * TFAP + kk], pb = Ps[(ar0 + gq + 8) * TFAP + kk];
      const double da = dPs[(ar0 + gq) * TFAP + kk], db = dPs[(ar0 + gq + 8) * TFAP + kk];
      const int bo = p * TFC + kk;
#pragma unroll
      for (int i = 0; i < TMAXT; i++) {
        const int jt = wc + TW * i;
        if (jt < ntt) {
          dmma16n8k4(acc[i], da, db, BTP[bo * TTP + 8 * jt + gq]);
          dmma16n8k4(acc[i], pa, pb, BTM[bo * TTP + 8 * jt + gq]);
        } else if (jt < ntiles) {
          dmma16n8k4(acc[i], pa, pb, BR[bo * TRP + 8 * (jt - ntt) + gq]);
        }
      }
    }
    __syncthreads();   // stage b and the B matrices are refilled next
  }
  // rows: degrees t0 + 2 (16 (rt >> 1) + gq (+ 8)) + p; columns 2 tq, 2 tq + 1
  // are the orders +m and -m
#pragma unroll
  for (int i = 0; i < TMAXT; i++) {
    const int jt = wc + TW * i;
    if (jt >= ntiles) continue;
    int kq, slot, kind;   // kind 0: r^2 g7 (poloidal), 1: r g7, 2: g6 (scalar)
    if (jt < ntt) {
      const int cc = 8 * jt + 2 * tq, kv = cc >> 2, v = kv % a.nvec;
      kq = kv / a.nvec;
      slot = a.slot[v] + 1 + ((cc & 3) >> 1);
      kind = 1;
    } else {
      const int cc = 8 * (jt - ntt) + 2 * tq;
      if (cc >= ncr) continue;
      const int kg = cc >> 1, g = kg % G;
      kq = kg / G;
      slot = a.slot[g];
      kind = (g < a.nvec) ? 0 : 2;
    }
    const int k = k0 + kq;
    if (k >= a.nr) continue;
    const double r = a.r[k];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int t = t0 + 2 * (16 * (rt >> 1) + gq + 8 * h) + p;
      if (t >= nl) continue;
      const int l = m + t;
#pragma unroll
      for (int s = 0; s < 2; s++) {
        if (s == 1 && m == 0) break;   // order -m exists for m > 0 only
        const int jj = jj_of(a, l, m, s);
        const double fac = (kind == 0) ? a.g7[jj] * r * r : (kind == 1) ? a.g7[jj] * r : a.g6[jj];
        a.f[(size_t)slot * a.fs + (size_t)k * a.jmax + jj] = acc[i][2 * h + s] * fac;
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

static void launch_bwd_tc(Ctx &c, const LegArgs &b, double *four) {
  static bool attr = false;   // the kernel's dynamic shared-memory limit, raised once
  if (!attr) {
    cudaFuncSetAttribute(k_leg_bwd_f64tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_bwd_smem());
    attr = true;
  }
  dim3 grid(cdiv(c.nh, 64), cdiv(c.nr, TKT), c.L + 1);
  k_leg_bwd_f64tc<<<grid, 4 * TW * 32, tc_bwd_smem(), c.stream>>>(b, four);
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
    // tuning value 1: the tensor-core kernel; 2 or 4: the CUDA-core kernel
    // with two or four radial levels per block
    if (c.tune[TUNE_BWD_KT] == 1) launch_bwd_tc(c, b, four);
    else if (c.tune[TUNE_BWD_KT] == 2) launch_bwd<2>(c, b, four, nb);
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

static void launch_fwd_tc(Ctx &c, const LegArgs &b, const double *four) {
  static bool attr = false;   // the kernel's dynamic shared-memory limit, raised once
  if (!attr) {
    cudaFuncSetAttribute(k_leg_fwd_f64tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_fwd_smem());
    attr = true;
  }
  dim3 grid(cdiv(c.L + 1, 64), cdiv(c.nr, TKT), c.L + 1);
  k_leg_fwd_f64tc<<<grid, 4 * TW * 32, tc_fwd_smem(), c.stream>>>(b, four);
}

void leg_fwd_f64(Ctx &c, int nvec, int nscal, const double *four, const int *slots) {
  LegArgs a = leg_args(c, nvec, nscal, slots);
  if (c.tune[TUNE_FWD_KT] == 3 && nvec <= 5) {
    // the tensor-core kernel: launches of at most TMAXG groups, vectors
    // first (at most 16 components in a launch: its staging maps the raw
    // values of a node with a stride of 128 = 4 x 16 x TKT)
    int g = 0, comp = 0;
    const int ngrp = nvec + nscal;
    while (g < ngrp) {
      const int nb = std::min(TMAXG, ngrp - g);
      LegArgs b = a;
      b.nvec = std::max(0, std::min(nvec - g, nb));
      b.nscal = nb - b.nvec;
      b.cbase = comp;
      for (int q = 0; q < nb; q++) b.slot[q] = slots[g + q];
      launch_fwd_tc(c, b, four);
      comp += 3 * b.nvec + b.nscal;
      g += nb;
    }
    return;
  }
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
