// cb2_legendre_mixed.cu -- Legendre transforms on the tcgen05 tensor cores.
//
// Arithmetic: every operand x is scaled by a power of two s (per GEMM row or
// column, so the largest |x s| lies in [2^13, 2^14)) and split into two
// float16 halves
//     x s = hi + lo,  hi = fp16(x s),  lo = fp16(x s - hi),
// and a product is accumulated in float32 as hi*hi' + hi*lo' + lo*hi'
// (three tcgen05.mma kind::f16), unscaled in the epilogue.  Scaling to 2^14
// rather than 1 keeps lo a normal fp16 number for every value within 2^17 of
// the row (column) maximum, so those values carry 22 significant bits;
// smaller ones keep an absolute error of ~2^-38 of the maximum.  The float32
// accumulator is rounded after every MMA, which sets the error of these
// transforms (dropping the lo*lo' term changes nothing measurable): the
// backward kernel adds the three products into one TMEM accumulator, the
// forward kernel (longer K: all colatitudes of a hemisphere, twice for the
// theta/phi block) keeps hi*hi' and the cross terms, 2^-11 smaller, in two
// accumulators summed in the epilogue, so the large one is rounded a third
// as often.
//
// Mathematics: the per-order contractions of legendre_bwd_trans_org.f90 /
// legendre_fwd_trans_org.f90 of the reference (the float64 version is
// cb2_legendre_f64.cu), written as GEMMs per order m with the equatorial
// symmetry P_l^m(pi - t) = (-1)^(l-m) P_l^m(t):
//
// backward, D[row][theta] = sum_K A[row][K] B[K][theta] over the nh south
//   nodes; two TMEM accumulators, one per reflection parity of the basis
//   function, give the south (acc0 + acc1) and north (acc0 - acc1) nodes.
//   gemm P   rows (k, group, +-m): A = S l(l+1)/r^2 (vectors) or the scalar,
//            B = P_l^m; K runs over the degrees of one parity of l-m.
//   gemm DM  rows (k, vector, {theta +m, theta -m, phi +m, phi -m}):
//            K = [dP part | mP part], B = [dP_l^m/dtheta ; m P_l^m/sin theta]
//            grouped as {dP of odd l-m, mP of even l-m} (parity 0) and the
//            converse (parity 1); A = dP part {D+, D-, -T+, -T-}, mP part
//            {T-, -T+, D-, -D+} with D = (dS/dr)/r, T = T/r.
// forward, D[row][l] = sum_theta A[row][theta] B[theta][l] with the Gauss
//   weights and the north/south fold in A (sym = f(i)w_i + f(i')w_i',
//   anti = f(i)w_i - f(i')w_i'); one accumulator per parity of l-m.
//   gemm P   rows (k, group, +-m): A = sym/anti of the r component (vectors)
//            or the scalar, B = P_l^m.
//   gemm DM  rows (k, vector, {dS +m, dS -m, T +m, T -m}), K = [dP | mP].
//
// One CTA = (order m, gemm, tile of 128 rows), 4 warps.  The warps build the
// A tile (scaled fp16 hi/lo, 128-byte swizzled, K-major) in shared memory
// while one thread issues the TMA loads of the B tiles (hi/lo) and the MMAs;
// two pipeline stages overlap the three.  The accumulators live in TMEM (two
// x up to 256 fp32 columns) and the 4 warps read them back with tcgen05.ld
// (warp w owns TMEM lanes 32w..32w+31 = tile rows).  Every mbarrier wait is
// bounded in time: a wait that runs out sets bit 2 of the context's status
// word, the CTA drains its own TMA loads and MMAs (bounded again), releases
// TMEM and returns without writing results; the host reports the status.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cb2_internal.cuh"
#include "cb2_tc.cuh"

namespace cb2 {

namespace {

constexpr int TM = 128;          // GEMM rows per tile (= TMEM lanes)
using namespace tc;

// largest scaled magnitude: 2^13 <= mx s < 2^14 (fp16 holds up to 65504)
constexpr int kScaleExp = 14;

// power-of-two scale for a row (column) whose largest |x| is mx; the exponent
// is clamped so neither s nor 1/s leaves the float range (1 for an all-zero row)
__host__ __device__ inline float pow2_scale(double mx) {
  if (!(mx > 0.0) || !(mx < 1e300)) return 1.0f;
  int e;
  frexp(mx, &e);
  int sh = kScaleExp - e;
  sh = sh < -120 ? -120 : (sh > 120 ? 120 : sh);
  return ldexpf(1.0f, sh);
}

// x0, x1 -> fp16 hi and lo pairs (x = hi + lo to 22 bits), x0 in the low
// half; the paired conversions run on the full-rate pipes
__device__ inline void split_pair(float x0, float x1, uint32_t &hi, uint32_t &lo) {
  const __half2 h = __floats2half2_rn(x0, x1);
  const float2 f = __half22float2(h);
  const __half2 l = __floats2half2_rn(x0 - f.x, x1 - f.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// the same with hi on a fixed grid: hi = x rounded to a multiple of 16 (x
// scaled below 2^14, so hi is an fp16 number of at most 11 bits), lo = the
// remainder (|lo| <= 8, 11 bits of it kept, 2^-23 of the row maximum).  Every
// product hi*hi' is then a multiple of 256 below 2^28, and an FP32
// accumulator holds their sums exactly while they stay below 2^32.
// The scalings by 2^-4 and 2^4 and the difference x - hi are exact, so the
// packed float32x2 forms of sm_100 give the scalar results bit for bit.
__device__ inline void split_pair_q(float x0, float x1, uint32_t &hi, uint32_t &lo) {
  const float2 x = make_float2(x0, x1);
  const float2 s = __fmul2_rn(x, make_float2(0.0625f, 0.0625f));
  const float2 hq = __fmul2_rn(make_float2(rintf(s.x), rintf(s.y)), make_float2(16.0f, 16.0f));
  const float2 r = __ffma2_rn(hq, make_float2(-1.0f, -1.0f), x);
  const __half2 h = __floats2half2_rn(hq.x, hq.y);
  const __half2 l = __floats2half2_rn(r.x, r.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// ---------------------------------------------------------------------------
// forward: order-major Fourier rows -> spectra f[slot][k][jj]
//
// A tile = (order m, gemm, 128 rows).  For each block of 32 south nodes tb,
// TMA brings the raw float32 rows of the tile at those 32 colatitudes and at
// their 32 mirror nodes ([theta][row], 16 KB each); converter threads form
// the folded, weighted operands of both parities of l-m
//   A[row][i] = sg * s_row * (f(i) w_i +- f(i') w_i')     (i' = nth-1-i)
// split into fp16 hi / lo (64-byte swizzled, K = 32) while TMA brings the
// B tiles (P_l^m rows of each parity, 64-byte swizzled).  gemm P takes one
// K block per tb; gemm DM two (dP part: element `row`, fold 1-p; mP part:
// element row - q + 3 - q, fold p).  One accumulator per parity
// (N = degrees of that parity).
constexpr int FKB = 32;            // K per block (64-byte rows)
constexpr uint32_t RAW_BYTES = 2 * FKB * TM * 4;    // south + north, float32
constexpr uint32_t FA_BYTES = TM * FKB * 2;         // one of hi / lo

struct FwdArgs {
  int L, nr, jmax, nh, nhp, nth, nvec, nscal, NFmax, boxr, nfb;   // nfb: B rows in smem
  int slot[8];
  const int *moff;
  const double *g6, *g7, *r;
  const float *wgt;      // Gauss weights (float), nth
  double *f;
  size_t fs;
  size_t sP, sD;         // block strides of the input layout
  const float *bunscale; // [gemm][(m, parity)][NFmax] 1 / column scale of B
  const int *roff, *nlp; // B row offset and number of degrees of (m, parity)
  const float *rowmax;   // [m][element], k_rowmax_four
  int *status;
  unsigned long long wait_ns;   // budget of each pipeline wait (Ctx::pipe_wait_ns)
  int split;             // 1: hi*hi' and the cross terms in separate accumulators
};

// Forward stages: both parities come from one raw tile (the symmetric and
// the antisymmetric fold), so a K block has two raw halves (south + north,
// 32 KB together), the A tiles of both parities (4 x 8 KB) and their B
// tiles.
constexpr int FRS = 2;   // raw stages
constexpr int FAB = 2;   // A/B stages

// ---------------------------------------------------------------------------
// forward, warp-specialised and persistent: one CTA per SM walks the tiles
// (m, gemm, 128 rows) in order-major order, so the CTAs in flight share the
// basis tables of a few orders in L2.  Roles:
//   warps 0-7   converters: raw float32 rows (TMA) -> scaled, folded, split
//               fp16 hi/lo A operands (64-byte swizzle), both parities
//   warps 8-15  epilogue: TMEM (16x256b loads, the two parities side by
//               side) -> float64 degree runs of each row, geometric factors
//   warp 16     TMA producer (raw rows and basis tiles)
//   warp 17     MMA issuer (tcgen05, one elected thread)
// Two TMEM accumulator sets (when they fit) let the epilogue of one tile
// overlap the main loop of the next; with one set, the tiles narrow enough
// for half of tensor memory alternate between the halves (AccSched).
constexpr int FW_CONV = 256, FW_EPI = 256, FW_THREADS = FW_CONV + FW_EPI + 64;
constexpr int FW_PROD_WARP = (FW_CONV + FW_EPI) / 32, FW_MMA_WARP = FW_PROD_WARP + 1;

// epilogue staging of one warp: 16 rows x 16 degrees (+1 pad) floats, then
// the row metadata (destination offset, scale, factor select) of its 16 rows
constexpr int FW_STG_P = 17;
constexpr uint32_t FW_STG_BYTES = ((16 * FW_STG_P * 8 + 16 * 8 + 16 * 8 + 16 * 4) + 15) & ~15u;

struct FwdWsLayout {
  uint32_t raw, ab, stg, w, bar, total;   // byte offsets from the aligned base
};

__host__ __device__ inline FwdWsLayout fwd_ws_layout(int nfb, int L, int nth) {
  FwdWsLayout o;
  uint32_t p = 0;
  const uint32_t bbytes = (uint32_t)nfb * FKB * 2;
  o.raw = p; p += FRS * RAW_BYTES;
  o.ab = p; p += FAB * (4 * FA_BYTES + 4 * bbytes);
  o.stg = p; p += (FW_EPI / 32) * FW_STG_BYTES;
  o.w = p; p += ((uint32_t)nth * 4 + 15) & ~15u;
  o.bar = p; p += 256;
  o.total = p;
  return o;
}

struct FwdWsBars {
  uint64_t rawfull[FRS], rawempty[FRS], afull[FAB], bfull[FAB], abempty[FAB];
  uint64_t accfull[2], accempty[2], fin;
  uint32_t tmem_base;
  int abort, skip;
};

struct FwdTile {
  int m, g, row0, nrows, np0, np1, npad0, npad1, nbox0, nbox1, brow0, brow1, NB;
};

__device__ inline FwdTile fwd_tile(const FwdArgs &a, int t, int rows_g0, int rows_g1, int tiles_g0, int tiles_g1) {
  FwdTile q;
  const int tpm = tiles_g0 + tiles_g1;
  q.m = t / tpm;
  const int x = t - q.m * tpm;
  q.g = (x >= tiles_g0) ? 1 : 0;
  q.row0 = (q.g ? x - tiles_g0 : x) * TM;
  q.nrows = q.g ? rows_g1 : rows_g0;
  q.np0 = a.nlp[q.m * 2];
  q.np1 = a.nlp[q.m * 2 + 1];
  q.npad0 = ((q.np0 + 15) / 16) * 16;
  q.npad1 = ((q.np1 + 15) / 16) * 16;
  q.nbox0 = (q.npad0 + a.boxr - 1) / a.boxr;
  q.nbox1 = (q.npad1 + a.boxr - 1) / a.boxr;
  q.brow0 = a.roff[q.m * 2];
  q.brow1 = a.roff[q.m * 2 + 1];
  const int NT = (a.nh + FKB - 1) / FKB;
  q.NB = q.g ? 2 * NT : NT;
  return q;
}

// row scale of tile row `row` (converters and epilogue compute the same value)
__device__ inline float fwd_row_scale(const FwdArgs &a, const FwdTile &q, int row) {
  float mx = 0.0f;
  if (row < q.nrows) {
    const float *Mf = a.rowmax + (size_t)q.m * (a.sP + a.sD);
    const int q4 = row & 3;
    if (q.g == 0) mx = Mf[row];
    else mx = fmaxf(Mf[a.sP + row], Mf[a.sP + row - q4 + 3 - q4]);
  }
  return pow2_scale(mx);
}

template <typename Bars>
__device__ inline bool ws_aborted(const Bars *sb) { return *(volatile const int *)&sb->abort != 0; }

// One shell of a forward launch: its tensor maps (raw Fourier rows of both
// gemms, B tables hi / lo of both gemms), arguments and tile counts.  A
// single-shell launch takes it as a kernel parameter; an ensemble launch
// reads a table of them from device memory, shell s owning the tiles
// tile0(s) .. tile0(s + 1) - 1 of the launch.
struct FwdShell {
  CUtensorMap rawP, rawD, phi, plo, dhi, dlo;   // 64-byte aligned
  FwdArgs a;
  int rows_g0, rows_g1, tiles_g0, tiles_g1, tile0;
};

// the shell that owns tile t (tile0 ascending, tab[0].tile0 == 0)
template <typename S>
__device__ inline const S &shell_of(const S *tab, int nsh, int t) {
  int lo = 0, hi = nsh - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&tab[mid].tile0) <= t) lo = mid;
    else hi = mid - 1;
  }
  return tab[lo];
}

// Accumulator schedule of a forward CTA, stepped tile by tile in the same
// way by the MMA thread and by the epilogue warps.  With two accumulator
// sets the tiles alternate between them.  With one set of four 128-column
// accumulators (the split layout at L255: 512 columns), a tile whose
// accumulators fit in 64 columns takes one half of tensor memory, the halves
// alternating, so its epilogue overlaps the next such tile's MMAs; a wider
// tile takes both halves.  Per half: how often it has been taken (the MMA
// waits for the previous release); per full barrier: how often committed.
struct AccSched {
  int dyn, next;
  uint32_t acq0, acq1, full0, full1;
};
struct AccUse {
  int nh, h0, sfull, wait0, wait1;   // halves h0 (and 1 when nh = 2)
  uint32_t par0, par1, full_par, base, acc1;
};
__device__ inline AccUse acc_take(AccSched &st, int nacc, bool narrow, uint32_t accw, uint32_t acc1) {
  AccUse u;
  if (nacc == 2 || (st.dyn && narrow)) {
    const int s = st.next;
    st.next ^= 1;
    u.nh = 1; u.h0 = s;
    u.base = (uint32_t)s * (nacc == 2 ? accw : 256u);
    u.acc1 = (nacc == 2) ? acc1 : 64u;
  } else {
    u.nh = st.dyn ? 2 : 1; u.h0 = 0;
    u.base = 0; u.acc1 = acc1;
  }
  const uint32_t a0 = u.h0 ? st.acq1 : st.acq0;
  u.wait0 = a0 > 0;
  u.par0 = (a0 - 1) & 1;
  if (u.h0) st.acq1++;
  else st.acq0++;
  u.wait1 = 0;
  u.par1 = 0;
  if (u.nh == 2) {   // a wide tile also takes half 1
    u.wait1 = st.acq1 > 0;
    u.par1 = (st.acq1 - 1) & 1;
    st.acq1++;
  }
  u.sfull = u.h0;
  const uint32_t f = u.h0 ? st.full1 : st.full0;
  u.full_par = f & 1;
  if (u.h0) st.full1++;
  else st.full0++;
  return u;
}

// a tensor map written to device memory by the host: order that write
// before the tensor-map proxy reads it
__device__ inline void tensormap_acquire(const CUtensorMap *tm) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tm) : "memory");
}

// MULTI: the tiles of the shells in `tab` (nsh of them, ntiles in all) in
// one launch, every shell with the same accumulator split; otherwise the
// tiles of `one`.  Shared memory holds B tiles of nfb_max rows (the largest
// shell) and, for one shell, its nth_w Gauss weights (an ensemble launch
// reads the weights of each tile's shell through the cache instead).
template <bool MULTI>
__global__ void __launch_bounds__(FW_THREADS, 1)
k_leg_fwd_ws(const __grid_constant__ FwdShell one, const FwdShell *__restrict__ tab, int nsh, int ntiles,
             int nfb_max, int nth_w, uint32_t tmem_cols, int nacc) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = smem_base_1024(smem_raw);
  const FwdWsLayout lay = fwd_ws_layout(nfb_max, one.a.L, nth_w);
  FwdWsBars *sb = reinterpret_cast<FwdWsBars *>(base + lay.bar);
  float *w = reinterpret_cast<float *>(base + lay.w);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t B_BYTES = (uint32_t)nfb_max * FKB * 2;    // one of hi / lo, one parity
  const uint32_t AB_BYTES = 4 * FA_BYTES + 4 * B_BYTES;    // A hi/lo x 2 parities, B hi/lo x 2 parities
  unsigned char *raw0 = base + lay.raw, *ab0 = base + lay.ab;
  const uint32_t accw = tmem_cols / (uint32_t)nacc;       // columns of one accumulator set
  // a set holds the accumulator of each parity (hi*hi' + cross terms), or
  // with split the hi*hi' accumulators at 0 and acc1 and the cross-term
  // accumulators at 2 acc1 and 3 acc1
  const int split = one.a.split;
  const uint32_t acc1 = split ? accw / 4 : accw / 2;
  // one set of four 128-column accumulators over all of tensor memory: tiles
  // whose accumulators fit in 64 columns take alternate halves (AccSched)
  const int dyn = (nacc == 1 && split && tmem_cols >= 512 && acc1 >= 128) ? 1 : 0;
  const unsigned long long wait_ns = one.a.wait_ns;
  auto shell = [&](int t) -> const FwdShell & { return MULTI ? shell_of(tab, nsh, t) : one; };

  if (tid == 0) {
    // consumer barriers count warps: one elected lane arrives for its warp
    for (int q = 0; q < FRS; q++) { mbar_init(&sb->rawfull[q], 1); mbar_init(&sb->rawempty[q], FW_CONV / 32); }
    for (int q = 0; q < FAB; q++) {
      mbar_init(&sb->afull[q], FW_CONV / 32); mbar_init(&sb->bfull[q], 1); mbar_init(&sb->abempty[q], 1);
    }
    for (int q = 0; q < 2; q++) { mbar_init(&sb->accfull[q], 1); mbar_init(&sb->accempty[q], FW_EPI / 32); }
    mbar_init(&sb->fin, 1);
    sb->abort = 0;
    // an earlier launch on any of the shells timed out: this one does nothing
    int st = *(volatile int *)one.a.status;
    if (MULTI)
      for (int s = 0; s < nsh; s++) st |= *(volatile int *)tab[s].a.status;
    sb->skip = (st & CB2_STATUS_PIPE_TIMEOUT) != 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int q = tid; q < nth_w; q += FW_THREADS) w[q] = one.a.wgt[q];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sb->tmem_base)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sb->tmem_base;
  const bool skip = sb->skip != 0;

  if (skip) {
    // an earlier launch timed out: do nothing
  } else if (warp == FW_PROD_WARP) {
    if (lane == 0) {
      uint32_t nraw = 0, nab = 0;
      bool bad = false;
      const FwdShell *last = nullptr;
      for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x) {
        if (ws_aborted(sb)) { bad = true; break; }
        const FwdShell &sh = shell(t);
        const FwdArgs &a = sh.a;
        const FwdTile q = fwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
        const CUtensorMap *traw = q.g ? &sh.rawD : &sh.rawP;
        const CUtensorMap *tbh = q.g ? &sh.dhi : &sh.phi, *tbl = q.g ? &sh.dlo : &sh.plo;
        if (MULTI && &sh != last) {   // the first tile of this CTA from this shell
          const CUtensorMap *maps[6] = {&sh.rawP, &sh.rawD, &sh.phi, &sh.plo, &sh.dhi, &sh.dlo};
          for (int u = 0; u < 6; u++) tensormap_acquire(maps[u]);
          last = &sh;
        }
        const uint32_t bbytes = 2u * (uint32_t)(q.nbox0 + q.nbox1) * a.boxr * FKB * 2;
        for (int b = 0; b < q.NB; b++) {
          const int tb = q.g ? (b >> 1) : b, part = q.g ? (b & 1) : 0;
          if (part == 0) {
            const uint32_t rs = nraw % FRS;
            if (nraw >= FRS && !mbar_wait(&sb->rawempty[rs], ((nraw / FRS) - 1) & 1, wait_ns)) { bad = true; break; }
            unsigned char *dst = raw0 + rs * RAW_BYTES;
            mbar_expect_tx(&sb->rawfull[rs], RAW_BYTES);
            const uint64_t pf = policy_evict_first();
            tma_load_2d_hint(dst, traw, &sb->rawfull[rs], q.row0, q.m * a.nth + tb * FKB, pf);
            tma_load_2d_hint(dst + RAW_BYTES / 2, traw, &sb->rawfull[rs], q.row0,
                             q.m * a.nth + a.nth - tb * FKB - FKB, pf);
            nraw++;
          }
          const uint32_t s = nab % FAB;
          if (nab >= FAB && !mbar_wait(&sb->abempty[s], ((nab / FAB) - 1) & 1, wait_ns)) { bad = true; break; }
          unsigned char *bb = ab0 + s * AB_BYTES + 4 * FA_BYTES;
          mbar_expect_tx(&sb->bfull[s], bbytes);
          const int x = part * a.nhp + tb * FKB;
          const uint64_t pl = policy_evict_last();
          for (int p = 0; p < 2; p++) {
            unsigned char *bh = bb + (2 * p) * B_BYTES, *bl = bh + B_BYTES;
            const int nbx = p ? q.nbox1 : q.nbox0, br = p ? q.brow1 : q.brow0;
            for (int j = 0; j < nbx; j++) {
              tma_load_2d_hint(bh + j * a.boxr * FKB * 2, tbh, &sb->bfull[s], x, br + j * a.boxr, pl);
              tma_load_2d_hint(bl + j * a.boxr * FKB * 2, tbl, &sb->bfull[s], x, br + j * a.boxr, pl);
            }
          }
          nab++;
        }
      }
      if (bad) {
        sb->abort = 1;
        // every copy still in flight lands before the CTA may exit
        for (uint32_t q = 0; q < FRS && q < nraw; q++) {
          const uint32_t last = ((nraw - 1 - q) / FRS) * FRS + q;   // last load issued to stage q
          mbar_wait(&sb->rawfull[q], (last / FRS) & 1);
        }
        for (uint32_t q = 0; q < FAB && q < nab; q++) {
          const uint32_t last = ((nab - 1 - q) / FAB) * FAB + q;
          mbar_wait(&sb->bfull[q], (last / FAB) & 1);
        }
      }
    }
  } else if (warp == FW_MMA_WARP) {
    if (lane == 0) {
      uint32_t nab = 0;
      bool bad = false, any = false;
      int i = 0;
      AccSched sched{dyn, 0, 0, 0, 0, 0};
      for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x, i++) {
        if (ws_aborted(sb)) { bad = true; break; }
        const FwdShell &sh = shell(t);
        const FwdTile q = fwd_tile(sh.a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
        const AccUse u = acc_take(sched, nacc, max(q.npad0, q.npad1) <= 64, accw, acc1);
        if (u.wait0 && !mbar_wait(&sb->accempty[u.h0], u.par0, wait_ns)) bad = true;
        if (!bad && u.wait1 && !mbar_wait(&sb->accempty[1], u.par1, wait_ns)) bad = true;
        if (bad) break;
        tc_fence_after();
        const uint32_t accb = tmem + u.base;
        for (int b = 0; b < q.NB; b++) {
          const uint32_t s = nab % FAB, ph = (nab / FAB) & 1;
          if (!mbar_wait(&sb->afull[s], ph, wait_ns) || !mbar_wait(&sb->bfull[s], ph, wait_ns)) { bad = true; break; }
          tc_fence_after();
          unsigned char *at = ab0 + s * AB_BYTES, *bb = at + 4 * FA_BYTES;
          for (int p = 0; p < 2; p++) {
            const int np = p ? q.np1 : q.np0, npad = p ? q.npad1 : q.npad0;
            if (np == 0) continue;
            const uint32_t idesc = idesc_f16_f32(TM, npad);
            const uint64_t dah = smem_desc_sw64(at + (2 * p) * FA_BYTES), dal = smem_desc_sw64(at + (2 * p + 1) * FA_BYTES);
            const uint64_t dbh = smem_desc_sw64(bb + (2 * p) * B_BYTES), dbl = smem_desc_sw64(bb + (2 * p + 1) * B_BYTES);
            const uint32_t acc = accb + (p ? u.acc1 : 0u);
            // split: hi*hi' (on the fixed grid, summed exactly) in its own
            // accumulator, the cross terms and lo*lo' (2^-11 and 2^-22 of
            // it) in the second
            const uint32_t accx = split ? acc + 2 * u.acc1 : acc;
#pragma unroll
            for (int ks = 0; ks < FKB / 16; ks++) {
              const uint64_t o = (uint64_t)(ks * 2);
              const uint32_t first = (b == 0 && ks == 0) ? 0u : 1u;
              mma_f16(acc, dah + o, dbh + o, idesc, first);
              mma_f16(accx, dah + o, dbl + o, idesc, split ? first : 1u);
              mma_f16(accx, dal + o, dbh + o, idesc, 1u);
              if (split) mma_f16(accx, dal + o, dbl + o, idesc, 1u);
            }
          }
          mma_commit(&sb->abempty[s]);
          any = true;
          nab++;
        }
        if (bad) break;
        mma_commit(&sb->accfull[u.sfull]);
      }
      // no MMA may still run when the CTA releases its tensor memory
      if (any) {
        mma_commit(&sb->fin);
        if (!mbar_wait(&sb->fin, 0)) bad = true;
      }
      if (bad) sb->abort = 1;
    }
  } else if (warp < FW_CONV / 32) {
    const int r = tid & (TM - 1), h = tid >> 7;
    uint32_t nraw = 0, nab = 0;
    bool bad = false;
    // every decision is warp-uniform: a warp arrives through one lane
    for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x) {
      if (__any_sync(0xffffffffu, ws_aborted(sb))) { bad = true; break; }
      const FwdShell &sh = shell(t);
      const FwdArgs &a = sh.a;
      const FwdTile q = fwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
      const int row = q.row0 + r, q4 = row & 3;
      const float sc = fwd_row_scale(a, q, row);
      // Gauss weight of node i: staged in shared memory for one shell
      auto wt = [&](int i) { return MULTI ? __ldg(a.wgt + i) : w[i]; };
      for (int b = 0; b < q.NB; b++) {
        const int tb = q.g ? (b >> 1) : b, part = q.g ? (b & 1) : 0;
        const uint32_t rs = nraw % FRS, s = nab % FAB;
        bool ok = true;
        if (part == 0) ok = mbar_wait(&sb->rawfull[rs], (nraw / FRS) & 1, wait_ns);
        if (ok && nab >= FAB) ok = mbar_wait(&sb->abempty[s], ((nab / FAB) - 1) & 1, wait_ns);
        if (!__all_sync(0xffffffffu, ok)) { bad = true; break; }
        // the two folds of this row's 16 K values; gemm P and the mP part
        // use fold p, the dP part fold 1 - p (with the signs of its rows)
        const float *rs_s = reinterpret_cast<const float *>(raw0 + rs * RAW_BYTES);
        const float *rs_n = rs_s + FKB * TM;
        int src = r;
        float sg = sc;
        bool swap = false;   // true: accumulator 0 takes the anti fold
        if (q.g) {
          if (part == 0) { sg = (q4 < 2) ? sc : -sc; swap = true; }
          else { src = r - q4 + 3 - q4; sg = (q4 & 1) ? sc : -sc; }
        }
        float x2[2][16];
#pragma unroll
        for (int e = 0; e < 16; e++) {
          const int kk = h * 16 + e, i = tb * FKB + kk;
          float vs = 0.0f, va = 0.0f;
          if (i < a.nh) {
            const float fa = rs_s[kk * TM + src] * wt(i);
            const float fb = rs_n[(FKB - 1 - kk) * TM + src] * wt(a.nth - 1 - i);
            vs = (fa + fb) * sg;
            va = (fa - fb) * sg;
          }
          x2[0][e] = swap ? va : vs;
          x2[1][e] = swap ? vs : va;
        }
        unsigned char *at = ab0 + s * AB_BYTES;
#pragma unroll
        for (int p = 0; p < 2; p++) {
          unsigned char *ahi = at + (2 * p) * FA_BYTES, *alo = ahi + FA_BYTES;
#pragma unroll
          for (int c = 0; c < 2; c++) {
            uint32_t hh[4], ll[4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
              if (split) split_pair_q(x2[p][c * 8 + e], x2[p][c * 8 + e + 1], hh[e >> 1], ll[e >> 1]);
              else split_pair(x2[p][c * 8 + e], x2[p][c * 8 + e + 1], hh[e >> 1], ll[e >> 1]);
            }
            const uint32_t off = sw64_chunk(r, 2 * h + c);
            *reinterpret_cast<uint4 *>(ahi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
            *reinterpret_cast<uint4 *>(alo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
          }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sb->afull[s]);
        nab++;
        if (!q.g || part == 1) {
          if (lane == 0) mbar_arrive(&sb->rawempty[rs]);
          nraw++;
        }
      }
    }
    if (bad) sb->abort = 1;
  } else {
    // epilogue warps 8-15: warp 8 + h * 4 + q reads TMEM lanes 32 q + 16 h ..
    // + 15 with 16x256b loads: thread (t0 = lane & 3, t1 = lane >> 2) gets
    // columns 2 t0, 2 t0 + 1 of rows t1, t1 + 8, and the two parity
    // accumulators interleave to the degrees 16 g + 4 t0 .. + 3 of a row.
    // Through the warp's shared staging [16 rows][16 degrees], a store then
    // writes 16 consecutive degrees of two rows (lanes 0-15, 16-31).
    // Decisions that guard the warp-collective TMEM loads are warp-uniform.
    const int ew = warp - FW_CONV / 32, qd = ew & 3, hf = ew >> 2;
    const int t0 = lane & 3, t1 = lane >> 2, lc = lane & 15, lr = lane >> 4;
    unsigned char *wst = base + lay.stg + ew * FW_STG_BYTES;
    double *stg = reinterpret_cast<double *>(wst);                                 // [16][FW_STG_P]
    long long *moff = reinterpret_cast<long long *>(wst + 16 * FW_STG_P * 8);     // [16]
    double *mc = reinterpret_cast<double *>(moff + 16);                           // [16]
    int *mg = reinterpret_cast<int *>(mc + 16);                                   // [16]
    int i = 0;
    AccSched sched{dyn, 0, 0, 0, 0, 0};
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
      if (__any_sync(0xffffffffu, ws_aborted(sb))) break;
      const FwdShell &sh = shell(t);
      const FwdArgs &a = sh.a;
      double *__restrict__ fout = a.f;
      const FwdTile q = fwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
      const int nl = a.L + 1 - q.m;
      // lanes 0-15: destination, scale and degree factor of row lane
      // (sel 0: g7, 1: g6; both depend on l and m only, not on s)
      __syncwarp();
      if (lane < 16) {
        const int rw = q.row0 + qd * 32 + hf * 16 + lane;
        long long off = -1;
        double cr = 0.0;
        int sel = 0;
        if (rw < q.nrows) {
          int k, slot, kind, s;   // kind 0: S (g7 r^2), 1: dS or T (g7 r), 2: scalar (g6)
          if (q.g == 0) {
            const int ng = a.nvec + a.nscal, v = (rw >> 1) % ng;
            s = rw & 1; k = (rw >> 1) / ng;
            slot = a.slot[v]; kind = (v < a.nvec) ? 0 : 2;
          } else {
            const int v = (rw >> 2) % a.nvec;
            k = (rw >> 2) / a.nvec; s = rw & 1;
            slot = a.slot[v] + 1 + ((rw & 3) >> 1); kind = 1;
          }
          if (!(q.m == 0 && s == 1)) {
            const double ua = 1.0 / (double)fwd_row_scale(a, q, rw), rk = a.r[k];
            cr = (kind == 0) ? ua * rk * rk : (kind == 1) ? ua * rk : ua;
            off = (long long)slot * (long long)a.fs + (long long)k * a.jmax + a.moff[q.m] + s * nl;
            sel = (kind == 2) ? 1 : 0;
          }
        }
        moff[lane] = off; mc[lane] = cr; mg[lane] = sel;
      }
      const AccUse u = acc_take(sched, nacc, max(q.npad0, q.npad1) <= 64, accw, acc1);
      const uint32_t acc1 = u.acc1;
      const bool ok = mbar_wait(&sb->accfull[u.sfull], u.full_par, wait_ns);
      if (!__all_sync(0xffffffffu, ok)) { sb->abort = 1; break; }
      tc_fence_after();
      const uint32_t tl = tmem + u.base + ((uint32_t)(qd * 32 + hf * 16) << 16);
      const int ng = (nl + 15) / 16, j0 = a.moff[q.m];
      const float *bun0 = a.bunscale + ((size_t)q.g * (a.L + 1) * 2 + q.m * 2) * a.NFmax, *bun1 = bun0 + a.NFmax;
      // degree factors of degree 16 g + lc (this lane's column), a group ahead
      auto fetch = [&](int g, double &g7v, double &g6v, float &buv) {
        const int lm = g * 16 + lc;
        g7v = 0.0; g6v = 0.0; buv = 0.0f;
        if (g < ng && lm < nl) {
          g7v = __ldg(a.g7 + j0 + lm);
          g6v = __ldg(a.g6 + j0 + lm);
          buv = (lm & 1) ? __ldg(bun1 + (lm >> 1)) : __ldg(bun0 + (lm >> 1));
        }
      };
      double n7, n6;
      float nbu;
      fetch(0, n7, n6, nbu);
      for (int g = 0; g < ng; g++) {
        float f0[4], f1[4];
        double p0[4], p1[4];
        if (split) {
          // hi*hi' and cross-term accumulators of both parities, one wait;
          // the two accumulators are added in float64: no rounding of the sum
          float x0[4], x1[4];
          const uint32_t o = (uint32_t)(g * 8);
          tmem_ld_16x256b_quad(tl + o, tl + acc1 + o, tl + 2 * acc1 + o, tl + 3 * acc1 + o, f0, f1, x0, x1);
#pragma unroll
          for (int j = 0; j < 4; j++) {
            p0[j] = (double)f0[j] + (double)x0[j];
            p1[j] = (double)f1[j] + (double)x1[j];
          }
        } else {
          tmem_ld_16x256b_pair(tl + (uint32_t)(g * 8), tl + acc1 + (uint32_t)(g * 8), f0, f1);
#pragma unroll
          for (int j = 0; j < 4; j++) { p0[j] = (double)f0[j]; p1[j] = (double)f1[j]; }
        }
        if (g == ng - 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) {
            mbar_arrive(&sb->accempty[u.h0]);
            if (u.nh == 2) mbar_arrive(&sb->accempty[1]);
          }
        }
        const double c7 = n7 * (double)nbu, c6 = n6 * (double)nbu;
        fetch(g + 1, n7, n6, nbu);
#pragma unroll
        for (int j = 0; j < 2; j++) {
          double *srow = stg + (t1 + 8 * j) * FW_STG_P + 4 * t0;
          srow[0] = p0[2 * j]; srow[1] = p1[2 * j]; srow[2] = p0[2 * j + 1]; srow[3] = p1[2 * j + 1];
        }
        __syncwarp();
        const int lm = g * 16 + lc;
        if (lm < nl) {
#pragma unroll 4
          for (int u = 0; u < 8; u++) {
            const int rr = u + 8 * lr;
            const long long o = moff[rr];
            if (o >= 0) fout[o + lm] = stg[rr * FW_STG_P + lc] * mc[rr] * (mg[rr] ? c6 : c7);
          }
        }
        __syncwarp();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && sb->abort) {
    // a multi-shell launch voids the state of every shell in it
    atomicOr(one.a.status, CB2_STATUS_PIPE_TIMEOUT);
    if (MULTI)
      for (int s = 0; s < nsh; s++) atomicOr(tab[s].a.status, CB2_STATUS_PIPE_TIMEOUT);
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ---------------------------------------------------------------------------
// backward: spectra f[slot][k][jj] -> order-major Fourier rows
//
// Step 1, k_pack_bwd (the reference's rj -> rlm transpose, on the device):
// the spectra of one order m are rewritten as float32 rows, one row per GEMM
// row and one contiguous run of rows per (m, parity of l-m, K index):
//   P block  rlmP[Kbase(m, par) + kk][(k, field, s)]  = S l(l+1)/r^2 (vector)
//                                                        or the scalar,
//   D block  rlmD[Kbase(m, par) + kk][(k, vector, q')] = X/r, q' = 2 c + s,
//            c = 0 dS/dr, 1 T,
// at l = m + par + 2 kk, with the row maxima over all l (for the scales).
// Step 2, k_leg_bwd_ws: a tile = (m, gemm, 128 rows).  For each K
// block TMA brings the raw rows [32 K][128 rows] and the B tile
// [nhp theta][32 K]; converter threads scale, sign and split into fp16 hi/lo
// (64-byte swizzled); two TMEM accumulators (parity of the basis function)
// give the south (acc0 + acc1) and north (acc0 - acc1) nodes.  gemm DM,
// accumulator p: dP part from D rows q at parity 1-p with sign {+,+,-,-},
// then mP part from rows 3-q at parity p with sign {+,-,+,-}.
struct PackArgs {
  int L, nr, jmax, nvec, ng, kc;
  int slot[8];
  const int *moff;
  const double *g3rlm, *ar1, *f;
  size_t fs;
  float *rlmP, *rlmD;
  int pitchP, pitchD;      // row pitch (floats) of the two blocks
  const int *kbase;        // [(L+1) * 2] first K row of (m, parity)
  float *maxP, *maxD;      // [m][pitch] row maxima
};

__global__ void __launch_bounds__(256)
k_pack_bwd(const __grid_constant__ PackArgs a) {
  extern __shared__ float T[];   // [kc * RK][NLP]
  const int m = blockIdx.x, k0 = blockIdx.y * a.kc, nk = min(a.kc, a.nr - k0);
  const int nl = a.L + 1 - m, NLP = nl | 1;
  const int RP = 2 * a.ng, RD = 4 * a.nvec, RK = RP + RD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int jm = a.moff[m];
  // rows in: one warp per (radial level, row), lanes along l (coalesced
  // float64 reads, 256 degrees per pass with all loads in flight together),
  // the row maximum on the way
  for (int rl = warp; rl < nk * RK; rl += nw) {
    const int kq = rl / RK, j = rl - kq * RK, k = k0 + kq;
    const double *src;
    double rowf;
    bool vec;
    int s;
    if (j < RP) {
      const int fl = j >> 1;
      s = j & 1;
      src = a.f + (size_t)a.slot[fl] * a.fs + (size_t)k * a.jmax + jm + s * nl;
      vec = fl < a.nvec;
      const double ar = a.ar1[k];
      rowf = vec ? ar * ar : 1.0;
    } else {
      const int jd = j - RP, vv = jd >> 2, comp = (jd & 3) >> 1;
      s = jd & 1;
      src = a.f + (size_t)(a.slot[vv] + 1 + comp) * a.fs + (size_t)k * a.jmax + jm + s * nl;
      vec = false;
      rowf = a.ar1[k];
    }
    const bool zero = (m == 0 && s == 1);
    const double *g3 = a.g3rlm + jm + s * nl;
    float mx = 0.0f;
    for (int l0 = 0; l0 < nl; l0 += 256) {
      double x[8], gg[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int lm = l0 + u * 32 + lane;
        const bool ok = !zero && lm < nl;
        x[u] = ok ? __ldg(src + lm) : 0.0;
        gg[u] = (ok && vec) ? __ldg(g3 + lm) : 1.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int lm = l0 + u * 32 + lane;
        if (lm < nl) {
          const float v = (float)(vec ? x[u] * (rowf * gg[u]) : x[u] * rowf);
          T[rl * NLP + lm] = v;
          mx = fmaxf(mx, fabsf(v));
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      if (j < RP) a.maxP[(size_t)m * a.pitchP + k * RP + j] = mx;
      else a.maxD[(size_t)m * a.pitchD + k * RD + (j - RP)] = mx;
    }
  }
  __syncthreads();
  // rows out: per (parity, kk) one contiguous run of nk RP (P block) and
  // nk RD (D block) values; a lane keeps its (level, row) for every kk
  const int wP = nk * RP, wD = nk * RD;
  for (int par = 0; par < 2; par++) {
    const int cnt = par ? nl / 2 : (nl + 1) / 2;
    const size_t base = a.kbase[m * 2 + par];
    for (int rr = lane; rr < wP; rr += 32) {
      const int kq = rr / RP, j = rr - kq * RP;
      const float *tr = T + (kq * RK + j) * NLP + par;
      float *dst = a.rlmP + base * a.pitchP + (size_t)k0 * RP + rr;
      for (int kk = warp; kk < cnt; kk += nw) dst[(size_t)kk * a.pitchP] = tr[2 * kk];
    }
    for (int rr = lane; rr < wD; rr += 32) {
      const int kq = rr / RD, j = rr - kq * RD;
      const float *tr = T + (kq * RK + RP + j) * NLP + par;
      float *dst = a.rlmD + base * a.pitchD + (size_t)k0 * RD + rr;
      for (int kk = warp; kk < cnt; kk += nw) dst[(size_t)kk * a.pitchD] = tr[2 * kk];
    }
  }
}

struct BwdArgs {
  int L, nr, nh, nhp, nth, nvec, nscal;
  int pitchP, pitchD;
  const int *kbase;        // as in PackArgs
  const int *ko;           // [(m * 4 + group) * 2 + part] B column offset (multiples of 32)
  const float *maxP, *maxD;
  const float *bunscale;   // [gemm][m][nhp] 1 / column scale of B
  MLayout out;
  int *status;
  unsigned long long wait_ns;   // budget of each pipeline wait (Ctx::pipe_wait_ns)
};

constexpr uint32_t BRAW_BYTES = FKB * TM * 4;   // raw rows of one K block

// One shell of a backward launch: its tensor maps, arguments and tile
// counts.  A single-shell launch takes it as a kernel parameter; an
// ensemble launch reads a table of them from device memory, shell s owning
// the tiles tile0(s) .. tile0(s + 1) - 1 of the launch.
struct BwdShell {
  CUtensorMap rawP, rawD, bhi, blo;   // 64-byte aligned
  BwdArgs a;
  int rows_g0, rows_g1, tiles_g0, tiles_g1, tile0;
};

// ---------------------------------------------------------------------------
// backward, warp-specialised and persistent: the roles of the forward kernel
// (converters, epilogue warps, TMA producer, MMA issuer), one CTA per SM over
// the tiles (m, gemm, 128 rows) in order-major order.  A stage holds one K
// block: the raw rows [32 K][128 rows], the A tiles (hi, lo) and the B
// tiles (hi, lo) [nhp theta][32 K].  The parity-p accumulator of a set sits
// at TMEM column p nhp; two sets (epilogue of one tile overlapping the main
// loop of the next) when 4 nhp columns fit, else one.
constexpr int BW_ST = 3;
// roles: converters warps 0-7, epilogue warps 8-15 (two per TMEM lane
// quarter, one per half of the colatitude columns), producer 16, MMA 17
constexpr int BW_CONV = 256, BW_EPI = 256, BW_THREADS = 576;
constexpr int BW_PROD_WARP = 16, BW_MMA_WARP = 17;

struct BwdWsBars {
  uint64_t full[BW_ST], afull[BW_ST], empty[BW_ST];
  uint64_t accfull[2], accempty[2], fin;
  uint32_t tmem_base;
  int abort, skip;
};

struct BwdTile {
  int m, g, row0, nrows;
  int len00, len01, len10, len11, blk00, blk10, nkb0, nkb1, nmin, total, pmore;
};

// K parts per accumulator p: gemm P one part (parity p); gemm DM the dP part
// (parity 1-p) then the mP part (parity p)
__device__ inline BwdTile bwd_tile(const BwdArgs &a, int t, int rows_g0, int rows_g1, int tiles_g0, int tiles_g1) {
  BwdTile q;
  const int tpm = tiles_g0 + tiles_g1;
  q.m = t / tpm;
  const int x = t - q.m * tpm;
  q.g = (x >= tiles_g0) ? 1 : 0;
  q.row0 = (q.g ? x - tiles_g0 : x) * TM;
  q.nrows = q.g ? rows_g1 : rows_g0;
  const int nl = a.L + 1 - q.m, cnt0 = (nl + 1) / 2, cnt1 = nl / 2;
  q.len00 = q.g ? cnt1 : cnt0;
  q.len01 = q.g ? cnt0 : 0;
  q.len10 = q.g ? cnt0 : cnt1;
  q.len11 = q.g ? cnt1 : 0;
  q.blk00 = (q.len00 + FKB - 1) / FKB;
  q.blk10 = (q.len10 + FKB - 1) / FKB;
  q.nkb0 = q.blk00 + (q.len01 + FKB - 1) / FKB;
  q.nkb1 = q.blk10 + (q.len11 + FKB - 1) / FKB;
  q.nmin = min(q.nkb0, q.nkb1);
  q.total = q.nkb0 + q.nkb1;
  q.pmore = (q.nkb0 >= q.nkb1) ? 0 : 1;
  return q;
}

// block b of a tile -> accumulator p, part, block index within the part and
// the valid K rows of that part (the two accumulators alternate)
__device__ inline void bwd_blk(const BwdTile &q, int b, int &p, int &part, int &ib, int &len) {
  int i;
  if (b < 2 * q.nmin) { p = b & 1; i = b >> 1; } else { p = q.pmore; i = q.nmin + (b - 2 * q.nmin); }
  const int b0 = p ? q.blk10 : q.blk00;
  part = (i < b0) ? 0 : 1;
  ib = part ? i - b0 : i;
  len = p ? (part ? q.len11 : q.len10) : (part ? q.len01 : q.len00);
}

// largest |value| of tile row `row` (gemm DM: over the row and its partner)
__device__ inline float bwd_row_max(const BwdArgs &a, const BwdTile &q, int row) {
  if (row >= q.nrows) return 0.0f;
  const int q4 = row & 3;
  if (q.g == 0) return a.maxP[(size_t)q.m * a.pitchP + row];
  return fmaxf(a.maxD[(size_t)q.m * a.pitchD + row], a.maxD[(size_t)q.m * a.pitchD + row - q4 + 3 - q4]);
}

// MULTI: the tiles of the shells in `tab` (nsh of them, ntiles in all) in
// one launch; otherwise the tiles of `one`.  Shared memory and tensor memory
// are laid out for nhp_max colatitudes (the largest shell); the parity-1
// accumulator of a tile sits at its own shell's nhp.
template <bool MULTI>
__global__ void __launch_bounds__(BW_THREADS, 1)
k_leg_bwd_ws(const __grid_constant__ BwdShell one, const BwdShell *__restrict__ tab, int nsh, int ntiles,
             int nhp_max, uint32_t tmem_cols, int nacc) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = smem_base_1024(smem_raw);
  const uint32_t B_BYTES = (uint32_t)nhp_max * FKB * 2;     // one of hi / lo
  const uint32_t ST_BYTES = BRAW_BYTES + 2 * FA_BYTES + 2 * B_BYTES;
  BwdWsBars *sb = reinterpret_cast<BwdWsBars *>(base + BW_ST * ST_BYTES);
  float *buntab = reinterpret_cast<float *>(base + BW_ST * ST_BYTES + 256);   // [8 epilogue warps][nhp_max]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t accw = tmem_cols / (uint32_t)nacc;         // columns of one accumulator set
  auto shell = [&](int t) -> const BwdShell & { return MULTI ? shell_of(tab, nsh, t) : one; };

  if (tid == 0) {
    for (int q = 0; q < BW_ST; q++) {
      // consumer barriers count warps: one elected lane arrives for its warp
      mbar_init(&sb->full[q], 1); mbar_init(&sb->afull[q], BW_CONV / 32); mbar_init(&sb->empty[q], 1);
    }
    for (int q = 0; q < 2; q++) { mbar_init(&sb->accfull[q], 1); mbar_init(&sb->accempty[q], BW_EPI / 32); }
    mbar_init(&sb->fin, 1);
    sb->abort = 0;
    // an earlier launch on any of the shells timed out: this one does nothing
    int st = *(volatile int *)one.a.status;
    if (MULTI)
      for (int s = 0; s < nsh; s++) st |= *(volatile int *)tab[s].a.status;
    sb->skip = (st & CB2_STATUS_PIPE_TIMEOUT) != 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sb->tmem_base)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sb->tmem_base;
  const bool skip = sb->skip != 0;
  const unsigned long long wait_ns = one.a.wait_ns;

  if (skip) {
    // an earlier launch timed out: do nothing
  } else if (warp == BW_PROD_WARP) {
    if (lane == 0) {
      uint32_t n = 0;
      bool bad = false;
      const BwdShell *last = nullptr;
      for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x) {
        if (ws_aborted(sb)) { bad = true; break; }
        const BwdShell &sh = shell(t);
        const BwdArgs &a = sh.a;
        const BwdTile q = bwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
        const CUtensorMap *traw = q.g ? &sh.rawD : &sh.rawP;
        if (MULTI && &sh != last) {   // the first tile of this CTA from this shell
          tensormap_acquire(&sh.rawP); tensormap_acquire(&sh.rawD);
          tensormap_acquire(&sh.bhi); tensormap_acquire(&sh.blo);
          last = &sh;
        }
        for (int b = 0; b < q.total; b++) {
          int p, part, ib, len;
          bwd_blk(q, b, p, part, ib, len);
          const uint32_t s = n % BW_ST;
          if (n >= BW_ST && !mbar_wait(&sb->empty[s], ((n / BW_ST) - 1) & 1, wait_ns)) { bad = true; break; }
          unsigned char *st = base + s * ST_BYTES;
          // raw rows: parity of l-m of this part
          const int par = (q.g == 0) ? p : (part == 0 ? 1 - p : p);
          const int ky = a.kbase[q.m * 2 + par] + ib * FKB;
          const int bx = a.ko[(q.m * 4 + q.g * 2 + p) * 2 + part] + ib * FKB;
          // the B tile of this shell: nhp rows of 64 bytes
          const uint32_t bbytes = (uint32_t)a.nhp * FKB * 2;
          mbar_expect_tx(&sb->full[s], BRAW_BYTES + 2 * bbytes);
          const uint64_t pf = policy_evict_first(), pl = policy_evict_last();
          tma_load_2d_hint(st, traw, &sb->full[s], q.row0, ky, pf);
          tma_load_2d_hint(st + BRAW_BYTES + 2 * FA_BYTES, &sh.bhi, &sb->full[s], bx, 0, pl);
          tma_load_2d_hint(st + BRAW_BYTES + 2 * FA_BYTES + B_BYTES, &sh.blo, &sb->full[s], bx, 0, pl);
          n++;
        }
      }
      if (bad) {
        sb->abort = 1;
        // every copy still in flight lands before the CTA may exit
        for (uint32_t q = 0; q < BW_ST && q < n; q++) {
          const uint32_t last = ((n - 1 - q) / BW_ST) * BW_ST + q;   // last load issued to stage q
          mbar_wait(&sb->full[q], (last / BW_ST) & 1);
        }
      }
    }
  } else if (warp == BW_MMA_WARP) {
    if (lane == 0) {
      uint32_t n = 0;
      bool bad = false, any = false;
      int i = 0;
      for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x, i++) {
        if (ws_aborted(sb)) { bad = true; break; }
        const BwdShell &sh = shell(t);
        const BwdArgs &a = sh.a;
        const BwdTile q = bwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
        const uint32_t idesc = idesc_f16_f32(TM, a.nhp);
        const uint32_t acc1 = (uint32_t)a.nhp;                  // parity-1 accumulator within a set
        const int ab = i % nacc;
        if (i >= nacc && !mbar_wait(&sb->accempty[ab], ((i / nacc) - 1) & 1, wait_ns)) { bad = true; break; }
        tc_fence_after();
        const uint32_t accb = tmem + (uint32_t)ab * accw;
        for (int b = 0; b < q.total; b++) {
          int p, part, ib, len;
          bwd_blk(q, b, p, part, ib, len);
          const uint32_t s = n % BW_ST, ph = (n / BW_ST) & 1;
          if (!mbar_wait(&sb->afull[s], ph, wait_ns) || !mbar_wait(&sb->full[s], ph, wait_ns)) { bad = true; break; }
          tc_fence_after();
          unsigned char *ahi = base + s * ST_BYTES + BRAW_BYTES, *alo = ahi + FA_BYTES;
          unsigned char *bh = alo + FA_BYTES, *bl = bh + B_BYTES;
          const uint64_t dah = smem_desc_sw64(ahi), dal = smem_desc_sw64(alo);
          const uint64_t dbh = smem_desc_sw64(bh), dbl = smem_desc_sw64(bl);
          const uint32_t acc = accb + (p ? acc1 : 0u);
          const bool first = (ib == 0) && (part == 0 || (p ? q.blk10 : q.blk00) == 0);   // first block of p
#pragma unroll
          for (int ks = 0; ks < FKB / 16; ks++) {
            const uint64_t o = (uint64_t)(ks * 2);
            mma_f16(acc, dah + o, dbh + o, idesc, (first && ks == 0) ? 0u : 1u);
            mma_f16(acc, dah + o, dbl + o, idesc, 1u);
            mma_f16(acc, dal + o, dbh + o, idesc, 1u);
          }
          mma_commit(&sb->empty[s]);
          any = true;
          n++;
        }
        if (bad) break;
        mma_commit(&sb->accfull[ab]);
      }
      // no MMA may still run when the CTA releases its tensor memory
      if (any) {
        mma_commit(&sb->fin);
        if (!mbar_wait(&sb->fin, 0)) bad = true;
      }
      if (bad) sb->abort = 1;
    }
  } else if (warp < BW_CONV / 32) {
    // converters: thread (r, h) builds K values 16 h .. 16 h + 15 of row r
    const int r = tid & (TM - 1), h = tid >> 7;
    uint32_t n = 0;
    bool bad = false;
    int t = blockIdx.x;
    float mx_next = 0.0f;
    // the row maximum of tile t (row r)
    auto tile_max = [&](int tt) {
      const BwdShell &sn = shell(tt);
      const BwdTile qn = bwd_tile(sn.a, tt - sn.tile0, sn.rows_g0, sn.rows_g1, sn.tiles_g0, sn.tiles_g1);
      return bwd_row_max(sn.a, qn, qn.row0 + r);
    };
    if (t < ntiles) mx_next = tile_max(t);
    // every decision is warp-uniform: a warp arrives through one lane
    for (; t < ntiles && !bad; t += gridDim.x) {
      if (__any_sync(0xffffffffu, ws_aborted(sb))) { bad = true; break; }
      const BwdShell &sh = shell(t);
      const BwdTile q = bwd_tile(sh.a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
      const int row = q.row0 + r, q4 = row & 3;
      const float sc = pow2_scale(mx_next);
      // the next tile's row maximum is fetched now and used a tile later
      const int tn = t + gridDim.x;
      if (tn < ntiles) mx_next = tile_max(tn);
      for (int b = 0; b < q.total; b++) {
        int p, part, ib, len;
        bwd_blk(q, b, p, part, ib, len);
        const uint32_t s = n % BW_ST;
        if (!__all_sync(0xffffffffu, mbar_wait(&sb->full[s], (n / BW_ST) & 1, wait_ns))) { bad = true; break; }
        unsigned char *st = base + s * ST_BYTES;
        const float *raw = reinterpret_cast<const float *>(st);
        int src = r;
        float sg = sc;
        if (q.g) {
          if (part == 0) sg = (q4 < 2) ? sc : -sc;
          else { src = r - q4 + 3 - q4; sg = (q4 & 1) ? -sc : sc; }
        }
        const int kv = len - ib * FKB;   // valid K entries of this block
        float x[16];
#pragma unroll
        for (int e = 0; e < 16; e++) {
          const int kk = h * 16 + e;
          x[e] = (kk < kv) ? raw[kk * TM + src] * sg : 0.0f;
        }
        unsigned char *ahi = st + BRAW_BYTES, *alo = ahi + FA_BYTES;
#pragma unroll
        for (int c = 0; c < 2; c++) {
          uint32_t hh[4], ll[4];
#pragma unroll
          for (int e = 0; e < 8; e += 2) {
            split_pair(x[c * 8 + e], x[c * 8 + e + 1], hh[e >> 1], ll[e >> 1]);
          }
          const uint32_t off = sw64_chunk(r, 2 * h + c);
          *reinterpret_cast<uint4 *>(ahi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
          *reinterpret_cast<uint4 *>(alo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sb->afull[s]);
        n++;
      }
    }
    if (bad) sb->abort = 1;
  } else {
    // epilogue warps 8-15: TMEM lanes 32 (warp % 4) .. + 31, one row per
    // thread, warps 8-11 the first half of the 32-column chunks and 12-15
    // the rest; south (acc0 + acc1) and north (acc0 - acc1) colatitudes,
    // each store 32 consecutive rows.  Each warp keeps its own copy of the
    // tile's column unscale (no barrier between the epilogue warps).
    // Decisions that guard the warp-collective TMEM loads are warp-uniform.
    const int ew = warp - BW_CONV / 32, er = (ew & 3) * 32 + lane, hc = ew >> 2;
    float *bw = buntab + ew * nhp_max;
    int i = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
      if (__any_sync(0xffffffffu, ws_aborted(sb))) break;
      const BwdShell &sh = shell(t);
      const BwdArgs &a = sh.a;
      const BwdTile q = bwd_tile(a, t - sh.tile0, sh.rows_g0, sh.rows_g1, sh.tiles_g0, sh.tiles_g1);
      const uint32_t acc1 = (uint32_t)a.nhp;
      const int row = q.row0 + er;
      const bool valid = row < q.nrows;
      const float ua = 1.0f / pow2_scale(bwd_row_max(a, q, row));
      float *outb = q.g ? a.out.D : a.out.P;
      const size_t so = q.g ? a.out.sD() : a.out.sP();
      float *ob = outb + (size_t)q.m * a.nth * so + row;
      const float *bun = a.bunscale + ((size_t)q.g * (a.L + 1) + q.m) * a.nhp;
      __syncwarp();
      for (int u = lane; u < a.nhp; u += 32) bw[u] = __ldg(bun + u);
      __syncwarp();
      const bool has1 = q.nkb1 > 0;
      const int ab = i % nacc;
      const bool ok = mbar_wait(&sb->accfull[ab], (i / nacc) & 1, wait_ns);
      if (!__all_sync(0xffffffffu, ok)) { sb->abort = 1; break; }
      tc_fence_after();
      const uint32_t tl = tmem + (uint32_t)ab * accw + ((uint32_t)((ew & 3) * 32) << 16);
      const int nch = (a.nh + 31) / 32, ch = (nch + 1) / 2;
      const int c0 = hc ? ch : 0, c1 = hc ? nch : ch;
      if (c0 == c1) {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sb->accempty[ab]);
      }
      for (int c = c0; c < c1; c++) {
        float e[32], o[32];
        if (has1) {
          tmem_ld32x2(tl + (uint32_t)(c * 32), tl + acc1 + (uint32_t)(c * 32), e, o);
        } else {
          tmem_ld32x2(tl + (uint32_t)(c * 32), tl + (uint32_t)(c * 32), e, o);
#pragma unroll
          for (int u = 0; u < 32; u++) o[u] = 0.0f;
        }
        if (c == c1 - 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&sb->accempty[ab]);
        }
        if (valid) {
#pragma unroll
          for (int u = 0; u < 32; u++) {
            const int th = c * 32 + u;
            if (th < a.nh) {
              const float us = ua * bw[th];
              ob[(size_t)th * so] = (e[u] + o[u]) * us;
              ob[(size_t)(a.nth - 1 - th) * so] = (e[u] - o[u]) * us;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && sb->abort) {
    // a multi-shell launch voids the state of every shell in it
    atomicOr(one.a.status, CB2_STATUS_PIPE_TIMEOUT);
    if (MULTI)
      for (int s = 0; s < nsh; s++) atomicOr(tab[s].a.status, CB2_STATUS_PIPE_TIMEOUT);
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ---------------------------------------------------------------------------
// Row maxima for the operand scales, one streaming pass each.
//
// Fourier rows: Mf[m][e] = 2 max over theta of |F(m, theta, e) w(theta)|
// for every element e of the P block and then the D block; one thread per
// (m, e), consecutive threads on consecutive elements.
__global__ void __launch_bounds__(256)
k_rowmax_four(MLayout in, const float *wgt, float *Mf) {
  const int m = blockIdx.y;
  const size_t sP = in.sP(), sD = in.sD();
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= sP + sD) return;
  const float *x = (e < sP) ? in.P + (size_t)m * in.nth * sP + e : in.D + (size_t)m * in.nth * sD + (e - sP);
  const size_t st = (e < sP) ? sP : sD;
  // 16 colatitudes per pass, all their loads in flight together
  float mx = 0.0f;
  int th = 0;
  for (; th + 16 <= in.nth; th += 16) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) v[u] = __ldg(x + (size_t)(th + u) * st);
#pragma unroll
    for (int u = 0; u < 16; u++) mx = fmaxf(mx, fabsf(v[u]) * __ldg(wgt + th + u));
  }
  for (; th < in.nth; th++) mx = fmaxf(mx, fabsf(__ldg(x + (size_t)th * st)) * __ldg(wgt + th));
  Mf[(size_t)m * (sP + sD) + e] = 2.0f * mx;
}

// the same maxima from the four-step FFT kernel's partial maxima
// pm[theta][mb][e] (largest |x| w over the 16 orders of block mb at one
// colatitude): a row's scale then covers its block of 16 orders
__global__ void __launch_bounds__(256)
k_rowmax_reduce(const float *__restrict__ pm, int nth, int MB, size_t E, int L, float *__restrict__ Mf) {
  const int mb = blockIdx.y;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const float *x = pm + (size_t)mb * E + e;
  const size_t st = (size_t)MB * E;
  float mx = 0.0f;
  int th = 0;
  for (; th + 16 <= nth; th += 16) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) v[u] = __ldg(x + (size_t)(th + u) * st);
#pragma unroll
    for (int u = 0; u < 16; u++) mx = fmaxf(mx, v[u]);
  }
  for (; th < nth; th++) mx = fmaxf(mx, __ldg(x + (size_t)th * st));
  const int m1 = min(L + 1, mb * 16 + 16);
  for (int m = mb * 16; m < m1; m++) Mf[(size_t)m * E + e] = 2.0f * mx;
}

// ---------------------------------------------------------------------------
// B operands: scaled fp16 hi/lo copies of the float64 P tables
__device__ inline void split_store(__half *hi, __half *lo, size_t at, double v, float s) {
  const double x = v * (double)s;
  const __half h = __float2half_rn((float)x);
  hi[at] = h;
  lo[at] = __float2half_rn((float)(x - (double)__half2float(h)));
}
// hi on a fixed grid (a multiple of q = 16 or 8), as split_pair_q does
__device__ inline void split_store_q(__half *hi, __half *lo, size_t at, double v, float s, double q) {
  const double x = v * (double)s, h = rint(x / q) * q;
  hi[at] = __float2half_rn((float)h);
  lo[at] = __float2half_rn((float)(x - h));
}

// backward B[theta][K]: one thread per (m, south node i).  Column groups per
// m: P0, P1 (P_l^m, l - m even / odd), D0 = {dP of odd l-m | mP of even l-m},
// D1 = {dP of even | mP of odd}; each part starts at ko[(m * 4 + group) * 2 +
// part], a multiple of 32, so no K block of 32 mixes two parts.
__global__ void k_build_bwd_b(int L, int nh, int nhp, const size_t *poff, const double *Plt, const double *dPlt,
                              const double *asin_t, const int *ko, int Kc, float *bunscale, __half *bhi,
                              __half *blo) {
  const int m = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L || i >= nh) return;
  const int nl = L + 1 - m, cnt[2] = {(nl + 1) / 2, nl / 2};
  const size_t po = poff[m];
  const double am = (double)m * asin_t[i];
  double mxp = 0.0, mxd = 0.0;
  for (int t = 0; t < nl; t++) {
    const double P = Plt[po + (size_t)t * nh + i], dP = dPlt[po + (size_t)t * nh + i];
    mxp = fmax(mxp, fabs(P));
    mxd = fmax(mxd, fmax(fabs(dP), fabs(P * am)));
  }
  const float sp = pow2_scale(mxp), sd = pow2_scale(mxd);
  bunscale[(size_t)m * nhp + i] = 1.0f / sp;                     // gemm P
  bunscale[((size_t)(L + 1) + m) * nhp + i] = 1.0f / sd;         // gemm DM
  __half *hrow = bhi + (size_t)i * Kc, *lrow = blo + (size_t)i * Kc;
  for (int p = 0; p < 2; p++) {
    // P_p: P at l = m + p + 2 kk
    const int oP = ko[(m * 4 + p) * 2];
    for (int kk = 0; kk < cnt[p]; kk++)
      split_store(hrow, lrow, oP + kk, Plt[po + (size_t)(p + 2 * kk) * nh + i], sp);
    // D_p: dP at l = m + (1-p) + 2 kk, then P m / sin(theta) at l = m + p + 2 kk
    const int oA = ko[(m * 4 + 2 + p) * 2], oB = ko[(m * 4 + 2 + p) * 2 + 1];
    for (int kk = 0; kk < cnt[1 - p]; kk++)
      split_store(hrow, lrow, oA + kk, dPlt[po + (size_t)((1 - p) + 2 * kk) * nh + i], sd);
    for (int kk = 0; kk < cnt[p]; kk++)
      split_store(hrow, lrow, oB + kk, Plt[po + (size_t)(p + 2 * kk) * nh + i] * am, sd);
  }
}

// forward B[l][theta] (P) and B[l][dP theta | mP theta] (DM): one thread per (m, degree)
__global__ void k_build_fwd_b(int L, int nh, int nhp, int NFmax, const size_t *poff, const double *Plt,
                              const double *dPlt, const double *asin_t, const int *roff, const int *nlp,
                              float *bunscale, __half *php, __half *plp, __half *dhp, __half *dlp, int quant) {
  const int m = blockIdx.y, t = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L) return;
  // quantised: the theta/phi tables on the grid of 16, the A operand's, so
  // the products hi*hi' are multiples of 256 below 2^28 and sum exactly
  // below 2^32; the P tables on the grid of 8 (products multiples of 128,
  // exact below 2^31), which halves their representation error.  A fixed
  // grid bounds the error by the column maximum rather than by each value:
  // in a row dominated by one smooth component (a scalar's mean) the small
  // high-degree outputs carry that bound (measured: 6e-6 relative on the
  // seeded scalars of the L255 round trip, against 1e-6 with the floating
  // split, whose FP32 accumulation leaves the L255 step's toroidal magnetic
  // energy 5 % above the 1e-6 target).
  auto put = [&](__half *hi, __half *lo, size_t at, double v, float s, double q) {
    if (quant && q > 0.0) split_store_q(hi, lo, at, v, s, q);
    else split_store(hi, lo, at, v, s);
  };
  const size_t po = poff[m];
  for (int p = 0; p < 2; p++) {
    if (t >= nlp[m * 2 + p]) continue;
    const int l = m + p + 2 * t;
    const size_t row = (size_t)roff[m * 2 + p] + t;
    double mxp = 0.0, mxd = 0.0;
    for (int i = 0; i < nh; i++) {
      const double P = Plt[po + (size_t)(l - m) * nh + i], dP = dPlt[po + (size_t)(l - m) * nh + i];
      mxp = fmax(mxp, fabs(P));
      mxd = fmax(mxd, fmax(fabs(dP), fabs(P * (double)m * asin_t[i])));
    }
    const float sp = pow2_scale(mxp), sd = pow2_scale(mxd);
    bunscale[(size_t)(m * 2 + p) * NFmax + t] = 1.0f / sp;                        // gemm P
    bunscale[((size_t)(L + 1) * 2 + m * 2 + p) * NFmax + t] = 1.0f / sd;          // gemm DM
    for (int i = 0; i < nh; i++) {
      const double P = Plt[po + (size_t)(l - m) * nh + i];
      put(php, plp, row * nhp + i, P, sp, 8.0);
      put(dhp, dlp, row * 2 * nhp + i, dPlt[po + (size_t)(l - m) * nh + i], sd, 16.0);
      put(dhp, dlp, row * 2 * nhp + nhp + i, P * (double)m * asin_t[i], sd, 16.0);
    }
  }
}

// ---------------------------------------------------------------------------
// host side
struct MixedTables {
  __half *bb_hi = nullptr, *bb_lo = nullptr;      // backward B [nhp][Kb_all]
  float *bb_unscale = nullptr;                    // [gemm][m][nhp]
  int *bb_ko = nullptr;                           // [(m * 4 + group) * 2 + part]
  int *kbase = nullptr;                           // [(L+1) * 2] first rlm row of (m, parity)
  float *rlmP = nullptr, *rlmD = nullptr;         // [Ktot][pitch] order-major spectra
  float *maxP = nullptr, *maxD = nullptr;         // [(L+1)][pitch] their row maxima
  int Ktot = 0, pitch_max = 0;
  __half *bfp_hi = nullptr, *bfp_lo = nullptr;    // forward B (P) [rows_all][nhp]
  __half *bfd_hi = nullptr, *bfd_lo = nullptr;    // forward B (DM) [rows_all][2 nhp]
  float *bf_unscale = nullptr;                    // [gemm][(m, parity)][NFmax]
  int *bf_roff = nullptr, *bf_nl = nullptr;
  float *wgt32 = nullptr;                         // Gauss weights in float
  float *rowmax_four = nullptr;                   // [(L+1)][26 nr + 8]
  float *fwd_pmax = nullptr;                      // [nth][(L+1)/16][E], four-step FFT maxima
  int pmax_mb = 0;
  int Kb_all = 0, rows_all = 0, nhp = 0, NFmax = 0;
  size_t smem_bwd = 0, smem_fwd = 0, smem_pack = 0;
  CUtensorMap tm_bb_hi, tm_bb_lo, tm_bfp_hi, tm_bfp_lo, tm_bfd_hi, tm_bfd_lo;
  int boxr = 0, nfb = 0;
  uint32_t tmem_fwd = 0;
  int nacc_fwd = 1, nsm = 148, split_fwd = 0;
  uint32_t tmem_bwd = 0;
  int nacc_bwd = 1;
};

using EncodeFn = PFN_cuTensorMapEncodeTiled_v12000;

EncodeFn get_encode() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeFn)p;
  }
  return fn;
}

// 2-D map over [rows][cols] (cols contiguous, a row a multiple of 16 bytes),
// box = box_cols x box_rows (box_cols * element size <= the swizzle span)
int make_map_any(CUtensorMap *tm, CUtensorMapDataType dt, size_t es, const void *ptr, uint64_t cols, uint64_t rows,
                 uint32_t box_cols, uint32_t box_rows, CUtensorMapSwizzle sw) {
  EncodeFn enc = get_encode();
  if (!enc) { set_error("cuTensorMapEncodeTiled is not available"); return CB2_ERR_CUDA; }
  if ((cols * es) % 16 != 0 || (box_cols * es) % 16 != 0 || box_rows == 0 || box_rows > 256 || box_cols > 256 ||
      (reinterpret_cast<uintptr_t>(ptr) & 15) != 0) {
    set_error("tensor map shape");
    return CB2_ERR_ARG;
  }
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * es};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t ests[2] = {1, 1};
  CUresult r = enc(tm, dt, 2, const_cast<void *>(ptr), dims, strides, box, ests, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed"); return CB2_ERR_CUDA; }
  return 0;
}


// fp16 [rows][cols], box 32 x box_rows, 64-byte swizzle (forward B tiles)
int make_map64(CUtensorMap *tm, const void *ptr, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  return make_map_any(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, ptr, cols, rows, FKB, box_rows,
                      CU_TENSOR_MAP_SWIZZLE_64B);
}


}  // namespace

int mixed_setup(Ctx &c) {
  MixedTables *t = new MixedTables();
  c.mixed = t;
  const int L = c.L, nh = c.nh;
  t->nhp = ((nh + 15) / 16) * 16;
  if (t->nhp > 256) { set_error("mixed precision path needs nth <= 512"); return CB2_ERR_ARG; }
  // backward B column parts per m (each padded to 32): P0 {P, l-m even},
  // P1 {P, odd}, D0 {dP odd | mP even}, D1 {dP even | mP odd}; and the first
  // order-major spectral row of each (m, parity)
  std::vector<int> ko((L + 1) * 8, 0), kbase((L + 1) * 2);
  int K = 0, Kr = 0;
  for (int m = 0; m <= L; m++) {
    const int nl = L + 1 - m, cnt[2] = {(nl + 1) / 2, nl / 2};
    const int lens[4][2] = {{cnt[0], 0}, {cnt[1], 0}, {cnt[1], cnt[0]}, {cnt[0], cnt[1]}};
    for (int gi = 0; gi < 4; gi++)
      for (int part = 0; part < 2; part++) {
        ko[(m * 4 + gi) * 2 + part] = K;
        K += ((lens[gi][part] + FKB - 1) / FKB) * FKB;
      }
    kbase[m * 2] = Kr;
    kbase[m * 2 + 1] = Kr + cnt[0];
    Kr += nl;
  }
  t->Kb_all = K + FKB;
  t->Ktot = Kr;
  t->pitch_max = ((16 * c.nr + 3) / 4) * 4;   // up to 8 fields (P) or 4 vectors (D)
  // forward B rows: per (m, parity) the degrees l = m + p + 2t
  std::vector<int> roff((L + 1) * 2), nlp((L + 1) * 2);
  int R = 0, nfmax = 16;
  for (int m = 0; m <= L; m++) {
    const int nl = L + 1 - m, cnt[2] = {(nl + 1) / 2, nl / 2};
    for (int p = 0; p < 2; p++) {
      roff[m * 2 + p] = R;
      nlp[m * 2 + p] = cnt[p];
      const int padded = ((cnt[p] + 15) / 16) * 16;
      R += padded;
      nfmax = std::max(nfmax, padded);
    }
  }
  t->NFmax = nfmax;
  if (t->NFmax > 256) { set_error("mixed precision path needs L <= 511"); return CB2_ERR_ARG; }
  if (c.nth % 8 != 0) { set_error("mixed precision path needs nth divisible by 8"); return CB2_ERR_ARG; }
  t->boxr = std::min(64, t->NFmax);
  t->nfb = ((t->NFmax + t->boxr - 1) / t->boxr) * t->boxr;
  // one accumulator set = both parities, each as a hi*hi' and a cross-term
  // accumulator where they fit in TMEM (L <= 255); two sets when they fit.
  // Measured on the L255/Nr129 state (relative error of the forward
  // transform, theta/phi outputs / radial outputs): one accumulator 1.1e-6 /
  // 3e-7; separate cross-term accumulators 5.5e-7 / 6e-8 (the large one is
  // rounded after one MMA in three); with hi*hi' on the fixed grid, summed
  // exactly, 2.0e-7 / 4e-8.
  t->split_fwd = (4 * t->NFmax <= 512) ? 1 : 0;
  const int per_set = (t->split_fwd ? 4 : 2) * t->NFmax;
  t->nacc_fwd = (2 * per_set <= 512) ? 2 : 1;
  t->tmem_fwd = 32;
  while ((int)t->tmem_fwd < t->nacc_fwd * per_set) t->tmem_fwd *= 2;
  t->rows_all = R + t->NFmax;   // every NFmax-row box stays in the array
  auto up = [&](int **d, const std::vector<int> &v) -> int {
    CB2_CUDA(cudaMalloc(d, v.size() * sizeof(int)));
    CB2_CUDA(cudaMemcpy(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  };
  int rc;
  if ((rc = up(&t->bb_ko, ko)) || (rc = up(&t->kbase, kbase)) || (rc = up(&t->bf_roff, roff)) ||
      (rc = up(&t->bf_nl, nlp)))
    return rc;
  CB2_CUDA(cudaMalloc(&t->rlmP, (size_t)t->Ktot * t->pitch_max * sizeof(float)));
  CB2_CUDA(cudaMalloc(&t->rlmD, (size_t)t->Ktot * t->pitch_max * sizeof(float)));
  CB2_CUDA(cudaMalloc(&t->maxP, (size_t)(L + 1) * t->pitch_max * sizeof(float)));
  CB2_CUDA(cudaMalloc(&t->maxD, (size_t)(L + 1) * t->pitch_max * sizeof(float)));
  const size_t nb = (size_t)t->nhp * t->Kb_all;
  const size_t nfp = (size_t)t->rows_all * t->nhp, nfd = 2 * nfp;
  __half **bufs[6] = {&t->bb_hi, &t->bb_lo, &t->bfp_hi, &t->bfp_lo, &t->bfd_hi, &t->bfd_lo};
  const size_t lens[6] = {nb, nb, nfp, nfp, nfd, nfd};
  for (int q = 0; q < 6; q++) {
    CB2_CUDA(cudaMalloc(bufs[q], lens[q] * sizeof(__half)));
    CB2_CUDA(cudaMemsetAsync(*bufs[q], 0, lens[q] * sizeof(__half), c.stream));
  }
  const size_t nbs = 2 * (size_t)(L + 1) * t->nhp, nfs = 2 * (size_t)(L + 1) * 2 * t->NFmax;
  CB2_CUDA(cudaMalloc(&t->bb_unscale, nbs * sizeof(float)));
  CB2_CUDA(cudaMemsetAsync(t->bb_unscale, 0, nbs * sizeof(float), c.stream));
  CB2_CUDA(cudaMalloc(&t->bf_unscale, nfs * sizeof(float)));
  CB2_CUDA(cudaMemsetAsync(t->bf_unscale, 0, nfs * sizeof(float), c.stream));
  {
    std::vector<float> w(c.h_wgt.begin(), c.h_wgt.end());
    CB2_CUDA(cudaMalloc(&t->wgt32, w.size() * sizeof(float)));
    CB2_CUDA(cudaMemcpy(t->wgt32, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  CB2_CUDA(cudaMalloc(&t->rowmax_four, (size_t)(L + 1) * (26 * (size_t)c.nr + 8) * sizeof(float)));
  // the four-step FFT kernel (nph = 3 (L + 1), L + 1 a multiple of 16)
  // writes maxima over blocks of 16 orders, which replace k_rowmax_four
  if (c.nph == 3 * (L + 1) && (L + 1) % 16 == 0) {
    MLayout o;
    o.nvec = 4; o.nscal = 0; o.nr = c.nr; o.nth = c.nth;
    t->pmax_mb = (L + 1) / 16;
    CB2_CUDA(cudaMalloc(&t->fwd_pmax, (size_t)c.nth * t->pmax_mb * (o.sP() + o.sD()) * sizeof(float)));
  }
  k_build_bwd_b<<<dim3(cdiv(nh, 64), L + 1), 64, 0, c.stream>>>(L, nh, t->nhp, c.d_poff, c.d_Plt, c.d_dPlt,
                                                                c.d_asin, t->bb_ko, t->Kb_all, t->bb_unscale,
                                                                t->bb_hi, t->bb_lo);
  CB2_CUDA(cudaGetLastError());
  k_build_fwd_b<<<dim3(cdiv(t->NFmax, 64), L + 1), 64, 0, c.stream>>>(
      L, nh, t->nhp, t->NFmax, c.d_poff, c.d_Plt, c.d_dPlt, c.d_asin, t->bf_roff, t->bf_nl, t->bf_unscale,
      t->bfp_hi, t->bfp_lo, t->bfd_hi, t->bfd_lo, t->split_fwd);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  if ((rc = make_map64(&t->tm_bb_hi, t->bb_hi, t->Kb_all, t->nhp, t->nhp)) ||
      (rc = make_map64(&t->tm_bb_lo, t->bb_lo, t->Kb_all, t->nhp, t->nhp)) ||
      (rc = make_map64(&t->tm_bfp_hi, t->bfp_hi, t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfp_lo, t->bfp_lo, t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfd_hi, t->bfd_hi, 2 * t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfd_lo, t->bfd_lo, 2 * t->nhp, t->rows_all, t->boxr)))
    return rc;
  static_assert(sizeof(BwdWsBars) <= 256, "backward barrier block");
  t->smem_bwd = 1024 + BW_ST * ((size_t)BRAW_BYTES + 2 * (size_t)FA_BYTES + 2 * (size_t)t->nhp * FKB * 2) + 256 +
                (BW_EPI / 32) * (size_t)t->nhp * sizeof(float);
  // backward accumulator set = both parities (parity 1 at column nhp; the
  // epilogue reads 32-column chunks); two sets when they fit
  const int setw = t->nhp + ((t->nhp + 31) / 32) * 32;
  t->nacc_bwd = (2 * setw <= 512) ? 2 : 1;
  t->tmem_bwd = 32;
  while ((int)t->tmem_bwd < t->nacc_bwd * setw) t->tmem_bwd *= 2;
  t->smem_pack = (size_t)4 * 26 * ((L + 1) | 1) * sizeof(float);   // up to 4 radial levels per block
  static_assert(sizeof(FwdWsBars) <= 256, "forward barrier block");
  t->smem_fwd = 1024 + fwd_ws_layout(t->nfb, L, c.nth).total;
  if (t->smem_bwd > 227 * 1024 || t->smem_fwd > 227 * 1024) {
    set_error("mixed precision tiles exceed shared memory");
    return CB2_ERR_ARG;
  }
  CB2_CUDA(raise_smem_limit(k_leg_bwd_ws<false>, (int)t->smem_bwd));
  CB2_CUDA(raise_smem_limit(k_pack_bwd, (int)t->smem_pack));
  CB2_CUDA(raise_smem_limit(k_leg_fwd_ws<false>, (int)t->smem_fwd));
  {
    int dev = 0, nsm = 0;
    CB2_CUDA(cudaGetDevice(&dev));
    CB2_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    t->nsm = std::max(1, nsm);
  }
  return 0;
}

void mixed_free(Ctx &c) {
  MixedTables *t = (MixedTables *)c.mixed;
  if (!t) return;
  void *ptrs[] = {t->bb_hi, t->bb_lo, t->bb_unscale, t->bb_ko, t->kbase, t->rlmP, t->rlmD, t->maxP, t->maxD,
                  t->bfp_hi, t->bfp_lo, t->bfd_hi, t->bfd_lo, t->bf_unscale, t->bf_roff, t->bf_nl, t->wgt32,
                  t->rowmax_four, t->fwd_pmax};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete t;
  c.mixed = nullptr;
}

size_t mlayout_floats(const Ctx &c) { return (size_t)(c.L + 1) * c.nth * (26 * (size_t)c.nr + 8); }

MLayout mlayout(const Ctx &c, void *buf, int nvec, int nscal) {
  MLayout l;
  l.nvec = nvec; l.nscal = nscal; l.nr = c.nr; l.nth = c.nth;
  l.P = static_cast<float *>(buf);
  l.D = l.P + (size_t)(c.L + 1) * c.nth * l.sP();
  return l;
}

// CTAs of a persistent Legendre launch over ntiles tiles
static int ws_grid(const Ctx &c, int ntiles) {
  const MixedTables *t = (const MixedTables *)c.mixed;
  const int per = std::max(1, c.ws_tiles_per_cta);
  return std::max(1, std::min(t->nsm, (ntiles + per - 1) / per));
}

// the backward transform's pack kernel (float32 order-major spectra and
// their row maxima), and the GEMM's shell descriptor (no launch)
static int bwd_check(const Ctx &c, const MLayout &out, int &pitchP, int &pitchD) {
  const MixedTables *t = (const MixedTables *)c.mixed;
  const int nvec = out.nvec, ng = out.nvec + out.nscal;
  pitchP = ((2 * ng * c.nr + 3) / 4) * 4;
  pitchD = ((4 * nvec * c.nr + 3) / 4) * 4;
  if (ng > 8 || nvec > 4 || pitchP > t->pitch_max || pitchD > t->pitch_max) {
    set_error("mixed backward transform: at most 8 fields and 4 vectors");
    return CB2_ERR_ARG;
  }
  return 0;
}

int leg_bwd_pack(Ctx &c, const int *slots, const MLayout &out) {
  MixedTables *t = (MixedTables *)c.mixed;
  int pitchP, pitchD, rc;
  if ((rc = bwd_check(c, out, pitchP, pitchD))) return rc;
  const int nvec = out.nvec, ng = out.nvec + out.nscal;
  PackArgs pk{};
  pk.L = c.L; pk.nr = c.nr; pk.jmax = c.jmax; pk.nvec = nvec; pk.ng = ng;
  pk.kc = (c.tune[TUNE_PACK_KC] == 1 || c.tune[TUNE_PACK_KC] == 4) ? c.tune[TUNE_PACK_KC] : 2;
  for (int q = 0; q < ng; q++) pk.slot[q] = slots[q];
  pk.moff = c.d_moff; pk.g3rlm = c.d_g3rlm; pk.ar1 = c.d_ar1; pk.f = c.d_f; pk.fs = c.fsize();
  pk.rlmP = t->rlmP; pk.rlmD = t->rlmD; pk.pitchP = pitchP; pk.pitchD = pitchD;
  pk.kbase = t->kbase; pk.maxP = t->maxP; pk.maxD = t->maxD;
  const size_t smp = (size_t)pk.kc * (2 * ng + 4 * nvec) * ((c.L + 1) | 1) * sizeof(float);
  k_pack_bwd<<<dim3(c.L + 1, cdiv(c.nr, pk.kc)), 256, smp, c.stream>>>(pk);
  return 0;
}

static int bwd_desc(Ctx &c, const MLayout &out, BwdShell &d, int &ntiles) {
  MixedTables *t = (MixedTables *)c.mixed;
  int pitchP, pitchD, rc;
  if ((rc = bwd_check(c, out, pitchP, pitchD))) return rc;
  const int nvec = out.nvec, nscal = out.nscal, ng = nvec + nscal;
  std::memset(&d, 0, sizeof(d));
  if (make_map_any(&d.rawP, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, t->rlmP, pitchP, t->Ktot, TM, FKB,
                   CU_TENSOR_MAP_SWIZZLE_NONE))
    return CB2_ERR_ARG;
  if (nvec > 0) {
    if (make_map_any(&d.rawD, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, t->rlmD, pitchD, t->Ktot, TM, FKB,
                     CU_TENSOR_MAP_SWIZZLE_NONE))
      return CB2_ERR_ARG;
  } else {
    d.rawD = d.rawP;
  }
  d.bhi = t->tm_bb_hi;
  d.blo = t->tm_bb_lo;
  BwdArgs &a = d.a;
  a.L = c.L; a.nr = c.nr; a.nh = c.nh; a.nhp = t->nhp; a.nth = c.nth; a.nvec = nvec; a.nscal = nscal;
  a.pitchP = pitchP; a.pitchD = pitchD;
  a.kbase = t->kbase; a.ko = t->bb_ko; a.maxP = t->maxP; a.maxD = t->maxD;
  a.bunscale = t->bb_unscale; a.out = out; a.status = c.d_status; a.wait_ns = c.pipe_wait_ns;
  d.rows_g0 = ng * 2 * c.nr;
  d.rows_g1 = nvec * 4 * c.nr;
  d.tiles_g0 = cdiv(d.rows_g0, TM);
  d.tiles_g1 = (nvec > 0) ? cdiv(d.rows_g1, TM) : 0;
  d.tile0 = 0;
  ntiles = (d.tiles_g0 + d.tiles_g1) * (c.L + 1);
  return 0;
}

int leg_bwd_gemm(Ctx &c, const MLayout &out) {
  MixedTables *t = (MixedTables *)c.mixed;
  BwdShell d;
  int ntiles, rc;
  if ((rc = bwd_desc(c, out, d, ntiles))) return rc;
  k_leg_bwd_ws<false><<<ws_grid(c, ntiles), BW_THREADS, t->smem_bwd, c.stream>>>(d, nullptr, 1, ntiles, t->nhp,
                                                                                 t->tmem_bwd, t->nacc_bwd);
  return 0;
}

int leg_bwd_mixed(Ctx &c, const int *slots, const MLayout &out) {
  int rc = leg_bwd_pack(c, slots, out);
  return rc ? rc : leg_bwd_gemm(c, out);
}

float *mixed_fwd_pmax(Ctx &c) {
  MixedTables *t = (MixedTables *)c.mixed;
  return t ? t->fwd_pmax : nullptr;
}

const float *mixed_weights32(Ctx &c) {
  MixedTables *t = (MixedTables *)c.mixed;
  return t ? t->wgt32 : nullptr;
}

// the forward transform's row scales: from the four-step FFT kernel's
// partial maxima when it wrote them, else one pass over the Fourier rows
void leg_fwd_rowmax(Ctx &c, const MLayout &in, bool rowmax_ready) {
  MixedTables *t = (MixedTables *)c.mixed;
  if (rowmax_ready && t->fwd_pmax && in.nvec == 4 && in.nscal == 0) {
    const size_t E = in.sP() + in.sD();
    k_rowmax_reduce<<<dim3(cdiv((long)E, 256), t->pmax_mb), 256, 0, c.stream>>>(t->fwd_pmax, c.nth, t->pmax_mb, E,
                                                                               c.L, t->rowmax_four);
  } else {
    k_rowmax_four<<<dim3(cdiv((long)(in.sP() + in.sD()), 256), c.L + 1), 256, 0, c.stream>>>(in, t->wgt32,
                                                                                         t->rowmax_four);
  }
}

static int fwd_desc(Ctx &c, const MLayout &in, const int *slots, FwdShell &d, int &ntiles) {
  MixedTables *t = (MixedTables *)c.mixed;
  const int nvec = in.nvec, nscal = in.nscal;
  std::memset(&d, 0, sizeof(d));
  FwdArgs &a = d.a;
  a.L = c.L; a.nr = c.nr; a.jmax = c.jmax; a.nh = c.nh; a.nhp = t->nhp; a.nth = c.nth; a.NFmax = t->NFmax;
  a.boxr = t->boxr; a.nfb = t->nfb;
  a.nvec = nvec; a.nscal = nscal;
  for (int q = 0; q < nvec + nscal && q < 8; q++) a.slot[q] = slots[q];
  a.moff = c.d_moff; a.g6 = c.d_g6; a.g7 = c.d_g7; a.r = c.d_r; a.wgt = t->wgt32;
  a.f = c.d_f; a.fs = c.fsize();
  a.sP = in.sP(); a.sD = in.sD();
  a.bunscale = t->bf_unscale; a.roff = t->bf_roff; a.nlp = t->bf_nl;
  a.rowmax = t->rowmax_four;
  a.status = c.d_status;
  a.wait_ns = c.pipe_wait_ns;
  a.split = t->split_fwd;
  // raw Fourier rows: float32 [(m, theta)][element], boxes of 128 elements x 32 colatitudes
  const uint64_t nthr = (uint64_t)(c.L + 1) * c.nth;
  if (make_map_any(&d.rawP, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, in.P, in.sP(), nthr, TM, FKB,
                   CU_TENSOR_MAP_SWIZZLE_NONE) ||
      (nvec > 0 && make_map_any(&d.rawD, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, in.D, in.sD(), nthr, TM, FKB,
                                CU_TENSOR_MAP_SWIZZLE_NONE)))
    return CB2_ERR_ARG;
  if (nvec == 0) d.rawD = d.rawP;
  d.phi = t->tm_bfp_hi; d.plo = t->tm_bfp_lo; d.dhi = t->tm_bfd_hi; d.dlo = t->tm_bfd_lo;
  d.rows_g0 = (nvec + nscal) * 2 * c.nr;
  d.rows_g1 = nvec * 4 * c.nr;
  d.tiles_g0 = cdiv(d.rows_g0, TM);
  d.tiles_g1 = (nvec > 0) ? cdiv(d.rows_g1, TM) : 0;
  d.tile0 = 0;
  ntiles = (d.tiles_g0 + d.tiles_g1) * (c.L + 1);
  return 0;
}

int leg_fwd_gemm(Ctx &c, const MLayout &in, const int *slots) {
  MixedTables *t = (MixedTables *)c.mixed;
  FwdShell d;
  int ntiles, rc;
  if ((rc = fwd_desc(c, in, slots, d, ntiles))) return rc;
  k_leg_fwd_ws<false><<<ws_grid(c, ntiles), FW_THREADS, t->smem_fwd, c.stream>>>(d, nullptr, 1, ntiles, t->nfb,
                                                                                 c.nth, t->tmem_fwd, t->nacc_fwd);
  return 0;
}

int leg_fwd_mixed(Ctx &c, const MLayout &in, const int *slots, bool rowmax_ready) {
  leg_fwd_rowmax(c, in, rowmax_ready);
  return leg_fwd_gemm(c, in, slots);
}

// ---------------------------------------------------------------------------
// Ensemble launches: one persistent launch per Legendre GEMM over the
// tiles of every shell (the shells' tables laid end to end, the largest
// first so the long tiles start early).
struct MultiLeg {
  BwdShell *d_bwd = nullptr;
  FwdShell *d_fwd = nullptr;
  BwdShell one_bwd;
  FwdShell one_fwd;
  int nsh = 0, ntiles_bwd = 0, ntiles_fwd = 0, grid = 1;
  int nhp_max = 0, nfb_max = 0;
  uint32_t tmem_bwd = 0, tmem_fwd = 0;
  int nacc_bwd = 1, nacc_fwd = 1;
  size_t smem_bwd = 0, smem_fwd = 0;
};

void multi_leg_free(MultiLeg *m) {
  if (!m) return;
  if (m->d_bwd) cudaFree(m->d_bwd);
  if (m->d_fwd) cudaFree(m->d_fwd);
  delete m;
}

int multi_leg_setup(const std::vector<Ctx *> &shells, int bnvec, int bnscal, const int *fslots, int fnvec, int fnscal,
                    MultiLeg **out) {
  *out = nullptr;
  const int n = (int)shells.size();
  if (n == 0) { set_error("multi-shell Legendre: no shells"); return CB2_ERR_ARG; }
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return (long long)shells[x]->L * shells[x]->nr > (long long)shells[y]->L * shells[y]->nr;
  });
  MultiLeg *m = new MultiLeg();
  std::vector<BwdShell> hb(n);
  std::vector<FwdShell> hf(n);
  int split = -1, rc = 0;
  for (int j = 0; j < n && !rc; j++) {
    Ctx &c = *shells[order[j]];
    const MixedTables *t = (const MixedTables *)c.mixed;
    if (!t || c.prec != CB2_PREC_MIXED) { set_error("multi-shell Legendre: mixed-precision shells only"); rc = CB2_ERR_ARG; break; }
    if (split >= 0 && split != t->split_fwd) {
      set_error("multi-shell Legendre: shells with and without the split forward accumulators");
      rc = CB2_ERR_ARG;
      break;
    }
    split = t->split_fwd;
    int nb, nf;
    if ((rc = bwd_desc(c, mlayout(c, c.d_four, bnvec, bnscal), hb[j], nb)) ||
        (rc = fwd_desc(c, mlayout(c, c.d_four2, fnvec, fnscal), fslots, hf[j], nf)))
      break;
    hb[j].tile0 = m->ntiles_bwd;
    hf[j].tile0 = m->ntiles_fwd;
    m->ntiles_bwd += nb;
    m->ntiles_fwd += nf;
    // shared and tensor memory of the largest shell hold every shell's tiles
    if (t->nhp > m->nhp_max) {
      m->nhp_max = t->nhp;
      m->tmem_bwd = t->tmem_bwd; m->nacc_bwd = t->nacc_bwd; m->smem_bwd = t->smem_bwd;
    }
    if (t->nfb > m->nfb_max || (t->nfb == m->nfb_max && t->tmem_fwd > m->tmem_fwd)) {
      m->nfb_max = t->nfb;
      m->tmem_fwd = t->tmem_fwd; m->nacc_fwd = t->nacc_fwd;
    }
    m->grid = std::max(m->grid, t->nsm);
  }
  if (!rc) {
    m->nsh = n;
    m->one_bwd = hb[0];
    m->one_fwd = hf[0];
    // the forward stages without the staged Gauss weights
    m->smem_fwd = 1024 + fwd_ws_layout(m->nfb_max, 0, 0).total;
    m->grid = std::min(m->grid, std::max(m->ntiles_bwd, m->ntiles_fwd));
    cudaError_t e = cudaMalloc(&m->d_bwd, n * sizeof(BwdShell));
    if (e == cudaSuccess) e = cudaMalloc(&m->d_fwd, n * sizeof(FwdShell));
    if (e == cudaSuccess) e = cudaMemcpy(m->d_bwd, hb.data(), n * sizeof(BwdShell), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_fwd, hf.data(), n * sizeof(FwdShell), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = raise_smem_limit(k_leg_bwd_ws<true>, (int)m->smem_bwd);
    if (e == cudaSuccess) e = raise_smem_limit(k_leg_fwd_ws<true>, (int)m->smem_fwd);
    if (e != cudaSuccess) rc = cuda_fail(e, "multi-shell Legendre tables");
  }
  if (rc) { multi_leg_free(m); return rc; }
  *out = m;
  return 0;
}

void multi_leg_bwd(const MultiLeg *m, cudaStream_t st) {
  k_leg_bwd_ws<true><<<m->grid, BW_THREADS, m->smem_bwd, st>>>(m->one_bwd, m->d_bwd, m->nsh, m->ntiles_bwd,
                                                               m->nhp_max, m->tmem_bwd, m->nacc_bwd);
}

void multi_leg_fwd(const MultiLeg *m, cudaStream_t st) {
  k_leg_fwd_ws<true><<<m->grid, FW_THREADS, m->smem_fwd, st>>>(m->one_fwd, m->d_fwd, m->nsh, m->ntiles_fwd,
                                                               m->nfb_max, 0, m->tmem_fwd, m->nacc_fwd);
}

}  // namespace cb2

