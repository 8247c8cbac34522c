// cb2_legendre_mixed.cu -- Legendre transforms on the tcgen05 tensor cores.
//
// Arithmetic: every operand x is scaled by a power of two s (per GEMM row or
// column, so the largest |x s| lies in [2^13, 2^14)) and split into two
// float16 halves
//     x s = hi + lo,  hi = fp16(x s),  lo = fp16(x s - hi),
// and a product is accumulated in float32 as hi*hi' + hi*lo' + lo*hi'
// (three tcgen05.mma kind::f16 into one TMEM accumulator), unscaled in the
// epilogue.  Scaling to 2^14 rather than 1 keeps lo a normal fp16 number for
// every value within 2^17 of the row (column) maximum, so those values carry
// 22 significant bits; smaller ones keep an absolute error of ~2^-38 of the
// maximum.  The float32 accumulator adds ~2^-24 of the running sum per term.
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
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

namespace {

constexpr int TM = 128;          // GEMM rows per CTA (= TMEM lanes)
constexpr int KB = 64;           // K per pipeline stage: one 128-byte swizzle row of fp16
constexpr int NSTAGE = 2;
constexpr int NTHR = 256;          // two threads per GEMM row
constexpr int ACC1 = 256;        // TMEM column of the parity-1 accumulator
constexpr uint32_t TMEM_COLS = 512;
constexpr unsigned long long kWaitNs = 200ull * 1000 * 1000;   // 200 ms per wait

__device__ inline uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ inline void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// wait for the phase with the given parity to complete; false after kWaitNs
__device__ inline bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 64) t0 = globaltimer();
    if (it > 64) {
      if (globaltimer() - t0 > kWaitNs) return false;
      __nanosleep(32);
    }
  }
}

__device__ inline void tma_load_2d(void *dst, const CUtensorMap *tm, uint64_t *bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (tile base 1024-byte aligned)
__device__ inline uint64_t smem_desc_sw128(const void *p) {
  uint64_t d = (uint64_t)((smem_u32(p) & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1 << 46;                 // descriptor version of tcgen05
  d |= (uint64_t)2 << 61;                 // 128-byte swizzle
  return d;
}

// instruction descriptor: D f32, A and B f16, both K-major, M x N
__device__ inline uint32_t idesc_f16_f32(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ inline void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ inline void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 8 consecutive fp32 columns of this thread's TMEM lane
__device__ inline void tmem_ld8(uint32_t taddr, float v[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                 "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// byte offset of the 16-byte chunk holding elements (row, 8c .. 8c+7) in a
// 128-byte-swizzled K-major tile (the layout TMA SWIZZLE_128B writes)
__device__ inline uint32_t sw128_chunk(int row, int c) {
  return (uint32_t)row * 128u + ((uint32_t)(c ^ (row & 7)) << 4);
}

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

__device__ inline uint32_t pack_half2(__half a, __half b) {
  return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

struct Smem {
  uint64_t full[NSTAGE], empty[NSTAGE], done;
  uint32_t tmem_base;
  int mma_any;
  float rowscale[TM];
};

// Order of the K blocks: both parities of block kb back to back (they read
// the same operand rows), then the blocks only parity 0 has.  Needs
// nkb0 >= nkb1, true for every gemm here.
__device__ inline void block_of(int kbi, int nkb1, int &p, int &kb) {
  if (kbi < 2 * nkb1) { p = kbi & 1; kb = kbi >> 1; }
  else { p = 0; kb = nkb1 + (kbi - 2 * nkb1); }
}

// ---------------------------------------------------------------------------
// The pipelined GEMM of one CTA, shared by the backward and forward kernels.
// Thread t works on tile row r = t % 128 and K half h = t / 128 (warps w and
// w + 4 share TMEM lanes 32 (w % 4) ..).  Prob supplies
//   nkb(p)                K blocks of parity p;
//   kpad(p)               K extent the MMAs read (multiple of 16);
//   n(p)                  MMA N (multiple of 16, <= 256);
//   tma_xy(p, kb, x, y)   origin of the B box;
//   rowmax(r)             an upper bound of |A| over row r (both parities),
//                         from the row-maximum tables;
//   fill(p, kb, r, h, s, hi, lo)  row r's K values 32 h .. 32 h + 31 of block
//                         (p, kb), scaled by s, split and stored as four
//                         16-byte chunks into the swizzled hi / lo tiles.
template <class Prob>
__device__ bool gemm_tile(const Prob &pr, Smem *sh, unsigned char *base, uint32_t b_rows,
                          const CUtensorMap *thi, const CUtensorMap *tlo, int *status) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (TM - 1), h = tid >> 7;
  const uint32_t A_BYTES = TM * 128, B_BYTES = b_rows * 128;
  const uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
  const int nkb1 = pr.nkb(1), total = pr.nkb(0) + nkb1;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; s++) { mbar_init(&sh->full[s], 1); mbar_init(&sh->empty[s], 1); }
    mbar_init(&sh->done, 1);
    sh->mma_any = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // per-row power-of-two scale over every K value of the row (both parities)
  if (h == 0) sh->rowscale[r] = pow2_scale(pr.rowmax(r));
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;
  const float sc = sh->rowscale[r];

  uint32_t ph_full = 0, ph_empty = 0;   // phase parity of each stage's barriers, one bit per stage
  int n_tma = 0, n_full = 0;            // thread 0: B stages requested / consumed
  // fail fast once a wait has run out anywhere in this launch
  int failed = __syncthreads_or((*(volatile int *)status & CB2_STATUS_PIPE_TIMEOUT) != 0);
  auto issue_tma = [&](int kbi) {
    int p, kb, x, y;
    block_of(kbi, nkb1, p, kb);
    pr.tma_xy(p, kb, x, y);
    const int s = kbi % NSTAGE;
    unsigned char *st = base + s * STAGE;
    mbar_expect_tx(&sh->full[s], 2 * B_BYTES);
    tma_load_2d(st + 2 * A_BYTES, thi, &sh->full[s], x, y);
    tma_load_2d(st + 2 * A_BYTES + B_BYTES, tlo, &sh->full[s], x, y);
  };
  if (tid == 0 && total > 0 && !failed) { issue_tma(0); n_tma = 1; }
  for (int kbi = 0; kbi < total && !failed; kbi++) {
    int p, kb;
    block_of(kbi, nkb1, p, kb);
    const int s = kbi % NSTAGE;
    unsigned char *st = base + s * STAGE;
    int f = 0;
    // the A buffers of stage s were last read by the MMAs of block kbi - NSTAGE
    if (kbi >= NSTAGE) {
      if (!mbar_wait(&sh->empty[s], (ph_empty >> s) & 1)) f = 1;
      ph_empty ^= 1u << s;
    }
    // the B tiles of the next block go into the stage the MMAs of block kbi-1 read
    if (tid == 0 && !f && kbi + 1 < total) {
      const int s1 = (kbi + 1) % NSTAGE;
      if (kbi + 1 >= NSTAGE && !mbar_wait(&sh->empty[s1], (ph_empty >> s1) & 1)) f = 1;
      if (!f) { issue_tma(kbi + 1); n_tma++; }
    }
    if (__syncthreads_or(f)) { failed = 1; break; }
    pr.fill(p, kb, r, h, sc, st, st + A_BYTES);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      if (!mbar_wait(&sh->full[s], (ph_full >> s) & 1)) {
        f = 1;
      } else {
        n_full++;
        tc_fence_after();
        const unsigned char *bhi = st + 2 * A_BYTES, *blo = st + 2 * A_BYTES + B_BYTES;
        const uint32_t acc = tmem + (uint32_t)(p * ACC1);
        const uint32_t idesc = idesc_f16_f32(TM, pr.n(p));
        const int nks = (min(KB, pr.kpad(p) - kb * KB) + 15) / 16;
        const uint64_t dah = smem_desc_sw128(st), dal = smem_desc_sw128(st + A_BYTES);
        const uint64_t dbh = smem_desc_sw128(bhi), dbl = smem_desc_sw128(blo);
        for (int ks = 0; ks < nks; ks++) {
          const uint64_t o = (uint64_t)(ks * 2);   // +32 bytes along K
          mma_f16(acc, dah + o, dbh + o, idesc, (kb == 0 && ks == 0) ? 0u : 1u);
          mma_f16(acc, dah + o, dbl + o, idesc, 1u);
          mma_f16(acc, dal + o, dbh + o, idesc, 1u);
        }
        mma_commit(&sh->empty[s]);
        sh->mma_any = 1;
      }
      ph_full ^= 1u << s;
    }
    if (__syncthreads_or(f)) { failed = 1; break; }
  }
  // drain: B loads still in flight, then every MMA this CTA issued
  if (tid == 0) {
    for (; n_full < n_tma; n_full++) {
      const int s = n_full % NSTAGE;
      if (!mbar_wait(&sh->full[s], (ph_full >> s) & 1)) failed = 1;
      ph_full ^= 1u << s;
    }
    if (sh->mma_any) mma_commit(&sh->done);
  }
  __syncthreads();
  int f = failed;
  if (sh->mma_any && !mbar_wait(&sh->done, 0)) f = 1;
  f = __syncthreads_or(f);
  tc_fence_after();
  if (f && tid == 0) atomicOr(status, CB2_STATUS_PIPE_TIMEOUT);
  return !f && total > 0;
}

__device__ inline void tmem_release(Smem *sh) {
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sh->tmem_base), "r"(TMEM_COLS));
}

__device__ inline unsigned char *smem_base_1024(unsigned char *raw) {
  return (unsigned char *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
}

// split 8 scaled values into fp16 hi / lo and store them as one 16-byte chunk each
__device__ inline void store_chunk(unsigned char *hi, unsigned char *lo, int r, int ch, const float x[8]) {
  uint32_t hh[4], ll[4];
#pragma unroll
  for (int e = 0; e < 8; e += 2) {
    const __half h0 = __float2half_rn(x[e]), h1 = __float2half_rn(x[e + 1]);
    hh[e >> 1] = pack_half2(h0, h1);
    ll[e >> 1] = pack_half2(__float2half_rn(x[e] - __half2float(h0)), __float2half_rn(x[e + 1] - __half2float(h1)));
  }
  const uint32_t off = sw128_chunk(r, ch);
  *reinterpret_cast<uint4 *>(hi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
  *reinterpret_cast<uint4 *>(lo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
}

// ---------------------------------------------------------------------------
// backward: spectra f[slot][k][jj] -> order-major Fourier rows
struct BwdArgs {
  int L, nr, jmax, nh, nhp, nth, nvec, nscal;
  int slot[8];
  const int *moff;
  const double *g3rlm, *ar1;
  const double *f;
  size_t fs;
  const float *bunscale;          // [gemm][m][nhp] 1 / column scale of B
  const int *koff, *klen, *n1;    // per (m, group) K offset / length; dP part length
  const float *rowmax;            // [field][comp][k][m][s], k_rowmax_spec
  MLayout out;
  int *status;
};

// One tile row of the backward gemms.  gemm P: row (k, field, s), value at
// K index kk of parity p is f(l = m + p + 2 kk) (times l(l+1)/r^2 for a
// vector).  gemm DM: row (k, vector, q); K = [dP part | mP part]:
// dP part, l = m + (1-p) + 2 kk, value sd * X_d(l); mP part, l = m + p +
// 2 (kk - n1), value sm * X_m(l), with X = (dS/dr)/r or T/r per q.
struct BwdRow {
  const double *xa = nullptr, *xb = nullptr;   // spectra at l = m (nullptr: zero)
  const double *g3 = nullptr;                  // l(l+1) table at l = m (gemm P vectors)
  double fa = 0.0, fb = 0.0;                   // factors incl. sign
};

struct BwdProb {
  const BwdArgs *A;
  int m, g, nrows, row0, nl;
  int kl[2], ko[2], n1[2];
  __device__ int nkb(int p) const { return (kl[p] + KB - 1) / KB; }
  __device__ int kpad(int p) const { return ((kl[p] + 15) / 16) * 16; }
  __device__ int n(int) const { return A->nhp; }
  __device__ void tma_xy(int p, int kb, int &x, int &y) const { x = ko[p] + kb * KB; y = 0; }

  __device__ BwdRow row_src(int r) const {
    const BwdArgs &b = *A;
    BwdRow w;
    const int row = row0 + r;
    if (row >= nrows) return w;
    if (g == 0) {
      const int ng = b.nvec + b.nscal, s = row & 1, v = (row >> 1) % ng, k = (row >> 1) / ng;
      if (m == 0 && s == 1) return w;
      const int jjb = b.moff[m] + s * (b.L + 1 - m);
      w.xa = b.f + (size_t)b.slot[v] * b.fs + (size_t)k * b.jmax + jjb;
      if (v < b.nvec) {
        const double ar = b.ar1[k];
        w.fa = ar * ar;
        w.g3 = b.g3rlm + jjb;
      } else {
        w.fa = 1.0;
      }
      return w;
    }
    // dP part {D+, D-, -T+, -T-}; mP part {T-, -T+, D-, -D+}; comp 1 = dS/dr, 2 = T
    const int q = row & 3, v = (row >> 2) % b.nvec, k = (row >> 2) / b.nvec;
    const double ar = b.ar1[k];
    const int cd = (q < 2) ? 1 : 2, sd = q & 1, cm = (q < 2) ? 2 : 1, smm = (q & 1) ^ 1;
    if (!(m == 0 && sd == 1)) {
      w.xa = b.f + (size_t)(b.slot[v] + cd) * b.fs + (size_t)k * b.jmax + b.moff[m] + sd * (b.L + 1 - m);
      w.fa = (q < 2) ? ar : -ar;
    }
    if (!(m == 0 && smm == 1)) {
      w.xb = b.f + (size_t)(b.slot[v] + cm) * b.fs + (size_t)k * b.jmax + b.moff[m] + smm * (b.L + 1 - m);
      w.fb = (q & 1) ? -ar : ar;
    }
    return w;
  }

  // from the table M[field][comp][k][m][s] = max over l of |S l(l+1)| (comp 0,
  // vectors), |S| (comp 0, scalars), |dS/dr| (comp 1), |T| (comp 2)
  __device__ float rowmax(int r) const {
    const BwdArgs &b = *A;
    const int row = row0 + r;
    if (row >= nrows) return 0.0f;
    const int M1 = b.L + 1;
    auto M = [&](int v, int c, int k, int s) { return b.rowmax[(((size_t)v * 3 + c) * b.nr + k) * 2 * M1 + 2 * m + s]; };
    if (g == 0) {
      const int ng = b.nvec + b.nscal, s = row & 1, v = (row >> 1) % ng, k = (row >> 1) / ng;
      const double ar = b.ar1[k];
      return (float)((double)M(v, 0, k, s) * ((v < b.nvec) ? ar * ar : 1.0));
    }
    const int q = row & 3, v = (row >> 2) % b.nvec, k = (row >> 2) / b.nvec;
    const int cd = (q < 2) ? 1 : 2, sd = q & 1, cm = (q < 2) ? 2 : 1, smm = (q & 1) ^ 1;
    return (float)((double)fmaxf(M(v, cd, k, sd), M(v, cm, k, smm)) * b.ar1[k]);
  }

  __device__ void fill(int p, int kb, int r, int h, float sc, unsigned char *hi, unsigned char *lo) const {
    const BwdRow w = row_src(r);
    const int kk0 = kb * KB + h * 32, klp = kl[p], n1p = n1[p];
    float x[32];
    if (g == 0) {
      const double fa = w.fa * (double)sc;
#pragma unroll
      for (int e = 0; e < 32; e++) {
        const int kk = kk0 + e, t = p + 2 * kk;
        double v = 0.0;
        if (w.xa && kk < klp) v = __ldg(w.xa + t) * (w.g3 ? __ldg(w.g3 + t) : 1.0);
        x[e] = (float)(v * fa);
      }
    } else {
      const double fa = w.fa * (double)sc, fb = w.fb * (double)sc;
#pragma unroll
      for (int e = 0; e < 32; e++) {
        const int kk = kk0 + e;
        double v = 0.0;
        if (kk < n1p) {
          if (w.xa) v = __ldg(w.xa + (1 - p) + 2 * kk) * fa;
        } else if (kk < klp) {
          if (w.xb) v = __ldg(w.xb + p + 2 * (kk - n1p)) * fb;
        }
        x[e] = (float)v;
      }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) store_chunk(hi, lo, r, h * 4 + c, x + 8 * c);
  }
};

__global__ void __launch_bounds__(NTHR, 1)
k_leg_bwd_mixed(const __grid_constant__ BwdArgs a, int rows_g0, int rows_g1, int tiles_g0,
                const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = smem_base_1024(smem_raw);
  const uint32_t BR = (uint32_t)a.nhp;
  Smem *sh = reinterpret_cast<Smem *>(base + NSTAGE * (2 * TM * 128 + 2 * BR * 128));
  BwdProb pr;
  pr.A = &a;
  pr.m = blockIdx.y;
  pr.g = (blockIdx.x < (unsigned)tiles_g0) ? 0 : 1;
  pr.nrows = pr.g ? rows_g1 : rows_g0;
  pr.row0 = (pr.g ? blockIdx.x - tiles_g0 : blockIdx.x) * TM;
  pr.nl = a.L + 1 - pr.m;
  const int m = pr.m;
  for (int p = 0; p < 2; p++) {
    pr.kl[p] = a.klen[m * 4 + 2 * pr.g + p];
    pr.ko[p] = a.koff[m * 4 + 2 * pr.g + p];
    pr.n1[p] = pr.g ? a.n1[m * 2 + p] : 0;
  }
  const bool ok = gemm_tile(pr, sh, base, BR, &tm_hi, &tm_lo, a.status);
  if (ok) {
    // thread: tile row r (TMEM lane), columns (theta) of half h
    const int warp = threadIdx.x >> 5;
    const int r = threadIdx.x & (TM - 1), h = threadIdx.x >> 7, row = pr.row0 + r;
    const bool valid = row < pr.nrows;
    const float ua = 1.0f / sh->rowscale[r];
    const uint32_t tl = sh->tmem_base + ((uint32_t)((warp & 3) * 32) << 16);
    const bool has1 = pr.kl[1] > 0;
    float *outb = pr.g ? a.out.D : a.out.P;
    const size_t so = pr.g ? a.out.sD() : a.out.sP();
    const float *bun = a.bunscale + ((size_t)pr.g * (a.L + 1) + m) * a.nhp;
    const int half = (int)BR / 2;
    for (int t0 = h * half; t0 < (h + 1) * half; t0 += 8) {
      float e[8], o[8];
      tmem_ld8(tl + (uint32_t)t0, e);
      if (has1) {
        tmem_ld8(tl + (uint32_t)(ACC1 + t0), o);
      } else {
#pragma unroll
        for (int q = 0; q < 8; q++) o[q] = 0.0f;
      }
      if (!valid) continue;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int i = t0 + q;
        if (i < a.nh) {
          const float us = ua * bun[i];
          outb[((size_t)m * a.nth + i) * so + row] = (e[q] + o[q]) * us;
          outb[((size_t)m * a.nth + (a.nth - 1 - i)) * so + row] = (e[q] - o[q]) * us;
        }
      }
    }
  }
  tmem_release(sh);
}

// ---------------------------------------------------------------------------
// forward: order-major Fourier rows -> spectra f[slot][k][jj]
//
// One CTA = (order m, parity p of l-m, gemm, tile of 128 rows).  For each
// block of 32 south nodes tb, TMA brings the raw float32 rows of the tile at
// those 32 colatitudes and at their 32 mirror nodes ([theta][row], 16 KB
// each); converter threads form the folded, weighted operand
//   A[row][i] = sg * s_row * (f(i) w_i +- f(i') w_i')     (i' = nth-1-i)
// split into fp16 hi / lo (64-byte swizzled, K = 32) while TMA brings the
// B tiles (P_l^m rows of this parity, 64-byte swizzled).  gemm P takes one
// K block per tb; gemm DM two (dP part: element `row`, fold 1-p; mP part:
// element row - q + 3 - q, fold p).  Three raw stages, three A/B stages, loads
// two blocks ahead.  One accumulator (N = degrees of this parity).
constexpr int FKB = 32;            // K per block (64-byte rows)
constexpr int FST = 3;             // stages (raw and A/B)
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
};

struct FwdSmem {
  uint64_t rawfull[FST], bfull[FST], mmadone[FST], done;
  uint32_t tmem_base;
  int mma_any;
  float rowscale[TM];
  float w[1024];         // Gauss weights (nth <= 1024)
};

// shared-memory descriptor, K-major, 64-byte swizzle (8-row groups 512 bytes apart)
__device__ inline uint64_t smem_desc_sw64(const void *p) {
  uint64_t d = (uint64_t)((smem_u32(p) & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;                 // 64-byte swizzle
  return d;
}

__device__ inline uint32_t sw64_chunk(int row, int c) {
  return (uint32_t)row * 64u + ((uint32_t)(c ^ ((row >> 1) & 3)) << 4);
}

__global__ void __launch_bounds__(NTHR, 1)
k_leg_fwd_tma(const __grid_constant__ FwdArgs a, int rows_g0, int rows_g1, int tiles_g0,
              const __grid_constant__ CUtensorMap tm_rawP, const __grid_constant__ CUtensorMap tm_rawD,
              const __grid_constant__ CUtensorMap tmp_hi, const __grid_constant__ CUtensorMap tmp_lo,
              const __grid_constant__ CUtensorMap tmd_hi, const __grid_constant__ CUtensorMap tmd_lo,
              uint32_t tmem_cols) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *base = smem_base_1024(smem_raw);
  const uint32_t B_BYTES = (uint32_t)a.nfb * FKB * 2;       // one of hi / lo
  const uint32_t AB_BYTES = 2 * FA_BYTES + 2 * B_BYTES;
  unsigned char *raw0 = base;                                // FST x RAW_BYTES
  unsigned char *ab0 = base + FST * RAW_BYTES;               // FST x AB_BYTES
  FwdSmem *sh = reinterpret_cast<FwdSmem *>(ab0 + FST * AB_BYTES);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r = tid & (TM - 1), h = tid >> 7;
  const int m = blockIdx.y, p = blockIdx.z;
  const int g = (blockIdx.x < (unsigned)tiles_g0) ? 0 : 1;
  const int nrows = g ? rows_g1 : rows_g0;
  const int row0 = (g ? blockIdx.x - tiles_g0 : blockIdx.x) * TM;
  const int np = a.nlp[m * 2 + p];
  const int npad = ((np + 15) / 16) * 16;
  const int nbox = (npad + a.boxr - 1) / a.boxr;
  const int NT = (a.nh + FKB - 1) / FKB;                    // theta blocks
  const int NB = g ? 2 * NT : NT;                           // K blocks
  const CUtensorMap *traw = g ? &tm_rawD : &tm_rawP;
  const CUtensorMap *tbh = g ? &tmd_hi : &tmp_hi, *tbl = g ? &tmd_lo : &tmp_lo;
  const int brow = a.roff[m * 2 + p];

  if (tid == 0) {
    for (int q = 0; q < FST; q++) {
      mbar_init(&sh->rawfull[q], 1); mbar_init(&sh->bfull[q], 1); mbar_init(&sh->mmadone[q], 1);
    }
    mbar_init(&sh->done, 1);
    sh->mma_any = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int q = tid; q < a.nth; q += NTHR) sh->w[q] = a.wgt[q];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // row scale from the row-maximum table (a bound of both folds)
  if (h == 0) {
    const int row = row0 + r;
    float mx = 0.0f;
    if (row < nrows && np > 0) {
      const float *Mf = a.rowmax + (size_t)m * (a.sP + a.sD);
      if (g == 0) mx = Mf[row];
      else { const int q = row & 3; mx = fmaxf(Mf[a.sP + row], Mf[a.sP + row - q + 3 - q]); }
    }
    sh->rowscale[r] = pow2_scale(mx);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;

  // block b -> (theta block, part)
  auto tb_of = [&](int b) { return g ? (b >> 1) : b; };
  auto part_of = [&](int b) { return g ? (b & 1) : 0; };
  auto issue_raw = [&](int tb) {
    const int q = tb % FST;
    unsigned char *dst = raw0 + q * RAW_BYTES;
    mbar_expect_tx(&sh->rawfull[q], RAW_BYTES);
    tma_load_2d(dst, traw, &sh->rawfull[q], row0, m * a.nth + tb * FKB);
    tma_load_2d(dst + RAW_BYTES / 2, traw, &sh->rawfull[q], row0, m * a.nth + a.nth - tb * FKB - FKB);
  };
  auto issue_b = [&](int b) {
    const int q = b % FST, tb = tb_of(b), part = part_of(b);
    unsigned char *bh = ab0 + q * AB_BYTES + 2 * FA_BYTES, *bl = bh + B_BYTES;
    const uint32_t bytes = (uint32_t)nbox * a.boxr * FKB * 2;
    mbar_expect_tx(&sh->bfull[q], 2 * bytes);
    const int x = part * a.nhp + tb * FKB;
    for (int j = 0; j < nbox; j++) {
      tma_load_2d(bh + j * a.boxr * FKB * 2, tbh, &sh->bfull[q], x, brow + j * a.boxr);
      tma_load_2d(bl + j * a.boxr * FKB * 2, tbl, &sh->bfull[q], x, brow + j * a.boxr);
    }
  };

  int n_raw = 0, n_b = 0, n_rawdone = 0, n_bdone = 0;     // thread 0 bookkeeping
  int failed = __syncthreads_or((*(volatile int *)a.status & CB2_STATUS_PIPE_TIMEOUT) != 0 || np == 0);
  if (tid == 0 && !failed) {
    for (int tb = 0; tb < min(NT, FST); tb++) { issue_raw(tb); n_raw++; }
    for (int b = 0; b < min(NB, FST - 1); b++) { issue_b(b); n_b++; }
  }
  const int row = row0 + r, q4 = row & 3;
  const float sc = sh->rowscale[r];
  for (int b = 0; b < NB && !failed; b++) {
    const int s = b % FST, tb = tb_of(b), part = part_of(b), rs = tb % FST;
    int f = 0;
    // raw tile of this theta block (all threads observe the phase)
    if (!mbar_wait(&sh->rawfull[rs], (uint32_t)((tb / FST) & 1))) f = 1;
    // A/B stage s was last read by the MMAs of block b - FST
    if (b >= FST && !mbar_wait(&sh->mmadone[s], (uint32_t)(((b - FST) / FST) & 1))) f = 1;
    if (__syncthreads_or(f)) { failed = 1; break; }
    // convert: thread (r, h) builds K values 16 h .. 16 h + 15 of row r
    {
      const float *rs_s = reinterpret_cast<const float *>(raw0 + rs * RAW_BYTES);
      const float *rs_n = rs_s + FKB * TM;
      int src = r, sigma = p;
      float sg = 1.0f;
      if (g) {
        if (part == 0) { sigma = 1 - p; sg = (q4 < 2) ? 1.0f : -1.0f; }
        else { src = r - q4 + 3 - q4; sigma = p; sg = (q4 & 1) ? 1.0f : -1.0f; }
      }
      sg *= sc;
      float x[16];
#pragma unroll
      for (int e = 0; e < 16; e++) {
        const int kk = h * 16 + e, i = tb * FKB + kk;
        float v = 0.0f;
        if (i < a.nh) {
          const float fa = rs_s[kk * TM + src] * sh->w[i];
          const float fb = rs_n[(FKB - 1 - kk) * TM + src] * sh->w[a.nth - 1 - i];
          v = (sigma ? fa - fb : fa + fb) * sg;
        }
        x[e] = v;
      }
      unsigned char *ahi = ab0 + s * AB_BYTES, *alo = ahi + FA_BYTES;
#pragma unroll
      for (int c = 0; c < 2; c++) {
        uint32_t hh[4], ll[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const float x0 = x[c * 8 + e], x1 = x[c * 8 + e + 1];
          const __half h0 = __float2half_rn(x0), h1 = __float2half_rn(x1);
          hh[e >> 1] = pack_half2(h0, h1);
          ll[e >> 1] = pack_half2(__float2half_rn(x0 - __half2float(h0)), __float2half_rn(x1 - __half2float(h1)));
        }
        const uint32_t off = sw64_chunk(r, 2 * h + c);
        *reinterpret_cast<uint4 *>(ahi + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
        *reinterpret_cast<uint4 *>(alo + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
      }
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      // the raw stage of tb is free once its last block is converted
      const bool last_of_tb = (!g) || part == 1;
      if (last_of_tb && tb + FST < NT) { issue_raw(tb + FST); n_raw++; }
      n_rawdone = last_of_tb ? tb + 1 : n_rawdone;
      if (!mbar_wait(&sh->bfull[s], (uint32_t)((b / FST) & 1))) {
        f = 1;
      } else {
        n_bdone = b + 1;
        tc_fence_after();
        unsigned char *ahi = ab0 + s * AB_BYTES, *alo = ahi + FA_BYTES;
        unsigned char *bh = ahi + 2 * FA_BYTES, *bl = bh + B_BYTES;
        const uint32_t idesc = idesc_f16_f32(TM, npad);
        const uint64_t dah = smem_desc_sw64(ahi), dal = smem_desc_sw64(alo);
        const uint64_t dbh = smem_desc_sw64(bh), dbl = smem_desc_sw64(bl);
#pragma unroll
        for (int ks = 0; ks < FKB / 16; ks++) {
          const uint64_t o = (uint64_t)(ks * 2);   // +32 bytes along K
          mma_f16(tmem, dah + o, dbh + o, idesc, (b == 0 && ks == 0) ? 0u : 1u);
          mma_f16(tmem, dah + o, dbl + o, idesc, 1u);
          mma_f16(tmem, dal + o, dbh + o, idesc, 1u);
        }
        mma_commit(&sh->mmadone[s]);
        sh->mma_any = 1;
        // the B tiles of block b + FST - 1 go to the stage the MMAs of block b - 1 used
        const int bn = b + FST - 1;
        if (bn < NB) {
          if (bn >= FST && !mbar_wait(&sh->mmadone[bn % FST], (uint32_t)(((bn - FST) / FST) & 1))) f = 1;
          else { issue_b(bn); n_b++; }
        }
      }
    }
    if (__syncthreads_or(f)) { failed = 1; break; }
  }
  // drain: loads still in flight (raw and B), then every MMA
  if (tid == 0) {
    for (int tb = n_rawdone; tb < n_raw; tb++)
      if (!mbar_wait(&sh->rawfull[tb % FST], (uint32_t)((tb / FST) & 1))) failed = 1;
    for (int b = n_bdone; b < n_b; b++)
      if (!mbar_wait(&sh->bfull[b % FST], (uint32_t)((b / FST) & 1))) failed = 1;
    if (sh->mma_any) mma_commit(&sh->done);
  }
  __syncthreads();
  int f = failed && np > 0;
  if (sh->mma_any && !mbar_wait(&sh->done, 0)) f = 1;
  f = __syncthreads_or(f);
  tc_fence_after();
  if (f && tid == 0) atomicOr(a.status, CB2_STATUS_PIPE_TIMEOUT);
  if (!f && np > 0) {
    int k, slot, kind, s;   // kind 0: S (g7 r^2), 1: dS or T (g7 r), 2: scalar (g6)
    if (g == 0) {
      const int ng = a.nvec + a.nscal, v = (row >> 1) % ng;
      s = row & 1; k = (row >> 1) / ng;
      slot = a.slot[v]; kind = (v < a.nvec) ? 0 : 2;
    } else {
      const int v = (row >> 2) % a.nvec;
      k = (row >> 2) / a.nvec; s = q4 & 1;
      slot = a.slot[v] + 1 + (q4 >> 1); kind = 1;
    }
    const bool valid = row < nrows && !(m == 0 && s == 1);
    const double ua = 1.0 / (double)sc;
    const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const double rk = valid ? a.r[k] : 0.0;
    const int jjb = a.moff[m] + s * (a.L + 1 - m);
    double *dst = a.f + (size_t)slot * a.fs + (size_t)k * a.jmax + jjb;
    const float *bun = a.bunscale + ((size_t)g * (a.L + 1) * 2 + m * 2 + p) * a.NFmax;
    const int nch = (np + 7) / 8;
    for (int c8 = h; c8 < nch; c8 += 2) {
      float v8[8];
      tmem_ld8(tl + (uint32_t)(c8 * 8), v8);
      if (!valid) continue;
#pragma unroll
      for (int qq = 0; qq < 8; qq++) {
        const int t = c8 * 8 + qq;
        if (t < np) {
          const int lm = p + 2 * t;   // l - m
          const double fac = (kind == 0) ? a.g7[jjb + lm] * rk * rk
                           : (kind == 2) ? a.g6[jjb + lm] : a.g7[jjb + lm] * rk;
          dst[lm] = (double)v8[qq] * (ua * (double)bun[t]) * fac;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// ---------------------------------------------------------------------------
// Row maxima for the operand scales, one streaming pass each.
//
// spectra: M[field][comp][k][m][s] = max over l = m..L of |X(l, m, s)|, X =
// S l(l+1) (vector comp 0; l(l+1) from g3rlm), S (scalar), dS/dr, T; one
// warp per (m, s) block of one (field, comp, k) row, lanes over l.
struct Slots8 {
  int s[8];
};

__global__ void __launch_bounds__(256)
k_rowmax_spec(int L, int nr, int jmax, int nvec, Slots8 slot, const int *moff, const double *g3rlm,
              const double *f, size_t fs, float *M) {
  const int k = blockIdx.x, v = blockIdx.y, c = blockIdx.z;
  const bool isvec = v < nvec;
  if (!isvec && c > 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, M1 = L + 1;
  const double *x = f + (size_t)(slot.s[v] + c) * fs + (size_t)k * jmax;
  float *out = M + (((size_t)v * 3 + c) * nr + k) * 2 * M1;
  for (int seg = warp; seg < 2 * M1; seg += blockDim.x >> 5) {
    const int m = seg >> 1, s = seg & 1;
    if (m == 0 && s == 1) {
      if (lane == 0) out[1] = 0.0f;
      continue;
    }
    const int nl = L + 1 - m, jjb = moff[m] + s * (L + 1 - m);
    double mx = 0.0;
    for (int t = lane; t < nl; t += 32) {
      double a = fabs(x[jjb + t]);
      if (isvec && c == 0) a *= g3rlm[jjb + t];
      mx = fmax(mx, a);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) out[seg] = (float)mx;
  }
}

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
  float mx = 0.0f;
#pragma unroll 8
  for (int th = 0; th < in.nth; th++) mx = fmaxf(mx, fabsf(__ldg(x + (size_t)th * st)) * __ldg(wgt + th));
  Mf[(size_t)m * (sP + sD) + e] = 2.0f * mx;
}

// ---------------------------------------------------------------------------
// B operands: scaled fp16 hi/lo copies of the float64 P tables
__device__ inline void split_store(__half *hi, __half *lo, size_t at, double v, float s) {
  const double x = v * (double)s;
  const __half h = __float2half_rn((float)x);
  hi[at] = h;
  lo[at] = __float2half_rn((float)(x - (double)__half2float(h)));
}

// backward B[theta][K]: one thread per (m, south node i)
__global__ void k_build_bwd_b(int L, int nh, int nhp, const size_t *poff, const double *Plt, const double *dPlt,
                              const double *asin_t, const int *koff, const int *klen, const int *n1, int Kb_all,
                              float *bunscale, __half *bhi, __half *blo) {
  const int m = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L || i >= nh) return;
  const int nl = L + 1 - m;
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
  for (int gi = 0; gi < 4; gi++) {
    const int ko = koff[m * 4 + gi], kl = klen[m * 4 + gi];
    const float s = (gi < 2) ? sp : sd;
    for (int kk = 0; kk < kl; kk++) {
      double v;
      if (gi < 2) {
        const int l = m + gi + 2 * kk;
        v = Plt[po + (size_t)(l - m) * nh + i];
      } else {
        const int p = gi - 2, nn = n1[m * 2 + p];
        if (kk < nn) {
          const int l = m + (1 - p) + 2 * kk;
          v = dPlt[po + (size_t)(l - m) * nh + i];
        } else {
          const int l = m + p + 2 * (kk - nn);
          v = Plt[po + (size_t)(l - m) * nh + i] * am;
        }
      }
      split_store(bhi, blo, (size_t)i * Kb_all + ko + kk, v, s);
    }
  }
}

// forward B[l][theta] (P) and B[l][dP theta | mP theta] (DM): one thread per (m, degree)
__global__ void k_build_fwd_b(int L, int nh, int nhp, int NFmax, const size_t *poff, const double *Plt,
                              const double *dPlt, const double *asin_t, const int *roff, const int *nlp,
                              float *bunscale, __half *php, __half *plp, __half *dhp, __half *dlp) {
  const int m = blockIdx.y, t = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L) return;
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
      split_store(php, plp, row * nhp + i, P, sp);
      split_store(dhp, dlp, row * 2 * nhp + i, dPlt[po + (size_t)(l - m) * nh + i], sd);
      split_store(dhp, dlp, row * 2 * nhp + nhp + i, P * (double)m * asin_t[i], sd);
    }
  }
}

// ---------------------------------------------------------------------------
// host side
struct MixedTables {
  __half *bb_hi = nullptr, *bb_lo = nullptr;      // backward B [nhp][Kb_all]
  float *bb_unscale = nullptr;                    // [gemm][m][nhp]
  int *bb_koff = nullptr, *bb_klen = nullptr, *bb_n1 = nullptr;
  __half *bfp_hi = nullptr, *bfp_lo = nullptr;    // forward B (P) [rows_all][nhp]
  __half *bfd_hi = nullptr, *bfd_lo = nullptr;    // forward B (DM) [rows_all][2 nhp]
  float *bf_unscale = nullptr;                    // [gemm][(m, parity)][NFmax]
  int *bf_roff = nullptr, *bf_nl = nullptr;
  float *wgt32 = nullptr;                         // Gauss weights in float
  float *rowmax_spec = nullptr;                   // [8 fields][3][nr][2 (L+1)]
  float *rowmax_four = nullptr;                   // [(L+1)][26 nr + 8]
  int Kb_all = 0, rows_all = 0, nhp = 0, NFmax = 0;
  size_t smem_bwd = 0, smem_fwd = 0;
  CUtensorMap tm_bb_hi, tm_bb_lo, tm_bfp_hi, tm_bfp_lo, tm_bfd_hi, tm_bfd_lo;
  int boxr = 0, nfb = 0;
  uint32_t tmem_fwd = 0;
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

// fp16 [rows][cols], box 64 x box_rows, 128-byte swizzle (backward B tiles)
int make_map(CUtensorMap *tm, const void *ptr, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  if (rows < box_rows) { set_error("tensor map shape"); return CB2_ERR_ARG; }
  return make_map_any(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, ptr, cols, rows, KB, box_rows,
                      CU_TENSOR_MAP_SWIZZLE_128B);
}

// fp16 [rows][cols], box 32 x box_rows, 64-byte swizzle (forward B tiles)
int make_map64(CUtensorMap *tm, const void *ptr, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  return make_map_any(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, ptr, cols, rows, FKB, box_rows,
                      CU_TENSOR_MAP_SWIZZLE_64B);
}

// 1024 alignment slack + stages + control block; at least 120 KB so a CTA
// holding 512 TMEM columns has the SM to itself
size_t smem_bytes(int b_rows) {
  size_t s = 1024 + (size_t)NSTAGE * (2 * TM * 128 + 2 * (size_t)b_rows * 128) + sizeof(Smem);
  return std::max(s, (size_t)120 * 1024);
}

}  // namespace

int mixed_setup(Ctx &c) {
  MixedTables *t = new MixedTables();
  c.mixed = t;
  const int L = c.L, nh = c.nh;
  t->nhp = ((nh + 15) / 16) * 16;
  if (t->nhp > 256) { set_error("mixed precision path needs nth <= 512"); return CB2_ERR_ARG; }
  // backward K groups per m: P0, P1 (l-m even / odd), D0 = {dP odd | mP even}, D1 = {dP even | mP odd}
  std::vector<int> koff((L + 1) * 4), klen((L + 1) * 4), n1((L + 1) * 2);
  int K = 0;
  for (int m = 0; m <= L; m++) {
    const int nl = L + 1 - m, ne = (nl + 1) / 2, no = nl / 2;
    const int lens[4] = {ne, no, no + ne, ne + no};
    n1[m * 2 + 0] = no;
    n1[m * 2 + 1] = ne;
    for (int gi = 0; gi < 4; gi++) {
      koff[m * 4 + gi] = K;
      klen[m * 4 + gi] = lens[gi];
      K += ((lens[gi] + 15) / 16) * 16;
    }
  }
  t->Kb_all = K + KB;   // every 64-wide box starting at a group stays in the array
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
  t->tmem_fwd = 32;
  while ((int)t->tmem_fwd < t->NFmax) t->tmem_fwd *= 2;
  t->rows_all = R + t->NFmax;   // every NFmax-row box stays in the array
  auto up = [&](int **d, const std::vector<int> &v) -> int {
    CB2_CUDA(cudaMalloc(d, v.size() * sizeof(int)));
    CB2_CUDA(cudaMemcpy(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  };
  int rc;
  if ((rc = up(&t->bb_koff, koff)) || (rc = up(&t->bb_klen, klen)) || (rc = up(&t->bb_n1, n1)) ||
      (rc = up(&t->bf_roff, roff)) || (rc = up(&t->bf_nl, nlp)))
    return rc;
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
  CB2_CUDA(cudaMalloc(&t->rowmax_spec, (size_t)8 * 3 * c.nr * 2 * (L + 1) * sizeof(float)));
  CB2_CUDA(cudaMalloc(&t->rowmax_four, (size_t)(L + 1) * (26 * (size_t)c.nr + 8) * sizeof(float)));
  k_build_bwd_b<<<dim3(cdiv(nh, 64), L + 1), 64, 0, c.stream>>>(L, nh, t->nhp, c.d_poff, c.d_Plt, c.d_dPlt,
                                                                c.d_asin, t->bb_koff, t->bb_klen, t->bb_n1,
                                                                t->Kb_all, t->bb_unscale, t->bb_hi, t->bb_lo);
  CB2_CUDA(cudaGetLastError());
  k_build_fwd_b<<<dim3(cdiv(t->NFmax, 64), L + 1), 64, 0, c.stream>>>(
      L, nh, t->nhp, t->NFmax, c.d_poff, c.d_Plt, c.d_dPlt, c.d_asin, t->bf_roff, t->bf_nl, t->bf_unscale,
      t->bfp_hi, t->bfp_lo, t->bfd_hi, t->bfd_lo);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  if ((rc = make_map(&t->tm_bb_hi, t->bb_hi, t->Kb_all, t->nhp, t->nhp)) ||
      (rc = make_map(&t->tm_bb_lo, t->bb_lo, t->Kb_all, t->nhp, t->nhp)) ||
      (rc = make_map64(&t->tm_bfp_hi, t->bfp_hi, t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfp_lo, t->bfp_lo, t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfd_hi, t->bfd_hi, 2 * t->nhp, t->rows_all, t->boxr)) ||
      (rc = make_map64(&t->tm_bfd_lo, t->bfd_lo, 2 * t->nhp, t->rows_all, t->boxr)))
    return rc;
  t->smem_bwd = smem_bytes(t->nhp);
  t->smem_fwd = 1024 + FST * (size_t)RAW_BYTES + FST * (2 * (size_t)FA_BYTES + 2 * (size_t)t->nfb * FKB * 2) +
                sizeof(FwdSmem);
  if (t->smem_bwd > 227 * 1024 || t->smem_fwd > 227 * 1024) {
    set_error("mixed precision tiles exceed shared memory");
    return CB2_ERR_ARG;
  }
  CB2_CUDA(cudaFuncSetAttribute(k_leg_bwd_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem_bwd));
  CB2_CUDA(cudaFuncSetAttribute(k_leg_fwd_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem_fwd));
  return 0;
}

void mixed_free(Ctx &c) {
  MixedTables *t = (MixedTables *)c.mixed;
  if (!t) return;
  void *ptrs[] = {t->bb_hi, t->bb_lo, t->bb_unscale, t->bb_koff, t->bb_klen, t->bb_n1, t->bfp_hi,
                  t->bfp_lo, t->bfd_hi, t->bfd_lo, t->bf_unscale, t->bf_roff, t->bf_nl, t->wgt32,
                  t->rowmax_spec, t->rowmax_four};
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

int leg_bwd_mixed(Ctx &c, const int *slots, const MLayout &out) {
  MixedTables *t = (MixedTables *)c.mixed;
  const int nvec = out.nvec, nscal = out.nscal;
  BwdArgs a{};
  a.L = c.L; a.nr = c.nr; a.jmax = c.jmax; a.nh = c.nh; a.nhp = t->nhp; a.nth = c.nth;
  a.nvec = nvec; a.nscal = nscal;
  for (int q = 0; q < nvec + nscal && q < 8; q++) a.slot[q] = slots[q];
  a.moff = c.d_moff; a.g3rlm = c.d_g3rlm; a.ar1 = c.d_ar1; a.f = c.d_f; a.fs = c.fsize();
  a.bunscale = t->bb_unscale; a.koff = t->bb_koff; a.klen = t->bb_klen; a.n1 = t->bb_n1;
  a.rowmax = t->rowmax_spec;
  a.out = out; a.status = c.d_status;
  Slots8 sl{};
  for (int q = 0; q < nvec + nscal && q < 8; q++) sl.s[q] = slots[q];
  k_rowmax_spec<<<dim3(c.nr, nvec + nscal, 3), 256, 0, c.stream>>>(c.L, c.nr, c.jmax, nvec, sl, c.d_moff, c.d_g3rlm,
                                                                  c.d_f, c.fsize(), t->rowmax_spec);
  const int rows0 = (nvec + nscal) * 2 * c.nr, rows1 = nvec * 4 * c.nr;
  const int tiles0 = cdiv(rows0, TM), tiles1 = (nvec > 0) ? cdiv(rows1, TM) : 0;
  k_leg_bwd_mixed<<<dim3(tiles0 + tiles1, c.L + 1), NTHR, t->smem_bwd, c.stream>>>(a, rows0, rows1, tiles0,
                                                                                  t->tm_bb_hi, t->tm_bb_lo);
  return 0;
}

int leg_fwd_mixed(Ctx &c, const MLayout &in, const int *slots) {
  MixedTables *t = (MixedTables *)c.mixed;
  const int nvec = in.nvec, nscal = in.nscal;
  FwdArgs a{};
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
  // raw Fourier rows: float32 [(m, theta)][element], boxes of 128 elements x 32 colatitudes
  CUtensorMap rawP{}, rawD{};
  const uint64_t nthr = (uint64_t)(c.L + 1) * c.nth;
  if (make_map_any(&rawP, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, in.P, in.sP(), nthr, TM, FKB,
                   CU_TENSOR_MAP_SWIZZLE_NONE) ||
      (nvec > 0 && make_map_any(&rawD, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, in.D, in.sD(), nthr, TM, FKB,
                                CU_TENSOR_MAP_SWIZZLE_NONE))) {
    return CB2_ERR_ARG;
  }
  if (nvec == 0) rawD = rawP;
  k_rowmax_four<<<dim3(cdiv((long)(in.sP() + in.sD()), 256), c.L + 1), 256, 0, c.stream>>>(in, t->wgt32,
                                                                                       t->rowmax_four);
  const int rows0 = (nvec + nscal) * 2 * c.nr, rows1 = nvec * 4 * c.nr;
  const int tiles0 = cdiv(rows0, TM), tiles1 = (nvec > 0) ? cdiv(rows1, TM) : 0;
  k_leg_fwd_tma<<<dim3(tiles0 + tiles1, c.L + 1, 2), NTHR, t->smem_fwd, c.stream>>>(
      a, rows0, rows1, tiles0, rawP, rawD, t->tm_bfp_hi, t->tm_bfp_lo, t->tm_bfd_hi, t->tm_bfd_lo, t->tmem_fwd);
  return 0;
}

}  // namespace cb2
