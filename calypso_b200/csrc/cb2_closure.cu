// cb2_closure.cu -- learned spectral subgrid closure (no counterpart in the
// reference: its SGS hooks, MHD_src/sph_MHD/cal_explicit_terms.f90:70-95,
// have no call sites on the spherical-shell path).
//
// A low-resolution shell (truncation L_lo) misses the part of its nonlinear
// terms that comes from the modes it does not carry.  The closure predicts
// that part per radial level and per (l, m) from local spectral features:
//   tau(k, l, m) = P_lo[N(u_hi)](k, l, m) - N_lo(P_lo u_hi)(k, l, m)
// for the five explicit nonlinear terms of the evolved equations (curl of
// the forces S and T, induction S and T, heat advection).  P_lo truncates
// to l <= L_lo and restricts to the low-resolution radial points (which must
// be a subset of the high-resolution Chebyshev points).
//
// Network: MLP nin -> nhid -> nhid -> nout, SiLU activations, weights kept
// in bfloat16 for every product (float32 master copy for the optimiser),
// float32 activations and accumulation.  Kernels: a tiled GEMM with either
// operand transposed (split-K with float32 atomics for the weight
// gradients), bias + activation, its derivative, column sums and Adam.
// Training runs on the GPU through these kernels; the oracle restates the
// same forward and backward in float64 (numpy) to check the gradients.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cb2_internal.cuh"
#include "cb2_tc.cuh"

namespace cb2 {
namespace {

constexpr int NF = 16;   // features per (k, l, m)
constexpr int NO = 5;    // predicted tendencies

struct Slots16 {
  int s[16];
};

// field slots read as features and the slots the closure adds to
Slots16 feat_slots() {
  return Slots16{{VELO, VELO + 1, VELO + 2, VORT, VORT + 1, VORT + 2, MAGNE, MAGNE + 1, MAGNE + 2, CURRENT,
                  CURRENT + 1, CURRENT + 2, TEMP, 0, 0, 0}};
}
Slots16 out_slots() { return Slots16{{FORCES, FORCES + 2, INDUCT, INDUCT + 2, HADV, 0}}; }

// ---------------------------------------------------------------------------
// filtering between shells: dst(k, l, m) = src(k * stride, l, m), l <= L_dst
__global__ void k_filter(int nr_dst, int jmax_dst, int jmax_src, int Lsrc, int stride, const int *jl, const int *jm,
                         const int *moff_src, const double *src, size_t fs_src, double *dst, size_t fs_dst,
                         Slots16 ss, Slots16 sd, int nslots, int to_buffer) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nr_dst * jmax_dst) return;
  const int k = (int)(i / jmax_dst), jj = (int)(i - (size_t)k * jmax_dst);
  const int l = jl[jj], m = jm[jj], am = m < 0 ? -m : m;
  const int jjs = moff_src[am] + (m < 0 ? (Lsrc + 1 - am) : 0) + (l - am);
  const size_t at_s = (size_t)(k * stride) * jmax_src + jjs;
  for (int q = 0; q < nslots; q++) {
    const double v = src[(size_t)ss.s[q] * fs_src + at_s];
    if (to_buffer) dst[(size_t)q * fs_dst + i] = v;
    else dst[(size_t)sd.s[q] * fs_dst + i] = v;
  }
}

// features X[row][16], row = k * jmax + jj: the 13 evolved / derived field
// coefficients, l / L, m / L (negative for the sin part), r mapped to [-1, 1]
__global__ void k_features(int nr, int jmax, int L, const int *jl, const int *jm, const double *r, double ri,
                           double ro, const double *f, size_t fs, Slots16 fsl, float *X) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nr * jmax) return;
  const int k = (int)(i / jmax), jj = (int)(i - (size_t)k * jmax);
  float *x = X + i * NF;
#pragma unroll
  for (int q = 0; q < 13; q++) x[q] = (float)f[(size_t)fsl.s[q] * fs + i];
  x[13] = (float)jl[jj] / (float)L;
  x[14] = (float)jm[jj] / (float)L;
  x[15] = (float)((2.0 * r[k] - (ri + ro)) / (ro - ri));
}

// normalised features: (x - mean[k]) / std[k] per radial level k
__global__ void k_normalise(size_t n, int jmax, const float *X, const float *mean, const float *istd, float *Xn) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * NF) return;
  const size_t row = i / NF;
  const int q = (int)(i - row * NF), k = (int)(row / jmax);
  Xn[i] = (X[i] - mean[k * NF + q]) * istd[k * NF + q];
}

// targets Y[row][5] = hi[c][row] - lo slot c (row)
__global__ void k_targets(size_t n, const double *hi, const double *f, size_t fs, Slots16 osl, float *Y) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int c = 0; c < NO; c++) Y[i * NO + c] = (float)(hi[(size_t)c * n + i] - f[(size_t)osl.s[c] * fs + i]);
}

// slot c (row) += Y[row][c] * scale[k][c] at the interior radial levels
// (the wall levels are set by the boundary conditions and left alone)
__global__ void k_add_tendency(size_t n, int nr, int jmax, const float *Y, const float *scale, double *f, size_t fs,
                               Slots16 osl) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = (int)(i / jmax);
  if (k == 0 || k == nr - 1) return;
#pragma unroll
  for (int c = 0; c < NO; c++) f[(size_t)osl.s[c] * fs + i] += (double)(Y[i * NO + c] * scale[k * NO + c]);
}

// ---------------------------------------------------------------------------
// GEMM on the tensor cores: C[M][N] (+)= sum_k opA[m][k] opB[k][n];
//   opA[m][k] = TA ? A[k * lda + m] : A[m * lda + k]
//   opB[k][n] = TB ? B[n * ldb + k] : B[k * ldb + n]
// One CTA (128 threads) per tile of 128 rows x NT <= 256 columns and per
// chunk of K (blockIdx.z, partial sums added with float32 atomics when
// `atomic`).  K runs in blocks of 32: the threads load both operand tiles,
// split float32 values into bfloat16 hi + lo (x = hi + lo to 16 bits;
// bfloat16 weights are one exact term) and write them K-major, 64-byte
// swizzled, into one of two shared-memory stages; one thread issues
// tcgen05.mma kind::f16 with bf16 operands (hi*hi', hi*lo', lo*hi': the
// products that reach 2^-16 of the result) into a float32 TMEM accumulator
// and commits to the stage's mbarrier, which the loads of the stage after
// next wait on.  Every wait is bounded; a wait that runs out sets bit 2 of
// *status and the CTA drains its MMAs, frees its TMEM and returns.
constexpr int GK = 32;                        // K per stage (64-byte rows)
constexpr unsigned long long kWaitNsGemm = 200ull * 1000 * 1000;
constexpr uint32_t GA_BYTES = 128 * GK * 2;   // one bf16 term of the A tile

template <typename T> struct Terms { static constexpr int n = 2; };
template <> struct Terms<__nv_bfloat16> { static constexpr int n = 1; };

__device__ inline float to_f(float x) { return x; }
__device__ inline float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

// 8 consecutive K values of one row -> nt bf16 terms, 16 bytes each
template <int NT_>
__device__ inline void put_row8(unsigned char *tile, uint32_t term_bytes, int row, int chunk, const float v[8]) {
  uint32_t hi[4], lo[4];
#pragma unroll
  for (int e = 0; e < 8; e += 2) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[e], v[e + 1]);
    const float2 f = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(v[e] - f.x, v[e + 1] - f.y);
    hi[e >> 1] = *reinterpret_cast<const uint32_t *>(&h);
    lo[e >> 1] = *reinterpret_cast<const uint32_t *>(&l);
  }
  const uint32_t off = tc::sw64_chunk(row, chunk);
  *reinterpret_cast<uint4 *>(tile + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  if (NT_ > 1) *reinterpret_cast<uint4 *>(tile + term_bytes + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

template <typename TAT, typename TBT, bool TA, bool TB>
__global__ void __launch_bounds__(128)
k_tc_gemm(int M, int N, int NT, int K, const TAT *__restrict__ A, int lda, const TBT *__restrict__ B, int ldb,
          float *C, int ldc, int kchunk, int atomic, uint32_t tmem_cols, int *status, unsigned long long wait_ns) {
  constexpr int NA = Terms<TAT>::n, NBT = Terms<TBT>::n;
  extern __shared__ unsigned char g_smem_raw[];
  unsigned char *base = tc::smem_base_1024(g_smem_raw);
  const uint32_t b_bytes = (uint32_t)NT * GK * 2;               // one bf16 term of the B tile
  const uint32_t stage_bytes = ((NA * GA_BYTES + NBT * b_bytes) + 1023u) & ~1023u;
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * stage_bytes);   // [2] stage done, [2] final
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 3);
  int *abort = reinterpret_cast<int *>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * 128, n0 = blockIdx.x * NT;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1); tc::mbar_init(&bar[1], 1); tc::mbar_init(&bar[2], 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(tslot, tmem_cols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = tc::idesc_bf16_f32(128, NT);
  const int nblk = (ke - kb + GK - 1) / GK;
  bool bad = false;
  for (int ib = 0; ib < nblk; ib++) {
    const int st = ib & 1, k0 = kb + ib * GK;
    unsigned char *ta = base + st * stage_bytes, *tbp = ta + NA * GA_BYTES;
    // the stage's previous MMAs (block ib - 2) must have read it
    if (ib >= 2 && !tc::mbar_wait(&bar[st], ((ib - 2) >> 1) & 1, wait_ns)) bad = true;
    if (__syncthreads_or(bad)) { bad = true; break; }
    // A tile: thread = row
    {
      const int m = m0 + tid;
#pragma unroll
      for (int c = 0; c < GK / 8; c++) {
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const int k = k0 + c * 8 + e;
          v[e] = (m < M && k < ke) ? to_f(TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : 0.0f;
        }
        put_row8<NA>(ta, GA_BYTES, tid, c, v);
      }
    }
    // B tile: rows n of the column tile
    for (int r = tid; r < NT; r += 128) {
      const int n = n0 + r;
#pragma unroll
      for (int c = 0; c < GK / 8; c++) {
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const int k = k0 + c * 8 + e;
          v[e] = (n < N && k < ke) ? to_f(TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) : 0.0f;
        }
        put_row8<NBT>(tbp, b_bytes, r, c, v);
      }
    }
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < GK / 16; ks++) {
        const uint64_t o = (uint64_t)(ks * 2);
        const uint64_t ah = tc::smem_desc_sw64(ta) + o, bh = tc::smem_desc_sw64(tbp) + o;
        tc::mma_f16(tmem, ah, bh, idesc, (ib == 0 && ks == 0) ? 0u : 1u);
        if (NBT > 1) tc::mma_f16(tmem, ah, tc::smem_desc_sw64(tbp + b_bytes) + o, idesc, 1u);
        if (NA > 1) tc::mma_f16(tmem, tc::smem_desc_sw64(ta + GA_BYTES) + o, bh, idesc, 1u);
      }
      tc::mma_commit(&bar[st]);
    }
  }
  // every MMA has completed before the accumulator is read and freed
  if (tid == 0) {
    if (nblk > 0) tc::mma_commit(&bar[2]);
  }
  __syncthreads();
  const bool done = nblk == 0 || tc::mbar_wait(&bar[2], 0, tc::kWaitNs);
  if (!done || bad) {
    if (tid == 0) atomicOr(status, CB2_STATUS_PIPE_TIMEOUT);
    *abort = 1;
  }
  __syncthreads();
  tc::tc_fence_after();
  if (!*abort && nblk > 0) {
    // epilogue: warp w holds TMEM lanes 32 w .. 32 w + 31 (tile rows), a
    // thread 64 columns of its row per load; through the warp's 32 x 65
    // staging (the stage buffers are free now) a store then writes 32
    // consecutive columns of one row
    float *stg = reinterpret_cast<float *>(base) + warp * 32 * 65;
    for (int c0 = 0; c0 < NT; c0 += 64) {
      float va[32], vb[32];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      tc::tmem_ld32x2(ta, ta + 32, va, vb);
#pragma unroll
      for (int j = 0; j < 32; j++) { stg[lane * 65 + j] = va[j]; stg[lane * 65 + 32 + j] = vb[j]; }
      __syncwarp();
      for (int r = 0; r < 32; r++) {
        const int m = m0 + warp * 32 + r;
        if (m >= M) break;
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
          const int cc = c0 + 32 * hh + lane, n = n0 + cc;
          if (cc < NT && n < N) {
            float *cp = C + (size_t)m * ldc + n;
            const float v = stg[r * 65 + 32 * hh + lane];
            if (atomic) atomicAdd(cp, v); else *cp = v;
          }
        }
      }
      __syncwarp();
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, tmem_cols);
}

__device__ inline float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }

// Z += b (per column); H = SiLU(Z) (act != 0) or Z
__global__ void k_bias_act(size_t n, int w, float *Z, const float *b, float *H, int act) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * w) return;
  const float z = Z[i] + b[i % w];
  Z[i] = z;
  H[i] = act ? z * sigm(z) : z;
}

// dZ = dH * SiLU'(Z)
__global__ void k_act_grad(size_t n, const float *Z, const float *dH, float *dZ) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float s = sigm(Z[i]);
  dZ[i] = dH[i] * s * (1.0f + Z[i] * (1.0f - s));
}

// dY = 2 (Y - T) / (n nout); partial loss sums (float64) per block
__global__ void k_mse(size_t n, int w, const float *Y, const float *T, float *dY, double *part) {
  __shared__ double sh[256];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < n * w) {
    const float d = Y[i] - T[i];
    dY[i] = 2.0f * d / (float)(n * (size_t)w);
    e = (double)d * (double)d;
  }
  sh[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// column sums of X[n][w] into out[w] (one block per column, float64 partials)
__global__ void k_colsum(size_t n, int w, const float *X, float *out) {
  __shared__ double sh[256];
  const int c = blockIdx.x;
  double s = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += X[i * w + c];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int q = blockDim.x / 2; q > 0; q >>= 1) {
    if (threadIdx.x < q) sh[threadIdx.x] += sh[threadIdx.x + q];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = (float)sh[0];
}

__global__ void k_adam(size_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_bf16(size_t n, const float *src, __nv_bfloat16 *dst) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

inline unsigned blocks(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace
}  // namespace cb2

using namespace cb2;

// ---------------------------------------------------------------------------
// the network
struct cb2_mlp {
  int F = 0, H = 0, O = 0;
  size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0, np = 0;
  float *master = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16 *w = nullptr;   // bfloat16 copy of every parameter (the products use W1, W2, W3)
  int t = 0;
  size_t cap = 0;               // rows of the work buffers
  float *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Yp = nullptr, *dY = nullptr;
  float *dH = nullptr, *dZ = nullptr;
  double *part = nullptr;       // loss partial sums
  int *status = nullptr;        // device status word of the GEMMs (bit 2: a wait ran out)
  size_t part_cap = 0;
  cudaStream_t stream = nullptr;
};

namespace cb2 {
namespace {

int mlp_reserve(cb2_mlp *n, size_t rows) {
  if (rows <= n->cap) return 0;
  float **bufs[8] = {&n->Z1, &n->H1, &n->Z2, &n->H2, &n->Yp, &n->dY, &n->dH, &n->dZ};
  const size_t width[8] = {(size_t)n->H, (size_t)n->H, (size_t)n->H, (size_t)n->H, (size_t)n->O, (size_t)n->O,
                           (size_t)n->H, (size_t)n->H};
  for (int q = 0; q < 8; q++) {
    if (*bufs[q]) cudaFree(*bufs[q]);
    *bufs[q] = nullptr;
    CB2_CUDA(cudaMalloc(bufs[q], rows * width[q] * sizeof(float)));
  }
  const size_t pc = blocks(rows * n->O) + 1;
  if (n->part) cudaFree(n->part);
  n->part = nullptr;
  CB2_CUDA(cudaMalloc(&n->part, pc * sizeof(double)));
  n->part_cap = pc;
  n->cap = rows;
  return 0;
}

// C = opA opB on the tensor cores (k_tc_gemm).  split_k: K is cut into
// chunks so that the grid covers the SMs about twice, C is cleared and the
// chunks' partial products are added with atomics.
template <typename TAT, typename TBT, bool TA, bool TB>
void gemm(cudaStream_t st, int *status, int M, int N, int K, const TAT *A, int lda, const TBT *B, int ldb, float *C,
          int ldc, bool split_k) {
  constexpr int NA = Terms<TAT>::n, NBT = Terms<TBT>::n;
  const int NT = std::min(256, ((N + 15) / 16) * 16);
  uint32_t cols = 64;
  while ((int)cols < NT) cols *= 2;
  const uint32_t stage = ((NA * GA_BYTES + NBT * (uint32_t)NT * GK * 2) + 1023u) & ~1023u;
  const size_t smem = 2 * (size_t)stage + 64 + 1024;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_tc_gemm<TAT, TBT, TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         2 * (2 * GA_BYTES + 2 * 256 * GK * 2) + 64 + 1024);
    attr_set = true;
  }
  const int tiles = ((N + NT - 1) / NT) * ((M + 127) / 128);
  int kchunk = K, nz = 1;
  if (split_k) {
    nz = std::max(1, std::min((K + 255) / 256, (2 * 148 + tiles - 1) / tiles));
    kchunk = (((K + nz - 1) / nz) + GK - 1) / GK * GK;
    nz = (K + kchunk - 1) / kchunk;
    cudaMemsetAsync(C, 0, (size_t)M * ldc * sizeof(float), st);
  }
  dim3 grid((N + NT - 1) / NT, (M + 127) / 128, nz);
  k_tc_gemm<TAT, TBT, TA, TB><<<grid, 128, smem, st>>>(M, N, NT, K, A, lda, B, ldb, C, ldc, kchunk,
                                                        split_k ? 1 : 0, cols, status, kWaitNsGemm);
}

// forward pass of n rows of X (normalised features) into n->Yp, on stream st
int mlp_forward(cb2_mlp *nt, const float *X, size_t n, cudaStream_t st, int *status = nullptr) {
  int rc = mlp_reserve(nt, n);
  if (rc) return rc;
  if (!status) status = nt->status;
  const int F = nt->F, H = nt->H, O = nt->O;
  gemm<float, __nv_bfloat16, false, true>(st, status, (int)n, H, F, X, F, nt->w + nt->oW1, F, nt->Z1, H, false);
  k_bias_act<<<blocks(n * H), 256, 0, st>>>(n, H, nt->Z1, nt->master + nt->ob1, nt->H1, 1);
  gemm<float, __nv_bfloat16, false, true>(st, status, (int)n, H, H, nt->H1, H, nt->w + nt->oW2, H, nt->Z2, H,
                                          false);
  k_bias_act<<<blocks(n * H), 256, 0, st>>>(n, H, nt->Z2, nt->master + nt->ob2, nt->H2, 1);
  gemm<float, __nv_bfloat16, false, true>(st, status, (int)n, O, H, nt->H2, H, nt->w + nt->oW3, H, nt->Yp, O,
                                          false);
  k_bias_act<<<blocks(n * O), 256, 0, st>>>(n, O, nt->Yp, nt->master + nt->ob3, nt->Yp, 0);
  CB2_CUDA(cudaGetLastError());
  return 0;
}

// loss and gradients of the mean squared error over n rows (grad <- dL/dparams)
int mlp_backward(cb2_mlp *nt, const float *X, const float *T, size_t n, double *loss) {
  cudaStream_t st = nt->stream;
  int rc = mlp_forward(nt, X, n, st);
  if (rc) return rc;
  const int F = nt->F, H = nt->H, O = nt->O;
  const unsigned nb = blocks(n * O);
  k_mse<<<nb, 256, 0, st>>>(n, O, nt->Yp, T, nt->dY, nt->part);
  // layer 3
  gemm<float, float, true, false>(st, nt->status, O, H, (int)n, nt->dY, O, nt->H2, H, nt->grad + nt->oW3, H, true);
  k_colsum<<<O, 256, 0, st>>>(n, O, nt->dY, nt->grad + nt->ob3);
  gemm<float, __nv_bfloat16, false, false>(st, nt->status, (int)n, H, O, nt->dY, O, nt->w + nt->oW3, H, nt->dH, H, false);
  k_act_grad<<<blocks(n * H), 256, 0, st>>>(n * H, nt->Z2, nt->dH, nt->dZ);
  // layer 2
  gemm<float, float, true, false>(st, nt->status, H, H, (int)n, nt->dZ, H, nt->H1, H, nt->grad + nt->oW2, H, true);
  k_colsum<<<H, 256, 0, st>>>(n, H, nt->dZ, nt->grad + nt->ob2);
  gemm<float, __nv_bfloat16, false, false>(st, nt->status, (int)n, H, H, nt->dZ, H, nt->w + nt->oW2, H, nt->dH, H, false);
  k_act_grad<<<blocks(n * H), 256, 0, st>>>(n * H, nt->Z1, nt->dH, nt->dZ);
  // layer 1
  gemm<float, float, true, false>(st, nt->status, H, F, (int)n, nt->dZ, H, X, F, nt->grad + nt->oW1, F, true);
  k_colsum<<<H, 256, 0, st>>>(n, H, nt->dZ, nt->grad + nt->ob1);
  CB2_CUDA(cudaGetLastError());
  if (loss) {
    std::vector<double> hp(nb);
    CB2_CUDA(cudaMemcpyAsync(hp.data(), nt->part, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CB2_CUDA(cudaStreamSynchronize(st));
    double s = 0.0;
    for (double x : hp) s += x;
    *loss = s / ((double)n * O);
  }
  return 0;
}

}  // namespace
}  // namespace cb2

// closure state of a context
struct ClosureState {
  cb2_mlp *net = nullptr;
  float *norm = nullptr;     // [nr][16 mean], [nr][16 1/std], [nr][5 out scale]
  float *X = nullptr, *Xn = nullptr;
  size_t rows = 0;
};

namespace cb2 {
// called by the time step after the explicit nonlinear terms are formed
int closure_apply(Ctx &c) {
  ClosureState *cs = static_cast<ClosureState *>(c.closure);
  if (!cs || !cs->net) return 0;
  const size_t n = cs->rows;
  k_features<<<blocks(n), 256, 0, c.stream>>>(c.nr, c.jmax, c.L, c.d_jl, c.d_jm, c.d_r, c.h_r[c.kin],
                                              c.h_r[c.kout], c.d_f, c.fsize(), feat_slots(), cs->X);
  const size_t nn = (size_t)c.nr * NF;
  k_normalise<<<blocks(n * NF), 256, 0, c.stream>>>(n, c.jmax, cs->X, cs->norm, cs->norm + nn, cs->Xn);
  int rc = mlp_forward(cs->net, cs->Xn, n, c.stream, c.d_status);
  if (rc) return rc;
  k_add_tendency<<<blocks(n), 256, 0, c.stream>>>(n, c.nr, c.jmax, cs->net->Yp, cs->norm + 2 * nn, c.d_f, c.fsize(),
                                                  out_slots());
  return 0;
}

void closure_free(Ctx &c) {
  ClosureState *cs = static_cast<ClosureState *>(c.closure);
  if (!cs) return;
  if (cs->norm) cudaFree(cs->norm);
  if (cs->X) cudaFree(cs->X);
  if (cs->Xn) cudaFree(cs->Xn);
  delete cs;
  c.closure = nullptr;
}
}  // namespace cb2

extern "C" {

int cb2_mlp_create(int nin, int nhid, int nout, unsigned seed, cb2_mlp **out) {
  if (!out || nin <= 0 || nhid <= 0 || nout <= 0) { set_error("cb2_mlp_create: bad argument"); return CB2_ERR_ARG; }
  *out = nullptr;
  cb2_mlp *n = new cb2_mlp();
  n->F = nin; n->H = nhid; n->O = nout;
  n->oW1 = 0; n->ob1 = n->oW1 + (size_t)nhid * nin; n->oW2 = n->ob1 + nhid;
  n->ob2 = n->oW2 + (size_t)nhid * nhid; n->oW3 = n->ob2 + nhid; n->ob3 = n->oW3 + (size_t)nout * nhid;
  n->np = n->ob3 + nout;
  // He-style uniform initialisation, biases zero (host generator: splitmix64)
  std::vector<float> p(n->np, 0.0f);
  unsigned long long s = 0x9E3779B97F4A7C15ULL ^ ((unsigned long long)seed << 21);
  auto uni = [&]() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](size_t off, size_t cnt, int fan_in) {
    const double a = std::sqrt(3.0 / fan_in);
    for (size_t q = 0; q < cnt; q++) p[off + q] = (float)((2.0 * uni() - 1.0) * a);
  };
  fill(n->oW1, (size_t)nhid * nin, nin);
  fill(n->oW2, (size_t)nhid * nhid, nhid);
  fill(n->oW3, (size_t)nout * nhid, nhid);
  auto fail = [&](int rc) { cb2_mlp_destroy(n); return rc; };
  if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&n->master, n->np * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->grad, n->np * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->m, n->np * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->v, n->np * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->w, n->np * sizeof(__nv_bfloat16)) != cudaSuccess ||
      cudaMalloc(&n->status, sizeof(int)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cb2_mlp_create"));
  cudaMemcpy(n->master, p.data(), n->np * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(n->grad, 0, n->np * sizeof(float));
  cudaMemset(n->m, 0, n->np * sizeof(float));
  cudaMemset(n->v, 0, n->np * sizeof(float));
  cudaMemset(n->status, 0, sizeof(int));
  k_to_bf16<<<blocks(n->np), 256, 0, n->stream>>>(n->np, n->master, n->w);
  if (cudaStreamSynchronize(n->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "cb2_mlp_create"));
  *out = n;
  return 0;
}

int cb2_mlp_destroy(cb2_mlp *n) {
  if (!n) return 0;
  if (n->stream) cudaStreamSynchronize(n->stream);
  void *ptrs[] = {n->master, n->grad, n->m, n->v, n->w, n->Z1, n->H1, n->Z2, n->H2, n->Yp, n->dY, n->dH, n->dZ,
                  n->part, n->status};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
  return 0;
}

int cb2_mlp_num_params(const cb2_mlp *n) { return n ? (int)n->np : -1; }

// float32 master parameters: W1 [H][F], b1 [H], W2 [H][H], b2 [H], W3 [O][H], b3 [O]
int cb2_mlp_get_params(cb2_mlp *n, float *host) {
  if (!n || !host) return CB2_ERR_ARG;
  CB2_CUDA(cudaMemcpy(host, n->master, n->np * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int cb2_mlp_set_params(cb2_mlp *n, const float *host) {
  if (!n || !host) return CB2_ERR_ARG;
  CB2_CUDA(cudaMemcpy(n->master, host, n->np * sizeof(float), cudaMemcpyHostToDevice));
  k_to_bf16<<<blocks(n->np), 256, 0, n->stream>>>(n->np, n->master, n->w);
  CB2_CUDA(cudaStreamSynchronize(n->stream));
  return 0;
}

// the GEMMs' status word after the stream has drained: a pipeline wait
// that ran out is reported (and the word cleared)
static int mlp_status(cb2_mlp *n) {
  int st = 0;
  CB2_CUDA(cudaMemcpyAsync(&st, n->status, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
  CB2_CUDA(cudaStreamSynchronize(n->stream));
  if (st) {
    CB2_CUDA(cudaMemsetAsync(n->status, 0, sizeof(int), n->stream));
    set_error("closure network: a tensor-core pipeline wait ran out");
    return CB2_ERR_TIMEOUT;
  }
  return 0;
}

int cb2_mlp_forward(cb2_mlp *n, const float *dev_x, long long rows, float *dev_y) {
  if (!n || !dev_x || !dev_y || rows <= 0) return CB2_ERR_ARG;
  int rc = mlp_forward(n, dev_x, (size_t)rows, n->stream);
  if (rc) return rc;
  CB2_CUDA(cudaMemcpyAsync(dev_y, n->Yp, (size_t)rows * n->O * sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
  return mlp_status(n);
}

// mean squared error of rows x (normalised features) against t, and its
// gradient (kept for cb2_mlp_adam_step; copied to host_grad when not NULL)
int cb2_mlp_loss_grad(cb2_mlp *n, const float *dev_x, const float *dev_t, long long rows, double *loss,
                      float *host_grad) {
  if (!n || !dev_x || !dev_t || rows <= 0) return CB2_ERR_ARG;
  double l = 0.0;
  int rc = mlp_backward(n, dev_x, dev_t, (size_t)rows, &l);
  if (rc || (rc = mlp_status(n))) return rc;
  if (loss) *loss = l;
  if (host_grad) CB2_CUDA(cudaMemcpy(host_grad, n->grad, n->np * sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

int cb2_mlp_adam_step(cb2_mlp *n, float lr, float beta1, float beta2, float eps) {
  if (!n) return CB2_ERR_ARG;
  n->t += 1;
  const float c1 = 1.0f - std::pow(beta1, (float)n->t), c2 = 1.0f - std::pow(beta2, (float)n->t);
  k_adam<<<blocks(n->np), 256, 0, n->stream>>>(n->np, n->master, n->grad, n->m, n->v, lr, beta1, beta2, eps, c1, c2);
  k_to_bf16<<<blocks(n->np), 256, 0, n->stream>>>(n->np, n->master, n->w);
  CB2_CUDA(cudaGetLastError());
  return 0;
}

int cb2_mlp_sync(cb2_mlp *n) {
  if (!n) return CB2_ERR_ARG;
  return mlp_status(n);
}

// dst's 13 state fields (velocity, vorticity, magnetic field, current,
// temperature) := src's, truncated to dst's L and restricted to dst's
// radial points; then dst's derived fields and nonlinear terms are rebuilt
// (cb2_start).  dst's radial points must be every stride-th point of src's.
static int filter_check(const cb2_ctx *s, const cb2_ctx *d, int *stride) {
  if (!s || !d) { set_error("filter: null context"); return CB2_ERR_ARG; }
  if (d->L > s->L || d->device != s->device || (s->nr - 1) % (d->nr - 1) != 0) {
    set_error("filter: destination needs L <= source L, the same device and a radial grid whose points are "
              "a subset of the source's");
    return CB2_ERR_ARG;
  }
  *stride = (s->nr - 1) / (d->nr - 1);
  for (int k = 0; k < d->nr; k++)
    if (std::fabs(d->h_r[k] - s->h_r[k * *stride]) > 1e-12 * std::fabs(s->h_r[k * *stride])) {
      set_error("filter: radial points of the destination are not points of the source");
      return CB2_ERR_ARG;
    }
  return 0;
}

int cb2_filter_fields(cb2_ctx *src, cb2_ctx *dst) {
  int stride = 1, rc = filter_check(src, dst, &stride);
  if (rc) return rc;
  CB2_CUDA(cudaStreamSynchronize(src->stream));
  Slots16 ss = feat_slots();
  k_filter<<<blocks((size_t)dst->nr * dst->jmax), 256, 0, dst->stream>>>(
      dst->nr, dst->jmax, src->jmax, src->L, stride, dst->d_jl, dst->d_jm, src->d_moff, src->d_f, src->fsize(),
      dst->d_f, dst->fsize(), ss, ss, 13, 0);
  CB2_CUDA(cudaGetLastError());
  return cb2_start(dst);
}

// src's five explicit nonlinear terms (curl of forces S, T; induction S, T;
// heat advection), filtered onto dst's shape: dev_out = 5 x nr x jmax
// (dst's device order, float64)
int cb2_filter_terms(cb2_ctx *src, cb2_ctx *dst, double *dev_out) {
  int stride = 1, rc = filter_check(src, dst, &stride);
  if (rc) return rc;
  if (!dev_out) return CB2_ERR_ARG;
  CB2_CUDA(cudaStreamSynchronize(src->stream));
  Slots16 so = out_slots();
  k_filter<<<blocks((size_t)dst->nr * dst->jmax), 256, 0, dst->stream>>>(
      dst->nr, dst->jmax, src->jmax, src->L, stride, dst->d_jl, dst->d_jm, src->d_moff, src->d_f, src->fsize(),
      dev_out, dst->fsize(), so, so, NO, 1);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(dst->stream));
  return 0;
}

// raw features of ctx's state: dev_x = (nr * jmax) x 16 float32
int cb2_closure_features(cb2_ctx *c, float *dev_x) {
  if (!c || !dev_x) return CB2_ERR_ARG;
  const size_t n = c->fsize();
  k_features<<<blocks(n), 256, 0, c->stream>>>(c->nr, c->jmax, c->L, c->d_jl, c->d_jm, c->d_r, c->h_r[c->kin],
                                               c->h_r[c->kout], c->d_f, c->fsize(), feat_slots(), dev_x);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// targets: dev_y = (nr * jmax) x 5 float32 = dev_hi (cb2_filter_terms) minus
// ctx's own five nonlinear terms
int cb2_closure_targets(cb2_ctx *c, const double *dev_hi, float *dev_y) {
  if (!c || !dev_hi || !dev_y) return CB2_ERR_ARG;
  const size_t n = c->fsize();
  k_targets<<<blocks(n), 256, 0, c->stream>>>(n, dev_hi, c->d_f, c->fsize(), out_slots(), dev_y);
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// attach (net != NULL) or detach the closure: every step then adds
// MLP((features - mean[k]) / std[k]) * scale[k] to the five nonlinear terms
// at the interior radial levels k.  norm (host floats) = nr x 16 means,
// nr x 16 standard deviations, nr x 5 output scales.  The network must have
// 16 inputs and 5 outputs and outlive the attachment.
int cb2_closure_attach(cb2_ctx *c, cb2_mlp *net, const float *norm) {
  if (!c) return CB2_ERR_ARG;
  if (c->graph_exec) { set_error("cb2_closure_attach: the step graph is already captured"); return CB2_ERR_STATE; }
  closure_free(*c);
  if (!net) return 0;
  if (net->F != NF || net->O != NO || !norm) {
    set_error("cb2_closure_attach: the network needs 16 inputs and 5 outputs, and norm nr x 37 floats");
    return CB2_ERR_ARG;
  }
  ClosureState *cs = new ClosureState();
  c->closure = cs;
  cs->net = net;
  cs->rows = c->fsize();
  const size_t nn = (size_t)c->nr * NF;
  std::vector<float> hn(norm, norm + 2 * nn + (size_t)c->nr * NO);
  for (size_t q = 0; q < nn; q++) hn[nn + q] = hn[nn + q] > 0.0f ? 1.0f / hn[nn + q] : 1.0f;
  CB2_CUDA(cudaMalloc(&cs->norm, hn.size() * sizeof(float)));
  CB2_CUDA(cudaMemcpy(cs->norm, hn.data(), hn.size() * sizeof(float), cudaMemcpyHostToDevice));
  CB2_CUDA(cudaMalloc(&cs->X, cs->rows * NF * sizeof(float)));
  CB2_CUDA(cudaMalloc(&cs->Xn, cs->rows * NF * sizeof(float)));
  return mlp_reserve(net, cs->rows);
}

}  // extern "C"
