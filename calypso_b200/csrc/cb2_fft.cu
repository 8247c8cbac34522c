// cb2_fft.cu -- longitudinal transform fused with the grid-space products.
//
// One thread block per (theta, r) row: the Fourier coefficients of the 13
// backward components (u, w, B, J vectors and T) are turned into grid values
// in shared memory, the nonlinear products are formed pointwise, and the 12
// product components are transformed back -- the grid never goes to HBM.
// This replaces back_MHD_FFT_sel_from_recv, s_cal_nonlinear_sph_MHD and
// fwd_MHD_FFT_sel_from_recv of the reference (MHD_src/sph_MHD/
// MHD_FFT_selector.F90:185-249, cal_nonlinear_sph_MHD.f90:35-84) and the
// rtm <-> rtp transposes around them.
//
// Normalisation (t_MHD_multi_FFTW.F90:220-355):
//   f(phi_p) = a_0 + sum_{m=1..L} (a_m cos m phi_p + b_m sin m phi_p),
//   a_0 = (1/N) sum f, a_m = (2/N) sum f cos, b_m = (2/N) sum f sin.
// Two real rows share one complex FFT (x + i y).  The complex FFT is a
// shared-memory Stockham autosort transform with radix 3, 4 and 2 stages,
// N = 3^a 2^b.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

template <typename T> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };

template <typename T2>
__device__ inline T2 cmul(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// Two real rows x, y share one complex transform z = x + i y.  The rounding
// error of a transform is relative to the larger row, so a row far below its
// partner would carry the partner's error.  Where the rows of a pair can be
// of any size -- the float64 step kernel (parity with the oracle for any
// field sizes), the generic float32 kernel and the standalone transforms of
// caller-given components -- the second row is multiplied by 2^(ex - ey),
// ex and ey the exponents of the two rows' largest magnitudes (passed as
// the bit patterns of non-negative floats), which puts both rows at the
// same size; the factor is exact and is undone after the transform (1 when
// either row is zero or subnormal).  The float32 four-step and Stockham step
// kernels pair rows of related size (components of one field, or a field
// and its curl) and do without: on the L255 bench state the scaling changed
// neither the per-term errors nor the energy drift and cost 14 % of the
// kernel's time.
__device__ __forceinline__ int pair_exp(unsigned mx_bits, unsigned my_bits) {
  const int ex = (int)(mx_bits >> 23), ey = (int)(my_bits >> 23);
  if (ex == 0 || ey == 0) return 0;
  return max(-120, min(120, ex - ey));
}
__device__ __forceinline__ float pow2i(int e) { return __int_as_float((127 + e) << 23); }
__device__ __forceinline__ unsigned abs_bits(float x) { return __float_as_uint(x) & 0x7FFFFFFFu; }

// the same for either precision: magnitudes as ordered bit patterns and the
// power-of-two factor of the second row (inverse when `inv`)
template <typename T> struct PairBits;
template <> struct PairBits<float> {
  using U = unsigned;
  __device__ static U abs_bits(float x) { return __float_as_uint(x) & 0x7FFFFFFFu; }
  __device__ static float factor(U mx, U my, bool inv) {
    const int e = pair_exp(mx, my);
    return pow2i(inv ? -e : e);
  }
};
template <> struct PairBits<double> {
  using U = unsigned long long;
  __device__ static U abs_bits(double x) { return (U)__double_as_longlong(x) & 0x7FFFFFFFFFFFFFFFull; }
  __device__ static double factor(U mx, U my, bool inv) {
    const int ex = (int)(mx >> 52), ey = (int)(my >> 52);
    if (ex == 0 || ey == 0) return 1.0;
    const int e = max(-1000, min(1000, ex - ey));
    return __longlong_as_double((long long)(1023 + (inv ? -e : e)) << 52);
  }
};

struct FFTPlan {
  int n, nst;
  int rad[24];
};

// one Stockham stage set; returns the buffer that holds the result
template <typename T, typename T2>
__device__ T2 *block_fft(T2 *x, T2 *y, const FFTPlan &pl, const T2 *tw, int sign) {
  const int N = pl.n;
  int Ns = 1;
  const T s32 = (T)(0.5 * sqrt(3.0));
  for (int st = 0; st < pl.nst; st++) {
    const int R = pl.rad[st];
    const int nb = N / R;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
      int k = j % Ns;
      T2 v[4];
      for (int r = 0; r < R; r++) {
        T2 a = x[j + r * nb];
        if (r > 0 && k > 0) {
          int e = (r * k * (N / (Ns * R))) % N;
          T2 w = tw[e];
          if (sign > 0) w.y = -w.y;
          a = cmul(a, w);
        }
        v[r] = a;
      }
      T2 o[4];
      if (R == 2) {
        o[0].x = v[0].x + v[1].x; o[0].y = v[0].y + v[1].y;
        o[1].x = v[0].x - v[1].x; o[1].y = v[0].y - v[1].y;
      } else if (R == 4) {
        T2 a0, a1, a2, a3;
        a0.x = v[0].x + v[2].x; a0.y = v[0].y + v[2].y;
        a1.x = v[0].x - v[2].x; a1.y = v[0].y - v[2].y;
        a2.x = v[1].x + v[3].x; a2.y = v[1].y + v[3].y;
        T dx = v[1].x - v[3].x, dy = v[1].y - v[3].y;
        // forward (sign < 0): (v1 - v3) * (-i); inverse: * (+i)
        if (sign < 0) { a3.x = dy; a3.y = -dx; } else { a3.x = -dy; a3.y = dx; }
        o[0].x = a0.x + a2.x; o[0].y = a0.y + a2.y;
        o[1].x = a1.x + a3.x; o[1].y = a1.y + a3.y;
        o[2].x = a0.x - a2.x; o[2].y = a0.y - a2.y;
        o[3].x = a1.x - a3.x; o[3].y = a1.y - a3.y;
      } else {  // R == 3
        T2 t1, t2, t3;
        t1.x = v[1].x + v[2].x; t1.y = v[1].y + v[2].y;
        t2.x = v[0].x - (T)0.5 * t1.x; t2.y = v[0].y - (T)0.5 * t1.y;
        T dx = v[1].x - v[2].x, dy = v[1].y - v[2].y;
        // forward: (v1 - v2) * (-i sqrt3/2); inverse: * (+i sqrt3/2)
        if (sign < 0) { t3.x = s32 * dy; t3.y = -s32 * dx; } else { t3.x = -s32 * dy; t3.y = s32 * dx; }
        o[0].x = v[0].x + t1.x; o[0].y = v[0].y + t1.y;
        o[1].x = t2.x + t3.x; o[1].y = t2.y + t3.y;
        o[2].x = t2.x - t3.x; o[2].y = t2.y - t3.y;
      }
      int d = (j / Ns) * Ns * R + k;
      for (int r = 0; r < R; r++) y[d + r * Ns] = o[r];
    }
    __syncthreads();
    T2 *t = x; x = y; y = t;
    Ns *= R;
  }
  return x;
}

// spectrum of two real rows -> z = x + i y (Z = X + i Y, X Hermitian)
template <typename T, typename T2>
__device__ void load_pair(T2 *Z, int N, int L, const T *f0, const T *f1) {
  for (int q = threadIdx.x; q < N; q += blockDim.x) Z[q] = T2{0, 0};
  __syncthreads();
  int mmax = min(L, (N + 1) / 2 - 1);
  for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
    T a0 = f0[2 * m], b0 = (m > 0) ? f0[2 * m + 1] : (T)0;
    T a1 = f1 ? f1[2 * m] : (T)0, b1 = (f1 && m > 0) ? f1[2 * m + 1] : (T)0;
    if (m == 0) {
      Z[0] = T2{a0, a1};
    } else {
      T xr = (T)0.5 * a0, xi = (T)-0.5 * b0, yr = (T)0.5 * a1, yi = (T)-0.5 * b1;
      Z[m] = T2{xr - yi, xi + yr};
      Z[N - m] = T2{xr + yi, -xi + yr};
    }
  }
  __syncthreads();
}

// FFT of z = x + i y -> (a_m, b_m) of both rows, m = 0..L
template <typename T, typename T2>
__device__ void store_pair(const T2 *Z, int N, int L, T *f0, T *f1) {
  T an = (T)(1.0 / (double)N);
  for (int m = threadIdx.x; m <= L; m += blockDim.x) {
    if (m == 0) {
      f0[0] = an * Z[0].x; f0[1] = 0;
      if (f1) { f1[0] = an * Z[0].y; f1[1] = 0; }
    } else if (m < N) {
      T2 zk = Z[m % N], zn = Z[(N - m) % N];
      T xr = (T)0.5 * (zk.x + zn.x), xi = (T)0.5 * (zk.y - zn.y);
      T yr = (T)0.5 * (zk.y + zn.y), yi = (T)-0.5 * (zk.x - zn.x);
      f0[2 * m] = (T)2 * an * xr; f0[2 * m + 1] = (T)-2 * an * xi;
      if (f1) { f1[2 * m] = (T)2 * an * yr; f1[2 * m + 1] = (T)-2 * an * yi; }
    }
  }
}

struct ProdCoef {
  double cv, cl, ci, ct;
};

// Stockham stages over nf independent FFTs held in x[f*N + n]; all FFTs of
// the row advance together so each stage costs one barrier
template <typename T, typename T2>
__device__ T2 *batch_fft(T2 *x, T2 *y, int nf, const FFTPlan &pl, const T2 *__restrict__ tw, int sign) {
  const int N = pl.n;
  int Ns = 1;
  const T s32 = (T)(0.5 * sqrt(3.0));
  for (int st = 0; st < pl.nst; st++) {
    const int R = pl.rad[st];
    const int nb = N / R, tstride = N / (Ns * R);
    for (int idx = threadIdx.x; idx < nf * nb; idx += blockDim.x) {
      int f = idx / nb, j = idx - f * nb;
      int k = j % Ns;
      const T2 *xf = x + f * N;
      T2 v[4];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        if (r < R) {
          T2 a = xf[j + r * nb];
          if (r > 0 && k > 0) {
            T2 w = tw[r * k * tstride];
            if (sign > 0) w.y = -w.y;
            a = cmul(a, w);
          }
          v[r] = a;
        }
      }
      T2 o[4];
      if (R == 4) {
        T2 a0, a1, a2, a3;
        a0.x = v[0].x + v[2].x; a0.y = v[0].y + v[2].y;
        a1.x = v[0].x - v[2].x; a1.y = v[0].y - v[2].y;
        a2.x = v[1].x + v[3].x; a2.y = v[1].y + v[3].y;
        T dx = v[1].x - v[3].x, dy = v[1].y - v[3].y;
        if (sign < 0) { a3.x = dy; a3.y = -dx; } else { a3.x = -dy; a3.y = dx; }
        o[0].x = a0.x + a2.x; o[0].y = a0.y + a2.y;
        o[1].x = a1.x + a3.x; o[1].y = a1.y + a3.y;
        o[2].x = a0.x - a2.x; o[2].y = a0.y - a2.y;
        o[3].x = a1.x - a3.x; o[3].y = a1.y - a3.y;
      } else if (R == 2) {
        o[0].x = v[0].x + v[1].x; o[0].y = v[0].y + v[1].y;
        o[1].x = v[0].x - v[1].x; o[1].y = v[0].y - v[1].y;
      } else {
        T2 t1, t2, t3;
        t1.x = v[1].x + v[2].x; t1.y = v[1].y + v[2].y;
        t2.x = v[0].x - (T)0.5 * t1.x; t2.y = v[0].y - (T)0.5 * t1.y;
        T dx = v[1].x - v[2].x, dy = v[1].y - v[2].y;
        if (sign < 0) { t3.x = s32 * dy; t3.y = -s32 * dx; } else { t3.x = -s32 * dy; t3.y = s32 * dx; }
        o[0].x = v[0].x + t1.x; o[0].y = v[0].y + t1.y;
        o[1].x = t2.x + t3.x; o[1].y = t2.y + t3.y;
        o[2].x = t2.x - t3.x; o[2].y = t2.y - t3.y;
      }
      T2 *yf = y + f * N;
      int d = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (r < R) yf[d + r * Ns] = o[r];
    }
    __syncthreads();
    T2 *t = x; x = y; y = t;
    Ns *= R;
  }
  return x;
}

// one block per (theta, r) row: 13 components -> grid -> 12 products -> spectra
template <typename T>
__global__ void __launch_bounds__(512)
k_fft_products(FFTPlan pl, int L, int NS, const T *__restrict__ four, T *__restrict__ four2,
               const typename C2<T>::t *__restrict__ tw, ProdCoef pc) {
  using T2 = typename C2<T>::t;
  using U = typename PairBits<T>::U;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n;
  T2 *A = reinterpret_cast<T2 *>(smraw);    // 7 x N
  T2 *B = A + 7 * N;                         // 7 x N
  U *cmx = reinterpret_cast<U *>(B + 7 * N); // [13] input maxima, [13..24] product maxima (bits)
  const size_t row = blockIdx.x;
  const T *fin = four + row * 13 * NS;
  T *fout = four2 + row * 12 * NS;
  const int mmax = min(L, (N + 1) / 2 - 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  if (threadIdx.x < 25) cmx[threadIdx.x] = 0;
  __syncthreads();
  // pair scaling (pair_exp): the largest coefficient of each component
  for (int c = warp; c < 13; c += nwarp) {
    U mx = 0;
    for (int q = lane; q < 2 * (mmax + 1); q += 32) mx = max(mx, PairBits<T>::abs_bits(fin[(size_t)c * NS + q]));
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, (U)__shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) cmx[c] = mx;
  }
  __syncthreads();
  // Hermitian spectra of the 7 pairs (z = x + i y), the second row scaled
  for (int idx = threadIdx.x; idx < 7 * N; idx += blockDim.x) {
    int p = idx / N, n = idx - p * N;
    const T *f0 = fin + (size_t)(2 * p) * NS;
    const T *f1 = (2 * p + 1 < 13) ? fin + (size_t)(2 * p + 1) * NS : nullptr;
    const T sy = f1 ? PairBits<T>::factor(cmx[2 * p], cmx[2 * p + 1], false) : (T)1;
    T2 z = T2{0, 0};
    if (n == 0) {
      z = T2{f0[0], f1 ? f1[0] * sy : (T)0};
    } else {
      int m = (n <= mmax) ? n : ((N - n <= mmax) ? N - n : -1);
      if (m > 0) {
        T a0 = f0[2 * m], b0 = f0[2 * m + 1];
        T a1 = f1 ? f1[2 * m] * sy : (T)0, b1 = f1 ? f1[2 * m + 1] * sy : (T)0;
        T xr = (T)0.5 * a0, xi = (T)-0.5 * b0, yr = (T)0.5 * a1, yi = (T)-0.5 * b1;
        z = (m == n) ? T2{xr - yi, xi + yr} : T2{xr + yi, -xi + yr};
      }
    }
    A[idx] = z;
  }
  __syncthreads();
  T2 *g = batch_fft<T, T2>(A, B, 7, pl, tw, +1);
  T2 *h = (g == A) ? B : A;
  const T cv = (T)pc.cv, cl = (T)pc.cl, ci = (T)pc.ci, ct = (T)pc.ct;
  T iy[6];
#pragma unroll
  for (int p = 0; p < 6; p++) iy[p] = PairBits<T>::factor(cmx[2 * p], cmx[2 * p + 1], true);
  U hm[12];
#pragma unroll
  for (int c = 0; c < 12; c++) hm[c] = 0;
  for (int q = threadIdx.x; q < N; q += blockDim.x) {
    T2 p0 = g[0 * N + q], p1 = g[1 * N + q], p2 = g[2 * N + q], p3 = g[3 * N + q];
    T2 p4 = g[4 * N + q], p5 = g[5 * N + q], p6 = g[6 * N + q];
    T ur = p0.x, ut = p0.y * iy[0], up = p1.x, wr = p1.y * iy[1], wt = p2.x, wp = p2.y * iy[2];
    T br = p3.x, bt = p3.y * iy[3], bp = p4.x, jr = p4.y * iy[4], jt = p5.x, jp = p5.y * iy[5], tt = p6.x;
    const T2 hv[6] = {T2{(wt * up - wp * ut) * cv, (wp * ur - wr * up) * cv},
                      T2{(wr * ut - wt * ur) * cv, (jt * bp - jp * bt) * cl},
                      T2{(jp * br - jr * bp) * cl, (jr * bt - jt * br) * cl},
                      T2{(ut * bp - up * bt) * ci, (up * br - ur * bp) * ci},
                      T2{(ur * bt - ut * br) * ci, ur * tt * ct},
                      T2{ut * tt * ct, up * tt * ct}};
#pragma unroll
    for (int p = 0; p < 6; p++) {
      h[p * N + q] = hv[p];
      hm[2 * p] = max(hm[2 * p], PairBits<T>::abs_bits(hv[p].x));
      hm[2 * p + 1] = max(hm[2 * p + 1], PairBits<T>::abs_bits(hv[p].y));
    }
  }
  // row maxima of the 12 product rows: every lane of every warp takes part
#pragma unroll
  for (int c = 0; c < 12; c++) {
    U v = hm[c];
    for (int o = 16; o > 0; o >>= 1) v = max(v, (U)__shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) atomicMax(cmx + 13 + c, v);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 6 * N; idx += blockDim.x) {
    const int p = idx / N;
    h[idx].y *= PairBits<T>::factor(cmx[13 + 2 * p], cmx[14 + 2 * p], false);
  }
  __syncthreads();
  T2 *zf = batch_fft<T, T2>(h, g, 6, pl, tw, -1);
  const T an = (T)(1.0 / (double)N);
  for (int idx = threadIdx.x; idx < 6 * (L + 1); idx += blockDim.x) {
    int p = idx / (L + 1), m = idx - p * (L + 1);
    T *f0 = fout + (size_t)(2 * p) * NS, *f1 = fout + (size_t)(2 * p + 1) * NS;
    const T2 *Z = zf + p * N;
    const T ay = an * PairBits<T>::factor(cmx[13 + 2 * p], cmx[14 + 2 * p], true);
    if (m == 0) {
      f0[0] = an * Z[0].x; f0[1] = 0;
      f1[0] = ay * Z[0].y; f1[1] = 0;
    } else {
      T2 zk = Z[m % N], zn = Z[(N - m) % N];
      T xr = (T)0.5 * (zk.x + zn.x), xi = (T)0.5 * (zk.y - zn.y);
      T yr = (T)0.5 * (zk.y + zn.y), yi = (T)-0.5 * (zk.x - zn.x);
      f0[2 * m] = (T)2 * an * xr; f0[2 * m + 1] = (T)-2 * an * xi;
      f1[2 * m] = (T)2 * ay * yr; f1[2 * m + 1] = (T)-2 * ay * yi;
    }
  }
}

// Fourier rows -> grid (float64), for the standalone transform API
template <typename T>
__global__ void __launch_bounds__(256)
k_fft_to_grid(FFTPlan pl, int L, int NS, int nc, int nr, int nth, const T *four, double *grid,
              const typename C2<T>::t *tw) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n;
  T2 *Z0 = reinterpret_cast<T2 *>(smraw), *Z1 = Z0 + N;
  const size_t row = blockIdx.x;
  const int th = (int)(row / nr), k = (int)(row % nr);
  const T *fin = four + row * nc * NS;
  for (int c = 0; c < nc; c += 2) {
    load_pair<T, T2>(Z0, N, L, fin + (size_t)c * NS, (c + 1 < nc) ? fin + (size_t)(c + 1) * NS : nullptr);
    T2 *z = block_fft<T, T2>(Z0, Z1, pl, tw, +1);
    for (int q = threadIdx.x; q < N; q += blockDim.x) {
      grid[(((size_t)c * nr + k) * nth + th) * N + q] = (double)z[q].x;
      if (c + 1 < nc) grid[(((size_t)(c + 1) * nr + k) * nth + th) * N + q] = (double)z[q].y;
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_grid_to_fft(FFTPlan pl, int L, int NS, int nc, int nr, int nth, const double *grid, T *four,
              const typename C2<T>::t *tw) {
  using T2 = typename C2<T>::t;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n;
  T2 *Z0 = reinterpret_cast<T2 *>(smraw), *Z1 = Z0 + N;
  const size_t row = blockIdx.x;
  const int th = (int)(row / nr), k = (int)(row % nr);
  T *fout = four + row * nc * NS;
  for (int c = 0; c < nc; c += 2) {
    for (int q = threadIdx.x; q < N; q += blockDim.x) {
      T x = (T)grid[(((size_t)c * nr + k) * nth + th) * N + q];
      T y = (c + 1 < nc) ? (T)grid[(((size_t)(c + 1) * nr + k) * nth + th) * N + q] : (T)0;
      Z0[q] = T2{x, y};
    }
    __syncthreads();
    T2 *z = block_fft<T, T2>(Z0, Z1, pl, tw, -1);
    store_pair<T, T2>(z, N, L, fout + (size_t)c * NS, (c + 1 < nc) ? fout + (size_t)(c + 1) * NS : nullptr);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Mixed-precision path: the same fused transform over the order-major
// Fourier layout (MLayout).  Input 4 vectors (u, w, B, J) + 1 scalar (T),
// output 4 vectors (w x u, J x B, u x B, u T).  At one (theta, k) the 26
// input floats of an order m are one run of 10 (P block) and one of 16
// (D block); threads take consecutive elements of a run, the values are
// staged in shared memory [component][s][m], and the Hermitian rows are
// built from there.  Output is written the same way, one run per m.
__device__ inline void m_comp_of_in(int j, int &c, int &s) {
  // P block (k, field, s): fields 0..3 = r of u, w, B, J; 4 = T
  if (j < 10) { const int f = j >> 1; s = j & 1; c = (f < 4) ? 3 * f : 12; return; }
  // D block (k, vector, {theta s0, theta s1, phi s0, phi s1})
  const int jd = j - 10, v = jd >> 2, q = jd & 3;
  c = 3 * v + 1 + (q >> 1); s = q & 1;
}

__device__ inline void m_comp_of_out(int j, int &c, int &s) {
  if (j < 8) { s = j & 1; c = 3 * (j >> 1); return; }
  const int jd = j - 8, v = jd >> 2, q = jd & 3;
  c = 3 * v + 1 + (q >> 1); s = q & 1;
}

__global__ void __launch_bounds__(512)
k_fft_products_m(FFTPlan pl, int L, MLayout fin, MLayout fout, const float2 *__restrict__ tw, ProdCoef pc) {
  using T = float;
  using T2 = float2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n;
  T2 *A = reinterpret_cast<T2 *>(smraw);    // 7 x N
  T2 *B = A + 7 * N;                         // 7 x N (first used as the staging buffer)
  T *S = reinterpret_cast<T *>(B);           // [c * 2 + s][m], 26 x (L+1)
  float *SC = reinterpret_cast<float *>(B + 7 * N);        // pair factors [7], inverses [8..14]
  unsigned *FMX = reinterpret_cast<unsigned *>(SC + 16);   // forward row maxima [12]
  const int th = blockIdx.x / fin.nr, k = blockIdx.x % fin.nr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int M1 = L + 1;
  if (threadIdx.x < 12) FMX[threadIdx.x] = 0u;
  const float *Pin = fin.P + (size_t)th * fin.sP() + (size_t)k * 10;
  const float *Din = fin.D + (size_t)th * fin.sD() + (size_t)k * 16;
  const size_t mstP = (size_t)fin.nth * fin.sP(), mstD = (size_t)fin.nth * fin.sD();
  for (int idx = threadIdx.x; idx < 26 * M1; idx += blockDim.x) {
    const int m = idx / 26, j = idx - 26 * m;
    int c, s;
    m_comp_of_in(j, c, s);
    S[(c * 2 + s) * M1 + m] = (j < 10) ? Pin[m * mstP + j] : Din[m * mstD + (j - 10)];
  }
  __syncthreads();
  // pair scaling (pair_exp) of the 6 full pairs; pair 6 (T alone) keeps 1
  for (int p = warp; p < 7; p += nwarp) {
    unsigned mx = 0u, my = 0u;
    if (p < 6)
      for (int m = lane; m < M1; m += 32) {
        mx = max(mx, max(abs_bits(S[(4 * p) * M1 + m]), abs_bits(S[(4 * p + 1) * M1 + m])));
        my = max(my, max(abs_bits(S[(4 * p + 2) * M1 + m]), abs_bits(S[(4 * p + 3) * M1 + m])));
      }
    mx = __reduce_max_sync(0xffffffffu, mx);
    my = __reduce_max_sync(0xffffffffu, my);
    const int e = pair_exp(mx, my);
    if (lane == 0) { SC[p] = pow2i(e); SC[8 + p] = pow2i(-e); }
  }
  __syncthreads();
  const int mmax = min(L, (N + 1) / 2 - 1);
  for (int idx = threadIdx.x; idx < 7 * N; idx += blockDim.x) {
    const int p = idx / N, n = idx - p * N;
    const int c0 = 2 * p, c1 = 2 * p + 1;
    const bool has1 = c1 < 13;
    const T sy = SC[p];
    T2 z = T2{0, 0};
    if (n == 0) {
      z = T2{S[(c0 * 2) * M1], has1 ? S[(c1 * 2) * M1] * sy : (T)0};
    } else {
      const int m = (n <= mmax) ? n : ((N - n <= mmax) ? N - n : -1);
      if (m > 0) {
        const T a0 = S[(c0 * 2) * M1 + m], b0 = S[(c0 * 2 + 1) * M1 + m];
        const T a1 = has1 ? S[(c1 * 2) * M1 + m] * sy : (T)0, b1 = has1 ? S[(c1 * 2 + 1) * M1 + m] * sy : (T)0;
        const T xr = (T)0.5 * a0, xi = (T)-0.5 * b0, yr = (T)0.5 * a1, yi = (T)-0.5 * b1;
        z = (m == n) ? T2{xr - yi, xi + yr} : T2{xr + yi, -xi + yr};
      }
    }
    A[idx] = z;
  }
  __syncthreads();
  T2 *g = batch_fft<T, T2>(A, B, 7, pl, tw, +1);
  T2 *hb = (g == A) ? B : A;
  const T cv = (T)pc.cv, cl = (T)pc.cl, ci = (T)pc.ci, ct = (T)pc.ct;
  {
    const T i0 = SC[8], i1 = SC[9], i2 = SC[10], i3 = SC[11], i4 = SC[12], i5 = SC[13];
    unsigned hm[12];
#pragma unroll
    for (int c = 0; c < 12; c++) hm[c] = 0u;
    for (int q = threadIdx.x; q < N; q += blockDim.x) {
      T2 p0 = g[0 * N + q], p1 = g[1 * N + q], p2 = g[2 * N + q], p3 = g[3 * N + q];
      T2 p4 = g[4 * N + q], p5 = g[5 * N + q], p6 = g[6 * N + q];
      T ur = p0.x, ut = p0.y * i0, up = p1.x, wr = p1.y * i1, wt = p2.x, wp = p2.y * i2;
      T br = p3.x, bt = p3.y * i3, bp = p4.x, jr = p4.y * i4, jt = p5.x, jp = p5.y * i5, tt = p6.x;
      const T2 h[6] = {T2{(wt * up - wp * ut) * cv, (wp * ur - wr * up) * cv},
                       T2{(wr * ut - wt * ur) * cv, (jt * bp - jp * bt) * cl},
                       T2{(jp * br - jr * bp) * cl, (jr * bt - jt * br) * cl},
                       T2{(ut * bp - up * bt) * ci, (up * br - ur * bp) * ci},
                       T2{(ur * bt - ut * br) * ci, ur * tt * ct},
                       T2{ut * tt * ct, up * tt * ct}};
#pragma unroll
      for (int p = 0; p < 6; p++) {
        hb[p * N + q] = h[p];
        hm[2 * p] = max(hm[2 * p], abs_bits(h[p].x));
        hm[2 * p + 1] = max(hm[2 * p + 1], abs_bits(h[p].y));
      }
    }
#pragma unroll
    for (int c = 0; c < 12; c++) {
      const unsigned r = __reduce_max_sync(0xffffffffu, hm[c]);
      if (lane == 0) atomicMax(FMX + c, r);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 6 * N; idx += blockDim.x) {
    const int p = idx / N;
    const int e = pair_exp(FMX[2 * p], FMX[2 * p + 1]);
    if (e != 0) hb[idx].y *= pow2i(e);
  }
  __syncthreads();
  const T2 *zf = batch_fft<T, T2>(hb, g, 6, pl, tw, -1);
  const T an = (T)(1.0 / (double)N);
  float *Pout = fout.P + (size_t)th * fout.sP() + (size_t)k * 8;
  float *Dout = fout.D + (size_t)th * fout.sD() + (size_t)k * 16;
  const size_t oP = (size_t)fout.nth * fout.sP(), oD = (size_t)fout.nth * fout.sD();
  for (int idx = threadIdx.x; idx < 24 * M1; idx += blockDim.x) {
    const int m = idx / 24, j = idx - 24 * m;
    int c, s;
    m_comp_of_out(j, c, s);
    const T2 *Z = zf + (c >> 1) * N;
    const bool isy = c & 1;
    const T a = isy ? an * pow2i(-pair_exp(FMX[c - 1], FMX[c])) : an;
    T v;
    if (m == 0) {
      v = (s == 0) ? a * (isy ? Z[0].y : Z[0].x) : (T)0;
    } else {
      const T2 zk = Z[m % N], zn = Z[(N - m) % N];
      if (!isy) v = (s == 0) ? (T)2 * a * (T)0.5 * (zk.x + zn.x) : (T)-2 * a * (T)0.5 * (zk.y - zn.y);
      else v = (s == 0) ? (T)2 * a * (T)0.5 * (zk.y + zn.y) : (T)2 * a * (T)0.5 * (zk.x - zn.x);
    }
    if (j < 8) Pout[m * oP + j] = v;
    else Dout[m * oD + (j - 8)] = v;
  }
}

// ---------------------------------------------------------------------------
// Compile-time FFT passes for N = 3 * 2^b (the zonal grids 96 .. 768 that
// the shells use): radix 3 first, then radix 16 while it divides, then the
// remaining 8, 4 or 2 (768 = 3 16 16: three passes).  Every butterfly is a
// register DFT; with N and the radices known at compile time every index
// division is by a constant.  The twiddles of stage st are one table
// w^(r k), r = 1..R-1, k = 0..NS-1, contiguous in k.  Rows in shared memory
// carry one pad element per 16 (index i -> i + i/16), which keeps the
// stride-NS writes of the radix-16 stages free of bank conflicts.
template <int N>
struct Plan3x2 {
  static constexpr int radix(int st) {
    if (st == 0) return 3;
    int n = N / 3;
    for (int q = 1; q < st; q++) n /= (n % 16 == 0) ? 16 : n;
    return (n % 16 == 0) ? 16 : n;
  }
  static constexpr int nst() {
    int n = N / 3, s = 1;
    while (n > 1) { n /= (n % 16 == 0) ? 16 : n; s++; }
    return s;
  }
  static constexpr int ns(int st) {   // product of the radices before stage st
    int p = 1;
    for (int q = 0; q < st; q++) p *= radix(q);
    return p;
  }
  static constexpr int off(int st) {
    int o = 0;
    for (int q = 0; q < st; q++) o += (radix(q) - 1) * ns(q);
    return o;
  }
  static constexpr int ntw() { return off(nst()); }
  static constexpr int NP = N + N / 16;   // padded row length
};

__host__ __device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

template <typename T2> struct ScalarOf;
template <> struct ScalarOf<float2> { using t = float; };
template <> struct ScalarOf<double2> { using t = double; };

template <typename T2>
__host__ __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return T2{a.x + b.x, a.y + b.y}; }
template <typename T2>
__host__ __device__ __forceinline__ T2 csub(T2 a, T2 b) { return T2{a.x - b.x, a.y - b.y}; }
// float32 pairs on sm_100: one packed float32x2 instruction for both lanes,
// each lane rounded as the scalar add (b (-1) + a is a - b exactly), so the
// results are those of the scalar forms
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return float2{a.x + b.x, a.y + b.y};
#endif
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(b, float2{-1.0f, -1.0f}, a);
#else
  return float2{a.x - b.x, a.y - b.y};
#endif
}
template <typename T2>
__host__ __device__ __forceinline__ T2 cmulf(T2 a, T2 b) {
  return T2{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// multiply by -i (forward) or +i (inverse)
template <int SIGN, typename T2>
__host__ __device__ __forceinline__ T2 rot90(T2 a) {
  return (SIGN < 0) ? T2{a.y, -a.x} : T2{-a.y, a.x};
}

// exp(SIGN 2 pi i q / 16) from exact values of the cosine at multiples of
// pi/8: cos(pi/8) = sqrt(2 + sqrt 2)/2, cos(pi/4) = sqrt(2)/2, sin(pi/8) =
// sqrt(2 - sqrt 2)/2
template <int SIGN, typename T2 = float2>
__host__ __device__ __forceinline__ T2 w16(int q) {
  using T = typename ScalarOf<T2>::t;
  constexpr T c1 = (T)0.92387953251128675613, c2 = (T)0.70710678118654752440, c3 = (T)0.38268343236508977173;
  const T cs[16] = {1, c1, c2, c3, 0, -c3, -c2, -c1, -1, -c1, -c2, -c3, 0, c3, c2, c1};
  const T sn[16] = {0, c3, c2, c1, 1, c1, c2, c3, 0, -c3, -c2, -c1, -1, -c1, -c2, -c3};
  return T2{cs[q & 15], (SIGN < 0) ? -sn[q & 15] : sn[q & 15]};
}

template <int SIGN, typename T2>
__host__ __device__ __forceinline__ void dft4(T2 &v0, T2 &v1, T2 &v2, T2 &v3) {
  const T2 a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = rot90<SIGN>(csub(v1, v3));
  v0 = cadd(a0, a2); v1 = cadd(a1, a3); v2 = csub(a0, a2); v3 = csub(a1, a3);
}

// in-register DFT of R points, natural order in and out
template <int R, int SIGN, typename T2>
__host__ __device__ __forceinline__ void dftr(T2 (&v)[R]) {
  using T = typename ScalarOf<T2>::t;
  if constexpr (R == 2) {
    const T2 a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    const T s32 = (T)0.86602540378443864676;   // sin(pi/3) = sqrt(3)/2
    const T2 t1 = cadd(v[1], v[2]);
    const T2 t2 = T2{v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y};
    const T dx = v[1].x - v[2].x, dy = v[1].y - v[2].y;
    const T2 t3 = (SIGN < 0) ? T2{s32 * dy, -s32 * dx} : T2{-s32 * dy, s32 * dx};
    v[0] = cadd(v[0], t1); v[1] = cadd(t2, t3); v[2] = csub(t2, t3);
  } else if constexpr (R == 4) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // 2 x 4: even / odd halves, then W8^k twiddles
    T2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    T2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<SIGN>(e0, e1, e2, e3);
    dft4<SIGN>(o0, o1, o2, o3);
    o1 = cmulf(o1, w16<SIGN, T2>(2));
    o2 = rot90<SIGN>(o2);
    o3 = cmulf(o3, w16<SIGN, T2>(6));
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
  } else {
    static_assert(R == 16, "radix");
    // 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2
    T2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
      a[n2][0] = v[n2]; a[n2][1] = v[4 + n2]; a[n2][2] = v[8 + n2]; a[n2][3] = v[12 + n2];
      dft4<SIGN>(a[n2][0], a[n2][1], a[n2][2], a[n2][3]);   // over n1 -> k1
    }
#pragma unroll
    for (int n2 = 1; n2 < 4; n2++)
#pragma unroll
      for (int k1 = 1; k1 < 4; k1++) a[n2][k1] = cmulf(a[n2][k1], w16<SIGN, T2>(n2 * k1));
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      T2 b0 = a[0][k1], b1 = a[1][k1], b2 = a[2][k1], b3 = a[3][k1];
      dft4<SIGN>(b0, b1, b2, b3);                              // over n2 -> k2
      v[k1] = b0; v[k1 + 4] = b1; v[k1 + 8] = b2; v[k1 + 12] = b3;
    }
  }
}

template <int N, int R, int NS, int NF, int SIGN>
__device__ __forceinline__ void fft_pass(const float2 *__restrict__ x, float2 *__restrict__ y,
                                         const float2 *__restrict__ tw) {
  constexpr int NB = N / R, NP = Plan3x2<N>::NP;
  for (int idx = threadIdx.x; idx < NF * NB; idx += blockDim.x) {
    const int f = idx / NB, j = idx - f * NB;
    const int k = j % NS;
    const float2 *xf = x + f * NP;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      float2 a = xf[fpad(j + r * NB)];
      if (NS > 1 && r > 0) {
        float2 w = tw[(r - 1) * NS + k];
        if (SIGN > 0) w.y = -w.y;
        a = cmulf(a, w);
      }
      v[r] = a;
    }
    dftr<R, SIGN>(v);
    float2 *yf = y + f * NP;
    const int d = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) yf[fpad(d + r * NS)] = v[r];
  }
  __syncthreads();
}

// all stages from `st` on; returns the buffer holding the result
template <int N, int NF, int SIGN, int ST>
__device__ __forceinline__ float2 *fft_passes(float2 *x, float2 *y, const float2 *tw) {
  using P = Plan3x2<N>;
  if constexpr (ST >= P::nst()) {
    return x;
  } else {
    fft_pass<N, P::radix(ST), P::ns(ST), NF, SIGN>(x, y, tw + P::off(ST));
    return fft_passes<N, NF, SIGN, ST + 1>(y, x, tw);
  }
}

// The fused row kernel for N = 3 * 2^b (see k_fft_products_m for the data
// flow).  Staging rows are padded to an odd stride so the transposes between
// the (m, element) order of HBM and the (element, m) order of the FFT rows
// are free of bank conflicts.
template <int N>
__global__ void __launch_bounds__(512, 2)
k_fft_products_t(int L, MLayout fin, MLayout fout, const float2 *__restrict__ twp, ProdCoef pc) {
  extern __shared__ __align__(16) unsigned char smraw[];
  using P = Plan3x2<N>;
  constexpr int NP = P::NP;
  static_assert(P::ntw() <= N, "twiddle table");
  float2 *A = reinterpret_cast<float2 *>(smraw);   // 7 x NP
  float2 *B = A + 7 * NP;                           // 7 x NP
  float2 *TW = B + 7 * NP;                          // per-stage twiddles (ntw)
  const int M1 = L + 1, MP = M1 | 1;                // padded (odd) staging stride
  float *S = reinterpret_cast<float *>(B);          // [c * 2 + s][MP]
  const int th = blockIdx.x / fin.nr, k = blockIdx.x % fin.nr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int e = tid; e < P::ntw(); e += blockDim.x) TW[e] = twp[e];
  // input: one warp per order m, lane j < 26 reads element j of the 10 + 16 run
  {
    int cs = 0;
    if (lane < 26) { int c, sg; m_comp_of_in(lane, c, sg); cs = c * 2 + sg; }
    const float *src = (lane < 10) ? fin.P + (size_t)th * fin.sP() + (size_t)k * 10 + lane
                                   : fin.D + (size_t)th * fin.sD() + (size_t)k * 16 + (lane - 10);
    const size_t mst = (size_t)fin.nth * ((lane < 10) ? fin.sP() : fin.sD());
    if (lane < 26)
      for (int m = warp; m <= L; m += nwarp) S[cs * MP + m] = __ldg(src + m * mst);
  }
  __syncthreads();
  // Hermitian rows z = x + i y of the 7 pairs: one thread per (pair, m) fills
  // n = m and n = N - m; the orders above L are zero
  for (int p = 0; p < 7; p++) {
    const int c0 = 2 * p, c1 = 2 * p + 1;
    const bool has1 = c1 < 13;
    float2 *Z = A + p * NP;
    for (int m = tid; m <= L; m += blockDim.x) {
      const float a0 = S[(c0 * 2) * MP + m], a1 = has1 ? S[(c1 * 2) * MP + m] : 0.0f;
      if (m == 0) {
        Z[0] = float2{a0, a1};
      } else {
        const float b0 = S[(c0 * 2 + 1) * MP + m], b1 = has1 ? S[(c1 * 2 + 1) * MP + m] : 0.0f;
        const float xr = 0.5f * a0, xi = -0.5f * b0, yr = 0.5f * a1, yi = -0.5f * b1;
        Z[fpad(m)] = float2{xr - yi, xi + yr};
        Z[fpad(N - m)] = float2{xr + yi, -xi + yr};
      }
    }
    for (int n = L + 1 + tid; n < N - L; n += blockDim.x) Z[fpad(n)] = float2{0.0f, 0.0f};
  }
  __syncthreads();
  float2 *g = fft_passes<N, 7, +1, 0>(A, B, TW);
  float2 *hb = (g == A) ? B : A;
  const float cv = (float)pc.cv, cl = (float)pc.cl, ci = (float)pc.ci, ct = (float)pc.ct;
  for (int qq = tid; qq < N; qq += blockDim.x) {
    const int q = fpad(qq);
    const float2 p0 = g[0 * NP + q], p1 = g[1 * NP + q], p2 = g[2 * NP + q], p3 = g[3 * NP + q];
    const float2 p4 = g[4 * NP + q], p5 = g[5 * NP + q], p6 = g[6 * NP + q];
    const float ur = p0.x, ut = p0.y, up = p1.x, wr = p1.y, wt = p2.x, wp = p2.y;
    const float br = p3.x, bt = p3.y, bp = p4.x, jr = p4.y, jt = p5.x, jp = p5.y, tt = p6.x;
    hb[0 * NP + q] = float2{(wt * up - wp * ut) * cv, (wp * ur - wr * up) * cv};
    hb[1 * NP + q] = float2{(wr * ut - wt * ur) * cv, (jt * bp - jp * bt) * cl};
    hb[2 * NP + q] = float2{(jp * br - jr * bp) * cl, (jr * bt - jt * br) * cl};
    hb[3 * NP + q] = float2{(ut * bp - up * bt) * ci, (up * br - ur * bp) * ci};
    hb[4 * NP + q] = float2{(ur * bt - ut * br) * ci, ur * tt * ct};
    hb[5 * NP + q] = float2{ut * tt * ct, up * tt * ct};
  }
  __syncthreads();
  float2 *zf = fft_passes<N, 6, -1, 0>(hb, g, TW);
  // (a_m, b_m) of both components of a pair from Z[m], Z[N - m]: one thread
  // per (pair, m), into the staging rows O[c * 2 + s][MP]
  float *O = reinterpret_cast<float *>((zf == A) ? B : A);
  const float an = 1.0f / (float)N;
  for (int p = 0; p < 6; p++) {
    const float2 *Z = zf + p * NP;
    float *o0 = O + (2 * p) * 2 * MP, *o1 = O + (2 * p + 1) * 2 * MP;
    for (int m = tid; m <= L; m += blockDim.x) {
      if (m == 0) {
        const float2 z0 = Z[0];
        o0[0] = an * z0.x; o0[MP] = 0.0f; o1[0] = an * z0.y; o1[MP] = 0.0f;
      } else {
        const float2 zk = Z[fpad(m)], zn = Z[fpad(N - m)];
        o0[m] = an * (zk.x + zn.x); o0[MP + m] = -an * (zk.y - zn.y);
        o1[m] = an * (zk.y + zn.y); o1[MP + m] = an * (zk.x - zn.x);
      }
    }
  }
  __syncthreads();
  // output: one warp per m, lane j < 24 writes element j of the 8 + 16 run
  {
    int cs = 0;
    if (lane < 24) { int c, sg; m_comp_of_out(lane, c, sg); cs = c * 2 + sg; }
    float *dst = (lane < 8) ? fout.P + (size_t)th * fout.sP() + (size_t)k * 8 + lane
                            : fout.D + (size_t)th * fout.sD() + (size_t)k * 16 + (lane - 8);
    const size_t mst = (size_t)fout.nth * ((lane < 8) ? fout.sP() : fout.sD());
    if (lane < 24)
      for (int m = warp; m <= L; m += nwarp) dst[m * mst] = O[cs * MP + m];
  }
}

// ---------------------------------------------------------------------------
// Four-step products kernel for N = 3 M, M = R1 R2 = L + 1 (the standard
// nphi = 3 (L + 1) grids).  One CTA per (theta, radial level) as above; 24
// groups of 16 threads, group (pair p, residue r) owns the M-point transform
// of the colatitude samples phi_j with j = 3 j' + r:
//   backward (spectrum -> grid, exponent +): the orders above L vanish, so
//     z(3 j' + r) = sum_{m < M} e^{2 pi i m j'/M} e^{2 pi i m r/N}
//                   (Z[m] + e^{4 pi i r/3} Z[N - (M - m)])
//   forward (grid -> spectrum, exponent -): F_r = M-point DFT of h(3 j' + r),
//     Z[m] = sum_r e^{-2 pi i m r/N} F_r[m],
//     Z[N - m] = sum_r e^{+2 pi i m r/N} F_r[(M - m) mod M].
// The M-point DFT is R1 x R2: n = n1 R2 + n2, k = k1 + R1 k2; a thread holds
// one n2 column (R1 values, DFT over n1 in registers, twiddle
// e^{+-2 pi i n2 k1/M}), a transpose through shared memory, then one k1 row
// (R2 values, DFT over n2).  The Hermitian pair rows are built on the fly
// from the staged (a_m, b_m) without the 1/2 of z = x + i y: the products
// are bilinear, so their coefficients carry the 1/4 instead (exact).
constexpr int F4_THREADS = 384;

template <int R1, int R2>
struct F4Plan {
  static constexpr int M = R1 * R2, N = 3 * M;
  static constexpr int TP = R2 + 1;            // transpose row pitch (complex)
  static constexpr int TG = R1 * TP;           // transpose block of one group
  static constexpr int X = (21 * TG > 7 * N) ? 21 * TG : 7 * N;   // work buffer (complex)
  static constexpr int MP2 = M + 1;            // staging row pitch (complex), slot M stays zero
  static constexpr int WP = R1 + 1;            // twiddle row pitch (complex)
  static constexpr int NTW = 3 * M + R2 * WP;  // tables: [3][M] e^{2 pi i m r/N}, [R2][WP] e^{2 pi i n2 k1/M}
  // staging (floats): 14 rows x MP2 complex in, later 12 rows x MP2 complex out
  static constexpr int SF = 28 * MP2;
  static constexpr size_t smem() { return (size_t)SF * 4 + ((size_t)X + NTW) * 8; }
};

template <typename T2>
__device__ __forceinline__ T2 cmulc(T2 a, T2 w) {   // a * conj(w)
  return T2{a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y};
}


// pmax (optional): the forward Legendre row scales' raw material, the
// largest |a_m| w(theta) of each output element over each block of 16
// orders, [theta][m / 16][element] with the elements of the output layout
// (P block k 8 + j, then D block sP + k 16 + j).
template <int R1, int R2>
__global__ void __launch_bounds__(F4_THREADS, 2)
k_fft_products_4s(MLayout fin, MLayout fout, const float2 *__restrict__ tables, ProdCoef pc,
                  float *__restrict__ pmax, const float *__restrict__ wgt) {
  using P = F4Plan<R1, R2>;
  constexpr int M = P::M, N = P::N, TP = P::TP, TG = P::TG, MP2 = P::MP2, WP = P::WP;
  extern __shared__ __align__(16) unsigned char smraw[];
  // input staging [7 pairs][MP2][2]: the (a_m, b_m) of components 2p and
  // 2p + 1 side by side (component 13 zero), so one 16-byte load reads both
  float2 *S2 = reinterpret_cast<float2 *>(smraw);
  float2 *X = reinterpret_cast<float2 *>(smraw + (size_t)P::SF * 4);   // transposes / grid rows / F_r
  float2 *TW3 = X + P::X;                                          // [3][M]
  float2 *TWM = TW3 + 3 * M;                                       // [R2][WP]
  const int th = blockIdx.x / fin.nr, k = blockIdx.x % fin.nr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = F4_THREADS / 32;
  const int grp = tid >> 4, lt = tid & 15;
  for (int e = tid; e < 14; e += F4_THREADS) S2[((e >> 1) * MP2 + M) * 2 + (e & 1)] = float2{0.0f, 0.0f};
  for (int e = tid; e < M; e += F4_THREADS) S2[(6 * MP2 + e) * 2 + 1] = float2{0.0f, 0.0f};
  // input and tables by asynchronous 8-byte copies, all in flight at once.
  // At one (theta, k) an order m has 13 (cos, sin) pairs: a run of 5 in the
  // P block and one of 8 in the D block; half-warp h of warp w copies the
  // orders 2 (w + nwarp i) + h, lane j < 13 of the half pair j into the
  // staging row of its component
  for (int e = tid; e < P::NTW; e += F4_THREADS) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(TW3 + e);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(tables + e) : "memory");
  }
  {
    const int j = lane & 15, hw = lane >> 4;
    int c = 0;
    const float *src = fin.P;
    size_t mst = 0;
    if (j < 5) {
      c = (j < 4) ? 3 * j : 12;
      src = fin.P + (size_t)th * fin.sP() + (size_t)k * 10 + 2 * j;
      mst = (size_t)fin.nth * fin.sP();
    } else if (j < 13) {
      const int jd = j - 5;
      c = 3 * (jd >> 1) + 1 + (jd & 1);
      src = fin.D + (size_t)th * fin.sD() + (size_t)k * 16 + 2 * jd;
      mst = (size_t)fin.nth * fin.sD();
    }
    if (j < 13)
      for (int m = 2 * warp + hw; m < M; m += 2 * nwarp) {
        const uint32_t d = (uint32_t)__cvta_generic_to_shared(S2 + ((c >> 1) * MP2 + m) * 2 + (c & 1));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src + m * mst) : "memory");
      }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
  }
  __syncthreads();
  const int gp = grp / 3, gr = grp - 3 * gp;   // pair, residue of this group
  // ---- backward, step 1: column n2 = lt, pair rows built from the staging
  if (grp < 21 && lt < R2) {
    const float4 *xy = reinterpret_cast<const float4 *>(S2) + gp * MP2;   // (x_m, y_m) of the pair
    const float2 om = (gr == 0) ? float2{1.0f, 0.0f}
                    : float2{-0.5f, (gr == 1) ? -0.86602540378443864676f : 0.86602540378443864676f};
    const float2 *tw = TW3 + gr * M;
    float2 v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) {
      const int m = n1 * R2 + lt, mq = M - m;
      const float4 ab = xy[m], cd = xy[mq];
      const float2 a = float2{ab.x, ab.y}, b = float2{ab.z, ab.w}, c = float2{cd.x, cd.y}, d = float2{cd.z, cd.w};
      float2 zm = float2{a.x + b.y, b.x - a.y};           // 2 Z[m]
      const float2 zp = float2{c.x - d.y, c.y + d.x};     // 2 Z[N - (M - m)] (zero at m = 0)
      if (n1 == 0 && lt == 0) zm = float2{2.0f * a.x, 2.0f * b.x};   // 2 Z[0] = 2 (a_0, a'_0)
      v[n1] = cmulf(cadd(zm, cmulf(om, zp)), tw[m]);
    }
    dftr<R1, +1>(v);
    float2 *T = X + grp * TG;
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) T[k1 * TP + lt] = (k1 == 0) ? v[0] : cmulf(v[k1], TWM[lt * WP + k1]);
  }
  // the transpose block T of a group is written and read by the group's own
  // 16 threads, half of one warp
  __syncwarp();
  // ---- backward, step 2: row k1 = lt -> grid samples j = 3 (k1 + R1 k2) + r
  float2 w[R2];
  if (grp < 21 && lt < R1) {
    const float2 *T = X + grp * TG + lt * TP;
#pragma unroll
    for (int n2 = 0; n2 < R2; n2++) w[n2] = T[n2];
    dftr<R2, +1>(w);
  }
  __syncthreads();
  if (grp < 21 && lt < R1) {
    float2 *G = X + gp * N + 3 * lt + gr;
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) G[3 * R1 * k2] = w[k2];
  }
  __syncthreads();
  // ---- products at every grid point (in place: 7 pair rows in, 6 out)
  {
    const float cv = 0.25f * (float)pc.cv, cl = 0.25f * (float)pc.cl, ci = 0.25f * (float)pc.ci,
                ct = 0.25f * (float)pc.ct;
    for (int q = tid; q < N; q += F4_THREADS) {
      const float2 p0 = X[0 * N + q], p1 = X[1 * N + q], p2 = X[2 * N + q], p3 = X[3 * N + q];
      const float2 p4 = X[4 * N + q], p5 = X[5 * N + q], p6 = X[6 * N + q];
      const float ur = p0.x, ut = p0.y, up = p1.x, wr = p1.y, wt = p2.x, wp = p2.y;
      const float br = p3.x, bt = p3.y, bp = p4.x, jr = p4.y, jt = p5.x, jp = p5.y, tt = p6.x;
      X[0 * N + q] = float2{(wt * up - wp * ut) * cv, (wp * ur - wr * up) * cv};
      X[1 * N + q] = float2{(wr * ut - wt * ur) * cv, (jt * bp - jp * bt) * cl};
      X[2 * N + q] = float2{(jp * br - jr * bp) * cl, (jr * bt - jt * br) * cl};
      X[3 * N + q] = float2{(ut * bp - up * bt) * ci, (up * br - ur * bp) * ci};
      X[4 * N + q] = float2{(ur * bt - ut * br) * ci, ur * tt * ct};
      X[5 * N + q] = float2{ut * tt * ct, up * tt * ct};
    }
  }
  __syncthreads();
  // ---- forward, step 1: column n2 = lt of the samples j = 3 (n1 R2 + n2) + r
  float2 v[R1];
  if (grp < 18 && lt < R2) {
    const float2 *G = X + gp * N + 3 * lt + gr;
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) v[n1] = G[3 * R2 * n1];
    dftr<R1, -1>(v);
#pragma unroll
    for (int k1 = 1; k1 < R1; k1++) v[k1] = cmulc(v[k1], TWM[lt * WP + k1]);
  }
  __syncthreads();
  if (grp < 18 && lt < R2) {
    float2 *T = X + grp * TG;
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) T[k1 * TP + lt] = v[k1];
  }
  __syncwarp();   // the group's own transpose block, as in the backward steps
  // ---- forward, step 2: row k1 = lt -> F_r[k1 + R1 k2]
  if (grp < 18 && lt < R1) {
    const float2 *T = X + grp * TG + lt * TP;
#pragma unroll
    for (int n2 = 0; n2 < R2; n2++) w[n2] = T[n2];
    dftr<R2, -1>(w);
  }
  __syncthreads();
  if (grp < 18 && lt < R1) {
    float2 *F = X + grp * M + lt;   // [pair][r][M]: grp = 3 p + r
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) F[R1 * k2] = w[k2];
  }
  __syncthreads();
  // ---- combine the residues: Z[m], Z[N - m] -> (a_m, b_m) of both
  // components of each pair, into the output staging rows [c][MP2] of
  // (a_m, b_m) pairs.  A thread takes the orders m and M - m together: both
  // read the same six F values.
  float2 *O2 = S2;
  {
    const float an = 1.0f / (float)N;
    constexpr int MH = M / 2 + 1;
    auto out = [&](float2 *o0, float2 *o1, int m, float2 zk, float2 zn) {
      if (m == 0) {
        o0[0] = float2{an * zk.x, 0.0f}; o1[0] = float2{an * zk.y, 0.0f};
      } else {
        o0[m] = float2{an * (zk.x + zn.x), -an * (zk.y - zn.y)};
        o1[m] = float2{an * (zk.y + zn.y), an * (zk.x - zn.x)};
      }
    };
    for (int idx = tid; idx < 6 * MH; idx += F4_THREADS) {
      const int p = idx / MH, m = idx - p * MH, mm = (M - m) & (M - 1);
      const float2 *F = X + p * 3 * M;
      float2 *o0 = O2 + (2 * p) * MP2, *o1 = o0 + MP2;
      const float2 f0 = F[m], f1 = F[M + m], f2 = F[2 * M + m];
      const float2 g0 = F[mm], g1 = F[M + mm], g2 = F[2 * M + mm];
      {
        const float2 t1 = TW3[M + m], t2 = TW3[2 * M + m];
        const float2 zk = cadd(f0, cadd(cmulc(f1, t1), cmulc(f2, t2)));
        const float2 zn = cadd(g0, cadd(cmulf(g1, t1), cmulf(g2, t2)));
        out(o0, o1, m, zk, zn);
      }
      if (m > 0 && mm != m) {   // the partner order M - m
        const float2 t1 = TW3[M + mm], t2 = TW3[2 * M + mm];
        const float2 zk = cadd(g0, cadd(cmulc(g1, t1), cmulc(g2, t2)));
        const float2 zn = cadd(f0, cadd(cmulf(f1, t1), cmulf(f2, t2)));
        out(o0, o1, mm, zk, zn);
      }
    }
  }
  __syncthreads();
  // output: 12 (cos, sin) pairs per order, a run of 4 in the P block and one
  // of 8 in the D block; half-warp h of warp w writes the orders
  // 2 (w + nwarp i) + h, lane j < 12 of the half pair j (8-byte stores)
  {
    const int j = lane & 15, hw = lane >> 4;
    int c = 0;
    float *dst = fout.P;
    size_t mst = 0;
    if (j < 4) {
      c = 3 * j;
      dst = fout.P + (size_t)th * fout.sP() + (size_t)k * 8 + 2 * j;
      mst = (size_t)fout.nth * fout.sP();
    } else if (j < 12) {
      const int jd = j - 4;
      c = 3 * (jd >> 1) + 1 + (jd & 1);
      dst = fout.D + (size_t)th * fout.sD() + (size_t)k * 16 + 2 * jd;
      mst = (size_t)fout.nth * fout.sD();
    }
    if (j < 12)
      for (int m = 2 * warp + hw; m < M; m += 2 * nwarp)
        *reinterpret_cast<float2 *>(dst + m * mst) = O2[c * MP2 + m];
  }
  if (pmax) {
    constexpr int MB = M / 16;
    const float wt = __ldg(wgt + th);
    const size_t E = fout.sP() + fout.sD();
    float *pm = pmax + (size_t)th * MB * E;
    for (int t = tid; t < 24 * MB; t += F4_THREADS) {
      const int j = t % 24, mb = t / 24;
      int c, sg;
      m_comp_of_out(j, c, sg);
      const float *row = reinterpret_cast<const float *>(O2 + c * MP2 + mb * 16) + sg;
      float mx = 0.0f;
#pragma unroll
      for (int u = 0; u < 16; u++) mx = fmaxf(mx, fabsf(row[2 * u]));
      const size_t e = (j < 8) ? (size_t)k * 8 + j : fout.sP() + (size_t)k * 16 + (j - 8);
      pm[(size_t)mb * E + e] = mx * wt;
    }
  }
}

// ---------------------------------------------------------------------------
// The float64 four-step products kernel (the plain path's step): the data
// flow of k_fft_products_4s on the float64 Fourier rows
// four[(theta, k)][c][2 m + s] (a_m at 2 m, b_m at 2 m + 1), with the pair
// scaling of k_fft_products (the second row of each pair, inputs and
// products, brought to the size of the first), so every row keeps float64
// precision whatever the sizes of the fields.  One CTA per (theta, k), 384
// threads, one CTA per SM (166 KB of shared memory at M = 256).
template <int R1, int R2>
struct F4Plan64 {
  static constexpr int M = R1 * R2, N = 3 * M;
  static constexpr int TP = R2 + 1;
  static constexpr int TG = R1 * TP;
  static constexpr int X = (21 * TG > 7 * N) ? 21 * TG : 7 * N;
  static constexpr int MP2 = M + 1;            // staging row pitch, slot M stays zero
  static constexpr int WP = R1 + 1;
  static constexpr int NTW = 3 * M + R2 * WP;
  static constexpr int SC = 14 * MP2;          // staging: 14 rows in, then 12 rows out
  static constexpr size_t smem() { return ((size_t)SC + X + NTW) * sizeof(double2) + 32 * sizeof(double); }
};

template <int R1, int R2>
__global__ void __launch_bounds__(F4_THREADS, 1)
k_fft_products_4s64(const double *__restrict__ four, double *__restrict__ four2, int NS,
                    const double2 *__restrict__ tables, ProdCoef pc) {
  using P = F4Plan64<R1, R2>;
  using PB = PairBits<double>;
  using U = PB::U;
  constexpr int M = P::M, N = P::N, TP = P::TP, TG = P::TG, MP2 = P::MP2, WP = P::WP;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2 *S2 = reinterpret_cast<double2 *>(smraw);   // [14][MP2] (a_m, b_m); later [12][MP2] out
  double2 *X = S2 + P::SC;                             // transposes / grid rows / F_r
  double2 *TW3 = X + P::X;                             // [3][M]
  double2 *TWM = TW3 + 3 * M;                          // [R2][WP]
  U *cmx = reinterpret_cast<U *>(TWM + R2 * WP);      // [0, 13) input maxima, [13, 25) products
  const size_t row = blockIdx.x;
  const double *fin = four + row * 13 * (size_t)NS;
  double *fout = four2 + row * 12 * (size_t)NS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = F4_THREADS / 32;
  const int grp = tid >> 4, lt = tid & 15;
  for (int e = tid; e < P::NTW; e += F4_THREADS) TW3[e] = tables[e];
  for (int e = tid; e < 14; e += F4_THREADS) S2[e * MP2 + M] = double2{0.0, 0.0};
  for (int e = tid; e < M; e += F4_THREADS) S2[13 * MP2 + e] = double2{0.0, 0.0};
  for (int e = tid; e < 13 * M; e += F4_THREADS) {
    const int c = e / M, m = e - c * M;
    S2[c * MP2 + m] = __ldg(reinterpret_cast<const double2 *>(fin + (size_t)c * NS) + m);
  }
  if (tid < 12) cmx[13 + tid] = 0;
  __syncthreads();
  // largest magnitude of each input row (one warp per row)
  for (int c = warp; c < 13; c += nwarp) {
    U mx = 0;
    for (int m = lane; m < M; m += 32) {
      const double2 v = S2[c * MP2 + m];
      mx = max(mx, max(PB::abs_bits(v.x), PB::abs_bits(v.y)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, (U)__shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) cmx[c] = mx;
  }
  __syncthreads();
  const int gp = grp / 3, gr = grp - 3 * gp;
  // ---- backward, step 1: column n2 = lt, pair rows from the staging (the
  // second row of the pair scaled by sy)
  if (grp < 21 && lt < R2) {
    const double2 *x0 = S2 + (2 * gp) * MP2, *y0 = S2 + (2 * gp + 1) * MP2;
    const double sy = (2 * gp + 1 < 13) ? PB::factor(cmx[2 * gp], cmx[2 * gp + 1], false) : 1.0;
    const double2 om = (gr == 0) ? double2{1.0, 0.0}
                     : double2{-0.5, (gr == 1) ? -0.86602540378443864676 : 0.86602540378443864676};
    const double2 *tw = TW3 + gr * M;
    double2 v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; n1++) {
      const int m = n1 * R2 + lt, mq = M - m;
      const double2 a = x0[m], c = x0[mq];
      const double2 b = double2{y0[m].x * sy, y0[m].y * sy}, d = double2{y0[mq].x * sy, y0[mq].y * sy};
      double2 zm = double2{a.x + b.y, b.x - a.y};           // 2 Z[m]
      const double2 zp = double2{c.x - d.y, c.y + d.x};     // 2 Z[N - (M - m)] (zero at m = 0)
      if (n1 == 0 && lt == 0) zm = double2{2.0 * a.x, 2.0 * b.x};
      v[n1] = cmulf(cadd(zm, cmulf(om, zp)), tw[m]);
    }
    dftr<R1, +1>(v);
    double2 *T = X + grp * TG;
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) T[k1 * TP + lt] = (k1 == 0) ? v[0] : cmulf(v[k1], TWM[lt * WP + k1]);
  }
  __syncthreads();
  // ---- backward, step 2: row k1 = lt -> grid samples j = 3 (k1 + R1 k2) + r
  {
    double2 w[R2];
    if (grp < 21 && lt < R1) {
      const double2 *T = X + grp * TG + lt * TP;
#pragma unroll
      for (int n2 = 0; n2 < R2; n2++) w[n2] = T[n2];
      dftr<R2, +1>(w);
    }
    __syncthreads();
    if (grp < 21 && lt < R1) {
      double2 *G = X + gp * N + 3 * lt + gr;
#pragma unroll
      for (int k2 = 0; k2 < R2; k2++) G[3 * R1 * k2] = w[k2];
    }
  }
  __syncthreads();
  // ---- products at every grid point (the second rows unscaled on the way
  // in), with the largest magnitude of each product row
  {
    const double cv = 0.25 * pc.cv, cl = 0.25 * pc.cl, ci = 0.25 * pc.ci, ct = 0.25 * pc.ct;
    double iy[6];
#pragma unroll
    for (int p = 0; p < 6; p++) iy[p] = PB::factor(cmx[2 * p], cmx[2 * p + 1], true);
    U hm[12];
#pragma unroll
    for (int c = 0; c < 12; c++) hm[c] = 0;
    for (int q = tid; q < N; q += F4_THREADS) {
      const double2 p0 = X[0 * N + q], p1 = X[1 * N + q], p2 = X[2 * N + q], p3 = X[3 * N + q];
      const double2 p4 = X[4 * N + q], p5 = X[5 * N + q], p6 = X[6 * N + q];
      const double ur = p0.x, ut = p0.y * iy[0], up = p1.x, wr = p1.y * iy[1], wt = p2.x, wp = p2.y * iy[2];
      const double br = p3.x, bt = p3.y * iy[3], bp = p4.x, jr = p4.y * iy[4], jt = p5.x, jp = p5.y * iy[5];
      const double tt = p6.x;
      const double2 hv[6] = {double2{(wt * up - wp * ut) * cv, (wp * ur - wr * up) * cv},
                             double2{(wr * ut - wt * ur) * cv, (jt * bp - jp * bt) * cl},
                             double2{(jp * br - jr * bp) * cl, (jr * bt - jt * br) * cl},
                             double2{(ut * bp - up * bt) * ci, (up * br - ur * bp) * ci},
                             double2{(ur * bt - ut * br) * ci, ur * tt * ct},
                             double2{ut * tt * ct, up * tt * ct}};
#pragma unroll
      for (int p = 0; p < 6; p++) {
        X[p * N + q] = hv[p];
        hm[2 * p] = max(hm[2 * p], PB::abs_bits(hv[p].x));
        hm[2 * p + 1] = max(hm[2 * p + 1], PB::abs_bits(hv[p].y));
      }
    }
#pragma unroll
    for (int c = 0; c < 12; c++) {
      U v = hm[c];
      for (int o = 16; o > 0; o >>= 1) v = max(v, (U)__shfl_xor_sync(0xffffffffu, v, o));
      if (lane == 0) atomicMax(cmx + 13 + c, v);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < 6 * N; idx += F4_THREADS) {
    const int p = idx / N;
    X[idx].y *= PB::factor(cmx[13 + 2 * p], cmx[14 + 2 * p], false);
  }
  __syncthreads();
  // ---- forward, step 1: column n2 = lt of the samples j = 3 (n1 R2 + n2) + r
  {
    double2 v[R1];
    if (grp < 18 && lt < R2) {
      const double2 *G = X + gp * N + 3 * lt + gr;
#pragma unroll
      for (int n1 = 0; n1 < R1; n1++) v[n1] = G[3 * R2 * n1];
      dftr<R1, -1>(v);
#pragma unroll
      for (int k1 = 1; k1 < R1; k1++) v[k1] = cmulc(v[k1], TWM[lt * WP + k1]);
    }
    __syncthreads();
    if (grp < 18 && lt < R2) {
      double2 *T = X + grp * TG;
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) T[k1 * TP + lt] = v[k1];
    }
  }
  __syncthreads();
  // ---- forward, step 2: row k1 = lt -> F_r[k1 + R1 k2]
  {
    double2 w[R2];
    if (grp < 18 && lt < R1) {
      const double2 *T = X + grp * TG + lt * TP;
#pragma unroll
      for (int n2 = 0; n2 < R2; n2++) w[n2] = T[n2];
      dftr<R2, -1>(w);
    }
    __syncthreads();
    if (grp < 18 && lt < R1) {
      double2 *F = X + grp * M + lt;   // [pair][r][M]: grp = 3 p + r
#pragma unroll
      for (int k2 = 0; k2 < R2; k2++) F[R1 * k2] = w[k2];
    }
  }
  __syncthreads();
  // ---- combine the residues: (a_m, b_m) of both rows of each pair (the
  // second unscaled), into the staging rows [c][MP2]
  {
    const double an = 1.0 / (double)N;
    for (int idx = tid; idx < 6 * M; idx += F4_THREADS) {
      const int p = idx / M, m = idx - p * M, mm = (M - m) & (M - 1);
      const double2 *F = X + p * 3 * M;
      const double2 t1 = TW3[M + m], t2 = TW3[2 * M + m];
      const double2 zk = cadd(F[m], cadd(cmulc(F[M + m], t1), cmulc(F[2 * M + m], t2)));
      const double2 zn = cadd(F[mm], cadd(cmulf(F[M + mm], t1), cmulf(F[2 * M + mm], t2)));
      const double ay = an * PB::factor(cmx[13 + 2 * p], cmx[14 + 2 * p], true);
      double2 *o0 = S2 + (2 * p) * MP2, *o1 = S2 + (2 * p + 1) * MP2;
      if (m == 0) {
        o0[0] = double2{an * zk.x, 0.0};
        o1[0] = double2{ay * zk.y, 0.0};
      } else {
        o0[m] = double2{an * (zk.x + zn.x), -an * (zk.y - zn.y)};
        o1[m] = double2{ay * (zk.y + zn.y), ay * (zk.x - zn.x)};
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < 12 * M; e += F4_THREADS) {
    const int c = e / M, m = e - c * M;
    reinterpret_cast<double2 *>(fout + (size_t)c * NS)[m] = S2[c * MP2 + m];
  }
}

// order-major Fourier rows -> grid (float64), for the standalone transform API
__global__ void __launch_bounds__(256)
k_fft_to_grid_m(FFTPlan pl, int L, MLayout fin, double *grid, const float2 *tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n, nc = 3 * fin.nvec + fin.nscal, nr = fin.nr, nth = fin.nth;
  float2 *Z0 = reinterpret_cast<float2 *>(smraw), *Z1 = Z0 + N;
  const int th = blockIdx.x / nr, k = blockIdx.x % nr;
  const int mmax = min(L, (N + 1) / 2 - 1);
  __shared__ unsigned pmx[2];
  for (int c = 0; c < nc; c += 2) {
    const bool has1 = c + 1 < nc;
    if (threadIdx.x < 2) pmx[threadIdx.x] = 0u;
    for (int q = threadIdx.x; q < N; q += blockDim.x) Z0[q] = float2{0, 0};
    __syncthreads();
    // pair scaling (pair_exp): the second row brought to the size of the first
    {
      unsigned mx = 0u, my = 0u;
      for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
        mx = max(mx, max(abs_bits(*fin.at(m, th, k, c, 0)), abs_bits(*fin.at(m, th, k, c, 1))));
        if (has1) my = max(my, max(abs_bits(*fin.at(m, th, k, c + 1, 0)), abs_bits(*fin.at(m, th, k, c + 1, 1))));
      }
      mx = __reduce_max_sync(0xffffffffu, mx);
      my = __reduce_max_sync(0xffffffffu, my);
      if ((threadIdx.x & 31) == 0) { atomicMax(pmx, mx); atomicMax(pmx + 1, my); }
    }
    __syncthreads();
    const int ep = pair_exp(pmx[0], pmx[1]);
    const float sy = pow2i(ep), iy = pow2i(-ep);
    for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
      const float a0 = *fin.at(m, th, k, c, 0), b0 = (m > 0) ? *fin.at(m, th, k, c, 1) : 0.0f;
      const float a1 = has1 ? *fin.at(m, th, k, c + 1, 0) * sy : 0.0f;
      const float b1 = (has1 && m > 0) ? *fin.at(m, th, k, c + 1, 1) * sy : 0.0f;
      if (m == 0) {
        Z0[0] = float2{a0, a1};
      } else {
        const float xr = 0.5f * a0, xi = -0.5f * b0, yr = 0.5f * a1, yi = -0.5f * b1;
        Z0[m] = float2{xr - yi, xi + yr};
        Z0[N - m] = float2{xr + yi, -xi + yr};
      }
    }
    __syncthreads();
    float2 *z = block_fft<float, float2>(Z0, Z1, pl, tw, +1);
    for (int q = threadIdx.x; q < N; q += blockDim.x) {
      grid[(((size_t)c * nr + k) * nth + th) * N + q] = (double)z[q].x;
      if (has1) grid[(((size_t)(c + 1) * nr + k) * nth + th) * N + q] = (double)(z[q].y * iy);
    }
    __syncthreads();
  }
}

// grid (float64) -> order-major Fourier rows
__global__ void __launch_bounds__(256)
k_grid_to_fft_m(FFTPlan pl, int L, const double *grid, MLayout fout, const float2 *tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int N = pl.n, nc = 3 * fout.nvec + fout.nscal, nr = fout.nr, nth = fout.nth;
  float2 *Z0 = reinterpret_cast<float2 *>(smraw), *Z1 = Z0 + N;
  const int th = blockIdx.x / nr, k = blockIdx.x % nr;
  const float an = (float)(1.0 / (double)N);
  __shared__ unsigned pmx[2];
  for (int c = 0; c < nc; c += 2) {
    const bool has1 = c + 1 < nc;
    if (threadIdx.x < 2) pmx[threadIdx.x] = 0u;
    __syncthreads();
    unsigned mx = 0u, my = 0u;
    for (int q = threadIdx.x; q < N; q += blockDim.x) {
      const float x = (float)grid[(((size_t)c * nr + k) * nth + th) * N + q];
      const float y = has1 ? (float)grid[(((size_t)(c + 1) * nr + k) * nth + th) * N + q] : 0.0f;
      Z0[q] = float2{x, y};
      mx = max(mx, abs_bits(x));
      my = max(my, abs_bits(y));
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    my = __reduce_max_sync(0xffffffffu, my);
    if ((threadIdx.x & 31) == 0) { atomicMax(pmx, mx); atomicMax(pmx + 1, my); }
    __syncthreads();
    // pair scaling (pair_exp): the second row brought to the size of the first
    const int ep = pair_exp(pmx[0], pmx[1]);
    if (ep != 0) {
      const float sy = pow2i(ep);
      for (int q = threadIdx.x; q < N; q += blockDim.x) Z0[q].y *= sy;
      __syncthreads();
    }
    const float ay = an * pow2i(-ep);
    const float2 *z = block_fft<float, float2>(Z0, Z1, pl, tw, -1);
    for (int m = threadIdx.x; m <= L; m += blockDim.x) {
      float a0, b0, a1, b1;
      if (m == 0) {
        a0 = an * z[0].x; b0 = 0.0f; a1 = ay * z[0].y; b1 = 0.0f;
      } else {
        const float2 zk = z[m % N], zn = z[(N - m) % N];
        const float xr = 0.5f * (zk.x + zn.x), xi = 0.5f * (zk.y - zn.y);
        const float yr = 0.5f * (zk.y + zn.y), yi = -0.5f * (zk.x - zn.x);
        a0 = 2.0f * an * xr; b0 = -2.0f * an * xi; a1 = 2.0f * ay * yr; b1 = -2.0f * ay * yi;
      }
      *fout.at(m, th, k, c, 0) = a0;
      *fout.at(m, th, k, c, 1) = b0;
      if (has1) {
        *fout.at(m, th, k, c + 1, 0) = a1;
        *fout.at(m, th, k, c + 1, 1) = b1;
      }
    }
    __syncthreads();
  }
}

__global__ void k_twiddles(int n, double2 *tw, float2 *tw32) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double s, c;
  sincospi(2.0 * (double)e / (double)n, &s, &c);
  tw[e] = make_double2(c, -s);
  tw32[e] = make_float2((float)c, (float)-s);
}

static FFTPlan make_plan(int n) {
  FFTPlan p{};
  p.n = n;
  int m = n;
  while (m % 3 == 0) { p.rad[p.nst++] = 3; m /= 3; }
  while (m % 4 == 0) { p.rad[p.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { p.rad[p.nst++] = 2; m /= 2; }
  if (m != 1) p.nst = -1;
  return p;
}

template <int N>
static size_t smem_fft_t() { return (14 * (size_t)Plan3x2<N>::NP + N) * sizeof(float2); }

// smem attribute and the per-stage twiddle table w^(r k) of Plan3x2<N>
template <int N>
static int attr_fft_t(Ctx &c) {
  using P = Plan3x2<N>;
  CB2_CUDA(raise_smem_limit(k_fft_products_t<N>, (int)smem_fft_t<N>()));
  std::vector<float2> t(P::ntw());
  const double pi = 3.14159265358979323846;
  for (int st = 0; st < P::nst(); st++) {
    const int R = P::radix(st), NS = P::ns(st), tstr = N / (NS * R);
    for (int r = 1; r < R; r++)
      for (int k = 0; k < NS; k++) {
        const double ang = -2.0 * pi * (double)(r * k * tstr) / (double)N;
        t[P::off(st) + (r - 1) * NS + k] = float2{(float)std::cos(ang), (float)std::sin(ang)};
      }
  }
  CB2_CUDA(cudaMalloc(&c.d_twp32, t.size() * sizeof(float2)));
  CB2_CUDA(cudaMemcpy(c.d_twp32, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice));
  return 0;
}

// smem attribute and the tables of the four-step kernel:
// [3][M] e^{2 pi i m r/N} (row 0 ones), [R2][R1 + 1] e^{2 pi i n2 k1/M}
template <int R1, int R2>
static int attr_fft_4s(Ctx &c) {
  using P = F4Plan<R1, R2>;
  CB2_CUDA(raise_smem_limit(k_fft_products_4s<R1, R2>, (int)P::smem()));
  std::vector<float2> t(P::NTW, float2{0.0f, 0.0f});
  const double pi = 3.14159265358979323846;
  for (int r = 0; r < 3; r++)
    for (int m = 0; m < P::M; m++) {
      const double ang = 2.0 * pi * (double)(m * r) / (double)P::N;
      t[r * P::M + m] = float2{(float)std::cos(ang), (float)std::sin(ang)};
    }
  for (int n2 = 0; n2 < R2; n2++)
    for (int k1 = 0; k1 < R1; k1++) {
      const double ang = 2.0 * pi * (double)(n2 * k1) / (double)P::M;
      t[3 * P::M + n2 * P::WP + k1] = float2{(float)std::cos(ang), (float)std::sin(ang)};
    }
  CB2_CUDA(cudaMalloc(&c.d_twf4, t.size() * sizeof(float2)));
  CB2_CUDA(cudaMemcpy(c.d_twf4, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice));
  return 0;
}

template <int R1, int R2>
static int attr_fft_4s64(Ctx &c) {
  using P = F4Plan64<R1, R2>;
  CB2_CUDA(raise_smem_limit(k_fft_products_4s64<R1, R2>, (int)P::smem()));
  std::vector<double2> t(P::NTW, double2{0.0, 0.0});
  const double pi = 3.14159265358979323846;
  for (int r = 0; r < 3; r++)
    for (int m = 0; m < P::M; m++) {
      const double ang = 2.0 * pi * (double)(m * r) / (double)P::N;
      t[r * P::M + m] = double2{std::cos(ang), std::sin(ang)};
    }
  for (int n2 = 0; n2 < R2; n2++)
    for (int k1 = 0; k1 < R1; k1++) {
      const double ang = 2.0 * pi * (double)(n2 * k1) / (double)P::M;
      t[3 * P::M + n2 * P::WP + k1] = double2{std::cos(ang), std::sin(ang)};
    }
  CB2_CUDA(cudaMalloc(&c.d_twf4_64, t.size() * sizeof(double2)));
  CB2_CUDA(cudaMemcpy(c.d_twf4_64, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice));
  return 0;
}

int fft_setup(Ctx &c) {
  FFTPlan p = make_plan(c.nph);
  if (p.nst < 0) {
    set_error("ngrid_zonal_ctl must be of the form 3^a 2^b");
    return CB2_ERR_ARG;
  }
  CB2_CUDA(cudaMalloc(&c.d_tw_fft, (size_t)c.nph * sizeof(double2)));
  CB2_CUDA(cudaMalloc(&c.d_tw_fft32, (size_t)c.nph * sizeof(float2)));
  k_twiddles<<<cdiv(c.nph, 256), 256, 0, c.stream>>>(c.nph, (double2 *)c.d_tw_fft,
                                                     (float2 *)c.d_tw_fft32);
  CB2_CUDA(cudaGetLastError());
  size_t big = 14 * (size_t)c.nph * sizeof(double2) + 32 * sizeof(double);
  if (big > 227 * 1024) {
    set_error("ngrid_zonal_ctl too large for the fused FFT kernel");
    return CB2_ERR_ARG;
  }
  CB2_CUDA(raise_smem_limit(k_fft_products<double>, (int)big));
  CB2_CUDA(raise_smem_limit(k_fft_products<float>, (int)big));
  CB2_CUDA(raise_smem_limit(k_fft_products_m, (int)(14 * (size_t)c.nph * sizeof(float2) + 32 * sizeof(float))));
  {
    int rc = 0;
    switch (c.nph) {
      case 768: rc = attr_fft_t<768>(c); break;
      case 384: rc = attr_fft_t<384>(c); break;
      case 192: rc = attr_fft_t<192>(c); break;
      case 96: rc = attr_fft_t<96>(c); break;
      default: break;
    }
    if (rc) return rc;
    if (c.nph == 3 * (c.L + 1)) {
      switch (c.nph) {
        case 768: rc = attr_fft_4s<16, 16>(c); break;
        case 384: rc = attr_fft_4s<16, 8>(c); break;
        case 192: rc = attr_fft_4s<8, 8>(c); break;
        case 96: rc = attr_fft_4s<8, 4>(c); break;
        default: break;
      }
      if (rc) return rc;
      switch (c.nph) {
        case 768: rc = attr_fft_4s64<16, 16>(c); break;
        case 384: rc = attr_fft_4s64<16, 8>(c); break;
        case 192: rc = attr_fft_4s64<8, 8>(c); break;
        case 96: rc = attr_fft_4s64<8, 4>(c); break;
        default: break;
      }
      if (rc) return rc;
    }
  }
  if (26 * (size_t)(c.L + 1) * sizeof(float) > 7 * (size_t)c.nph * sizeof(float2)) {
    set_error("ngrid_zonal_ctl too small for the staging of the fused FFT kernel");
    return CB2_ERR_ARG;
  }
  return 0;
}

template <typename T>
static const typename C2<T>::t *twid(Ctx &c) {
  if (sizeof(T) == 8) return (const typename C2<T>::t *)c.d_tw_fft;
  return (const typename C2<T>::t *)c.d_tw_fft32;
}

template <int R1, int R2>
static void launch_fft_4s64(Ctx &c, const double *four, double *four2, const ProdCoef &pc) {
  k_fft_products_4s64<R1, R2><<<(unsigned)(c.nth * c.nr), F4_THREADS, F4Plan64<R1, R2>::smem(), c.stream>>>(
      four, four2, c.NS, (const double2 *)c.d_twf4_64, pc);
}

template <typename T>
void fft_products(Ctx &c, const T *four, T *four2) {
  using T2 = typename C2<T>::t;
  if constexpr (sizeof(T) == 8) {
    // tuning value F4_THREADS selects the four-step kernel where it applies
    if (c.d_twf4_64 && c.tune[TUNE_FFT_THREADS] == F4_THREADS) {
      ProdCoef pc{c.p.coef_velo, c.p.coef_lor, c.p.coef_induct, c.p.coef_temp};
      switch (c.nph) {
        case 768: launch_fft_4s64<16, 16>(c, four, four2, pc); return;
        case 384: launch_fft_4s64<16, 8>(c, four, four2, pc); return;
        case 192: launch_fft_4s64<8, 8>(c, four, four2, pc); return;
        case 96: launch_fft_4s64<8, 4>(c, four, four2, pc); return;
        default: break;
      }
    }
  }
  FFTPlan p = make_plan(c.nph);
  size_t sm = 14 * (size_t)c.nph * sizeof(T2) + 32 * sizeof(double);
  ProdCoef pc{c.p.coef_velo, c.p.coef_lor, c.p.coef_induct, c.p.coef_temp};
  k_fft_products<T><<<(unsigned)(c.nth * c.nr), 512, sm, c.stream>>>(p, c.L, c.NS, four, four2,
                                                                     twid<T>(c), pc);
}

template <typename T>
void fft_backward_grid(Ctx &c, int ncomp, const T *four, double *grid) {
  using T2 = typename C2<T>::t;
  FFTPlan p = make_plan(c.nph);
  size_t sm = 2 * (size_t)c.nph * sizeof(T2);
  k_fft_to_grid<T><<<(unsigned)(c.nth * c.nr), 256, sm, c.stream>>>(p, c.L, c.NS, ncomp, c.nr, c.nth,
                                                                    four, grid, twid<T>(c));
}

template <typename T>
void fft_forward_grid(Ctx &c, int ncomp, const double *grid, T *four) {
  using T2 = typename C2<T>::t;
  FFTPlan p = make_plan(c.nph);
  size_t sm = 2 * (size_t)c.nph * sizeof(T2);
  k_grid_to_fft<T><<<(unsigned)(c.nth * c.nr), 256, sm, c.stream>>>(p, c.L, c.NS, ncomp, c.nr, c.nth,
                                                                    grid, four, twid<T>(c));
}

template <int N>
static void launch_fft_t(Ctx &c, const MLayout &in, const MLayout &out, const ProdCoef &pc) {
  const size_t sm = smem_fft_t<N>();
  const int nt = c.tune[TUNE_FFT_THREADS];
  const int threads = (nt == 128 || nt == 256) ? nt : 512;
  k_fft_products_t<N><<<(unsigned)(c.nth * c.nr), threads, sm, c.stream>>>(c.L, in, out, (const float2 *)c.d_twp32,
                                                                          pc);
}

template <int R1, int R2>
static bool launch_fft_4s(Ctx &c, const MLayout &in, const MLayout &out, const ProdCoef &pc, float *pmax) {
  k_fft_products_4s<R1, R2><<<(unsigned)(c.nth * c.nr), F4_THREADS, F4Plan<R1, R2>::smem(), c.stream>>>(
      in, out, (const float2 *)c.d_twf4, pc, pmax, pmax ? mixed_weights32(c) : nullptr);
  return pmax != nullptr;
}

bool fft_products_m(Ctx &c, const MLayout &in, const MLayout &out, float *pmax) {
  ProdCoef pc{c.p.coef_velo, c.p.coef_lor, c.p.coef_induct, c.p.coef_temp};
  // tuning value F4_THREADS selects the four-step kernel where it applies
  if (c.d_twf4 && c.tune[TUNE_FFT_THREADS] == F4_THREADS) {
    switch (c.nph) {
      case 768: return launch_fft_4s<16, 16>(c, in, out, pc, pmax);
      case 384: return launch_fft_4s<16, 8>(c, in, out, pc, pmax);
      case 192: return launch_fft_4s<8, 8>(c, in, out, pc, pmax);
      case 96: return launch_fft_4s<8, 4>(c, in, out, pc, pmax);
      default: break;
    }
  }
  switch (c.nph) {
    case 768: launch_fft_t<768>(c, in, out, pc); return false;
    case 384: launch_fft_t<384>(c, in, out, pc); return false;
    case 192: launch_fft_t<192>(c, in, out, pc); return false;
    case 96: launch_fft_t<96>(c, in, out, pc); return false;
    default: break;
  }
  FFTPlan p = make_plan(c.nph);
  size_t sm = 14 * (size_t)c.nph * sizeof(float2) + 32 * sizeof(float);
  k_fft_products_m<<<(unsigned)(c.nth * c.nr), 512, sm, c.stream>>>(p, c.L, in, out, (const float2 *)c.d_tw_fft32,
                                                                   pc);
  return false;
}

void fft_backward_grid_m(Ctx &c, const MLayout &in, double *grid) {
  FFTPlan p = make_plan(c.nph);
  size_t sm = 2 * (size_t)c.nph * sizeof(float2);
  k_fft_to_grid_m<<<(unsigned)(c.nth * c.nr), 256, sm, c.stream>>>(p, c.L, in, grid, (const float2 *)c.d_tw_fft32);
}

void fft_forward_grid_m(Ctx &c, const double *grid, const MLayout &out) {
  FFTPlan p = make_plan(c.nph);
  size_t sm = 2 * (size_t)c.nph * sizeof(float2);
  k_grid_to_fft_m<<<(unsigned)(c.nth * c.nr), 256, sm, c.stream>>>(p, c.L, grid, out, (const float2 *)c.d_tw_fft32);
}

template void fft_products<double>(Ctx &, const double *, double *);
template void fft_products<float>(Ctx &, const float *, float *);
template void fft_backward_grid<double>(Ctx &, int, const double *, double *);
template void fft_backward_grid<float>(Ctx &, int, const float *, double *);
template void fft_forward_grid<double>(Ctx &, int, const double *, double *);
template void fft_forward_grid<float>(Ctx &, int, const double *, float *);

}  // namespace cb2
