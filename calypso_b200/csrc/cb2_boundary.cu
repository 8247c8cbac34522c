// cb2_boundary.cu -- routine-level entry points on the reference's buffers.
//
// The reference reaches its Legendre and FFT stages through
//   sel_backward_legendre_trans / sel_forward_legendre_trans
//     (PARALLEL_src/SPH_SHELL_src/legendre_transform_select.f90:309-439):
//     spectra sp_rlm(comp + ncomp ((k-1) istep_rlm(1) + (j-1) istep_rlm(2)))
//     <-> Fourier coefficients vr_rtm(comp + ncomp ((k-1) istep_rtm(1)
//          + (l-1) istep_rtm(2) + (mp-1) istep_rtm(3)))
//     (legendre_bwd_trans_org.f90:45-209, legendre_fwd_trans_org.f90:45-169)
//   back_MHD_FFT_sel_from_recv / fwd_MHD_FFT_sel_from_recv
//     (MHD_src/sph_MHD/MHD_FFT_selector.F90:185-249): Fourier coefficients
//     <-> grid fld_rtp(inod, comp), inod = (k-1) istep_rtp(1)
//          + (l-1) istep_rtp(2) + (p-1) istep_rtp(3) + 1.
// Here the same buffers (host or device memory) go through the library's
// own layouts: the spectra into work slots of the field array (device
// m-major order), the Fourier coefficients into the Fourier rows of the
// context's precision, the grid into [comp][k][theta][phi].  The index
// permutations are the reference's rj <-> rlm and rtm <-> rtp transposes,
// done on the device.  Components are processed in chunks that fit the
// context's Fourier buffers.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

namespace {

bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int grow(void **buf, size_t *have, size_t need) {
  if (*have >= need) return 0;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  CB2_CUDA(cudaMalloc(buf, need));
  *have = need;
  return 0;
}

// device table of one call: jj of each j_rlm, then (|m|, s) of each mp
struct DevTab {
  const int *jj = nullptr;   // nidx_rlm(2)
  const int *mq = nullptr;   // nidx_rtm(3) x 2: |m|, s (0 cos / order +m, 1 sin / order -m)
};

int check_tables(const Ctx &c, const cb2_sph_tables *t, bool need_rlm, bool need_rtp) {
  if (!t) { set_error("null index tables"); return CB2_ERR_ARG; }
  if (t->nidx_rtm[0] != c.nr || t->nidx_rtm[1] != c.nth || t->nidx_rtm[2] < 1 || t->nidx_rtm[2] > 2 * c.L + 1 ||
      !t->idx_gl_1d_rtm_m) {
    set_error("rtm tables: need nidx_rtm = (nr, nth, 1..2L+1) and idx_gl_1d_rtm_m");
    return CB2_ERR_ARG;
  }
  for (int q = 0; q < 3; q++)
    if (t->istep_rtm[q] < 1) { set_error("istep_rtm must be positive"); return CB2_ERR_ARG; }
  for (int mp = 0; mp < t->nidx_rtm[2]; mp++) {
    const int m = t->idx_gl_1d_rtm_m[t->nidx_rtm[2] + mp];
    if (m < -c.L || m > c.L) { set_error("idx_gl_1d_rtm_m: order outside -L..L"); return CB2_ERR_ARG; }
  }
  if (need_rlm) {
    if (t->nidx_rlm[0] != c.nr || t->nidx_rlm[1] < 1 || t->nidx_rlm[1] > c.jmax || !t->idx_gl_1d_rlm_j ||
        t->istep_rlm[0] < 1 || t->istep_rlm[1] < 1) {
      set_error("rlm tables: need nidx_rlm = (nr, 1..(L+1)^2), positive istep_rlm and idx_gl_1d_rlm_j");
      return CB2_ERR_ARG;
    }
    const int nj = t->nidx_rlm[1];
    for (int j = 0; j < nj; j++) {
      const int l = t->idx_gl_1d_rlm_j[nj + j], m = t->idx_gl_1d_rlm_j[2 * nj + j];
      if (l < 0 || l > c.L || m < -l || m > l) {
        set_error("idx_gl_1d_rlm_j: (l, m) outside the truncation");
        return CB2_ERR_ARG;
      }
    }
  }
  if (need_rtp) {
    if (t->nidx_rtp[0] != c.nr || t->nidx_rtp[1] != c.nth || t->nidx_rtp[2] != c.nph || t->istep_rtp[0] < 1 ||
        t->istep_rtp[1] < 1 || t->istep_rtp[2] < 1) {
      set_error("rtp tables: need nidx_rtp = (nr, nth, nph) and positive istep_rtp");
      return CB2_ERR_ARG;
    }
    const size_t top = (size_t)(c.nr - 1) * t->istep_rtp[0] + (size_t)(c.nth - 1) * t->istep_rtp[1] +
                       (size_t)(c.nph - 1) * t->istep_rtp[2];
    if (top >= (size_t)c.nr * c.nth * c.nph) {
      set_error("istep_rtp: index beyond nnod_rtp = nr nth nph");
      return CB2_ERR_ARG;
    }
  }
  return 0;
}

// largest index + 1 of the rlm / rtm buffers for ncomp components
size_t rlm_extent(const cb2_sph_tables *t, int ncomp) {
  return (size_t)ncomp * ((size_t)(t->nidx_rlm[0] - 1) * t->istep_rlm[0] +
                          (size_t)(t->nidx_rlm[1] - 1) * t->istep_rlm[1] + 1);
}
size_t rtm_extent(const cb2_sph_tables *t, int ncomp) {
  return (size_t)ncomp * ((size_t)(t->nidx_rtm[0] - 1) * t->istep_rtm[0] +
                          (size_t)(t->nidx_rtm[1] - 1) * t->istep_rtm[1] +
                          (size_t)(t->nidx_rtm[2] - 1) * t->istep_rtm[2] + 1);
}

int jj_host(const Ctx &c, int l, int m) {
  const int am = std::abs(m);
  return c.h_moff[am] + ((m < 0) ? (c.L + 1 - am) : 0) + (l - am);
}

int upload_tables(Ctx &c, const cb2_sph_tables *t, bool rlm, DevTab *d) {
  const int nj = rlm ? t->nidx_rlm[1] : 0, nm = t->nidx_rtm[2];
  std::vector<int> h((size_t)nj + 2 * (size_t)nm);
  for (int j = 0; j < nj; j++) h[j] = jj_host(c, t->idx_gl_1d_rlm_j[nj + j], t->idx_gl_1d_rlm_j[2 * nj + j]);
  for (int mp = 0; mp < nm; mp++) {
    const int m = t->idx_gl_1d_rtm_m[nm + mp];
    h[nj + 2 * mp] = std::abs(m);
    h[nj + 2 * mp + 1] = (m < 0) ? 1 : 0;
  }
  if (int rc = grow((void **)&c.d_bnd_tab, &c.bnd_tab_bytes, h.size() * sizeof(int))) return rc;
  CB2_CUDA(cudaMemcpyAsync(c.d_bnd_tab, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  d->jj = c.d_bnd_tab;
  d->mq = c.d_bnd_tab + nj;
  return 0;
}

// the caller's buffer on the device: itself, or a copy in staging buffer `which`
int device_in(Ctx &c, const double *p, size_t n, int which, const double **out) {
  if (is_device_ptr(p)) { *out = p; return 0; }
  double **b = which ? &c.d_bnd_b : &c.d_bnd_a;
  size_t *have = which ? &c.bnd_b_bytes : &c.bnd_a_bytes;
  if (int rc = grow((void **)b, have, n * sizeof(double))) return rc;
  CB2_CUDA(cudaMemcpyAsync(*b, p, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  *out = *b;
  return 0;
}

int device_out(Ctx &c, double *p, size_t n, int which, double **out) {
  if (is_device_ptr(p)) { *out = p; return 0; }
  double **b = which ? &c.d_bnd_b : &c.d_bnd_a;
  size_t *have = which ? &c.bnd_b_bytes : &c.bnd_a_bytes;
  if (int rc = grow((void **)b, have, n * sizeof(double))) return rc;
  *out = *b;
  return 0;
}

int finish_out(Ctx &c, double *host, const double *dev, size_t n) {
  if (host != dev) CB2_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

// one chunk of components: comp0.. of the caller's numbering, the first nv
// of them vectors (3 components each), then ns scalars
struct Chunk {
  int comp0, nv, ns;
  int nc() const { return 3 * nv + ns; }
};

// chunks that fit the Fourier buffers: float64 rows hold 13 components;
// the mixed transforms take at most 4 vectors and 8 fields with 6 nv + 2 ns
// <= 26 floats per radial level
std::vector<Chunk> chunks(int prec, int nvec, int nscal) {
  std::vector<Chunk> out;
  int comp = 0, v = 0, s = 0;
  while (v < nvec || s < nscal) {
    Chunk ch{comp, 0, 0};
    ch.nv = std::min(4, nvec - v);
    int room = (prec == CB2_PREC_FP64) ? 13 - 3 * ch.nv : std::min(8 - ch.nv, (26 - 6 * ch.nv) / 2);
    ch.ns = (ch.nv == nvec - v) ? std::min(room, nscal - s) : 0;
    v += ch.nv;
    s += ch.ns;
    comp += ch.nc();
    out.push_back(ch);
  }
  return out;
}

constexpr int kBnd = 256;

// rlm buffer -> work slots (device order), one thread per (j_rlm, k)
__global__ void k_rlm_to_slots(int nj, int nr, int ncomp, int is0, int is1, int comp0, int nq, int slot0,
                               const int *jj, const double *WR, double *f, size_t fs, int jmax) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= nj || k >= nr) return;
  const size_t src = (size_t)ncomp * ((size_t)k * is0 + (size_t)j * is1) + comp0;
  const size_t dst = (size_t)k * jmax + jj[j];
  for (int q = 0; q < nq; q++) f[(size_t)(slot0 + q) * fs + dst] = WR[src + q];
}

__global__ void k_slots_to_rlm(int nj, int nr, int ncomp, int is0, int is1, int comp0, int nq, int slot0,
                               const int *jj, const double *f, size_t fs, int jmax, double *WS) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= nj || k >= nr) return;
  const size_t dst = (size_t)ncomp * ((size_t)k * is0 + (size_t)j * is1) + comp0;
  const size_t src = (size_t)k * jmax + jj[j];
  for (int q = 0; q < nq; q++) WS[dst + q] = f[(size_t)(slot0 + q) * fs + src];
}

// Fourier rows of the context (float64 [theta][k][c][slot] with nc
// components, or the mixed float32 layout) <-> rtm buffer; one thread per
// (theta, k), blockIdx.y = mp
struct FourView {
  double *f64 = nullptr;   // float64 rows, nc components, NS slots
  int nc = 0, NS = 0, nr = 0;
  MLayout ml;              // mixed rows when f64 is null
  __device__ double get(int m, int th, int k, int c, int s) const {
    if (f64) return f64[(((size_t)th * nr + k) * nc + c) * NS + 2 * m + s];
    return (double)*ml.at(m, th, k, c, s);
  }
  __device__ void put(int m, int th, int k, int c, int s, double v) const {
    if (f64) f64[(((size_t)th * nr + k) * nc + c) * NS + 2 * m + s] = v;
    else *ml.at(m, th, k, c, s) = (float)v;
  }
};

__global__ void k_four_to_rtm(FourView fv, int nth, int nr, int ncomp, int is0, int is1, int is2, int comp0,
                              const int *mq, double *WS) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, mp = blockIdx.y;
  if (i >= nth * nr) return;
  const int th = i / nr, k = i - th * nr;
  const int m = mq[2 * mp], s = mq[2 * mp + 1];
  const size_t dst = (size_t)ncomp * ((size_t)k * is0 + (size_t)th * is1 + (size_t)mp * is2) + comp0;
  for (int q = 0; q < fv.nc; q++) WS[dst + q] = (m == 0 && s == 1) ? 0.0 : fv.get(m, th, k, q, s);
}

// rows of orders the table does not list stay zero (cleared before)
__global__ void k_rtm_to_four(FourView fv, int nth, int nr, int ncomp, int is0, int is1, int is2, int comp0,
                              const int *mq, const double *WR) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, mp = blockIdx.y;
  if (i >= nth * nr) return;
  const int th = i / nr, k = i - th * nr;
  const int m = mq[2 * mp], s = mq[2 * mp + 1];
  const size_t src = (size_t)ncomp * ((size_t)k * is0 + (size_t)th * is1 + (size_t)mp * is2) + comp0;
  for (int q = 0; q < fv.nc; q++) fv.put(m, th, k, q, s, (m == 0 && s == 1) ? 0.0 : WR[src + q]);
}

// grid [c][k][theta][phi] <-> fld_rtp(inod, comp), one thread per grid point
__global__ void k_grid_to_rtp(int nc, int nr, int nth, int nph, int is0, int is1, int is2, int comp0,
                              size_t nnod, const double *grid, double *fld) {
  const size_t n = (size_t)nr * nth * nph;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = (int)(i % nph);
  const size_t t = i / nph;
  const int th = (int)(t % nth), k = (int)(t / nth);
  const size_t inod = (size_t)k * is0 + (size_t)th * is1 + (size_t)p * is2;
  for (int q = 0; q < nc; q++) fld[inod + nnod * (comp0 + q)] = grid[(size_t)q * n + i];
}

__global__ void k_rtp_to_grid(int nc, int nr, int nth, int nph, int is0, int is1, int is2, int comp0,
                              size_t nnod, const double *fld, double *grid) {
  const size_t n = (size_t)nr * nth * nph;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = (int)(i % nph);
  const size_t t = i / nph;
  const int th = (int)(t % nth), k = (int)(t / nth);
  const size_t inod = (size_t)k * is0 + (size_t)th * is1 + (size_t)p * is2;
  for (int q = 0; q < nc; q++) grid[(size_t)q * n + i] = fld[inod + nnod * (comp0 + q)];
}

FourView four_view(Ctx &c, int nv, int ns, void *buf = nullptr) {
  if (!buf) buf = c.d_four;
  FourView fv;
  fv.nr = c.nr;
  fv.NS = c.NS;
  fv.nc = 3 * nv + ns;
  if (c.prec == CB2_PREC_FP64) fv.f64 = (double *)buf;
  else fv.ml = mlayout(c, buf, nv, ns);
  return fv;
}

size_t four_bytes(const Ctx &c) {
  return (c.prec == CB2_PREC_FP64) ? (size_t)c.nth * c.nr * c.NS * 13 * sizeof(double)
                                   : mlayout_floats(c) * sizeof(float);
}

int leg_args_ok(const Ctx &c, int ncomp, int nvec, int nscal) {
  if (nvec < 0 || nscal < 0 || nvec + nscal == 0 || ncomp < 3 * nvec + nscal) {
    set_error("Legendre transform: need nvector, nscalar >= 0, at least one field, ncomp >= 3 nvector + nscalar");
    return CB2_ERR_ARG;
  }
  if (3 * nvec + nscal > NSLOT - MADV) {
    set_error("Legendre transform: at most 38 components per call");
    return CB2_ERR_ARG;
  }
  return 0;
}

}  // namespace

}  // namespace cb2

using namespace cb2;

extern "C" {

int cb2_leg_bwd(cb2_ctx *c, const cb2_sph_tables *t, int ncomp, int nvector, int nscalar, size_t n_WR,
                size_t n_WS, const double *WR, double *WS) {
  if (!c || !WR || !WS) { set_error("null argument"); return CB2_ERR_ARG; }
  if (int rc = leg_args_ok(*c, ncomp, nvector, nscalar)) return rc;
  if (int rc = check_tables(*c, t, true, false)) return rc;
  if (n_WR < rlm_extent(t, ncomp) || n_WS < rtm_extent(t, ncomp)) {
    set_error("cb2_leg_bwd: n_WR or n_WS smaller than the tables' extent");
    return CB2_ERR_ARG;
  }
  DevTab dt;
  const double *dWR;
  double *dWS;
  int rc;
  if ((rc = upload_tables(*c, t, true, &dt)) || (rc = device_in(*c, WR, n_WR, 0, &dWR)) ||
      (rc = device_out(*c, WS, n_WS, 1, &dWS)))
    return rc;
  // the callee clears WS, as the reference's backward transforms do
  CB2_CUDA(cudaMemsetAsync(dWS, 0, n_WS * sizeof(double), c->stream));
  const int nj = t->nidx_rlm[1];
  for (const Chunk &ch : chunks(c->prec, nvector, nscalar)) {
    const int nc = ch.nc();
    // vectors occupy three slots each from MADV, scalars follow
    int slots[13];
    for (int g = 0; g < ch.nv; g++) slots[g] = MADV + 3 * g;
    for (int s = 0; s < ch.ns; s++) slots[ch.nv + s] = MADV + 3 * ch.nv + s;
    // modes the table leaves out are zero
    if (nj < c->jmax)
      CB2_CUDA(cudaMemsetAsync(c->fld(MADV), 0, (size_t)nc * c->fsize() * sizeof(double), c->stream));
    k_rlm_to_slots<<<dim3(cdiv(nj, kBnd), c->nr), kBnd, 0, c->stream>>>(
        nj, c->nr, ncomp, t->istep_rlm[0], t->istep_rlm[1], ch.comp0, nc, MADV, dt.jj, dWR, c->d_f, c->fsize(),
        c->jmax);
    if (c->prec == CB2_PREC_FP64) {
      leg_bwd_f64(*c, ch.nv, ch.ns, slots, (double *)c->d_four);
    } else {
      const MLayout l = mlayout(*c, c->d_four, ch.nv, ch.ns);
      if ((rc = leg_bwd_mixed(*c, slots, l))) return rc;
    }
    k_four_to_rtm<<<dim3(cdiv((long)c->nth * c->nr, kBnd), t->nidx_rtm[2]), kBnd, 0, c->stream>>>(
        four_view(*c, ch.nv, ch.ns), c->nth, c->nr, ncomp, t->istep_rtm[0], t->istep_rtm[1], t->istep_rtm[2],
        ch.comp0, dt.mq, dWS);
  }
  CB2_CUDA(cudaGetLastError());
  if ((rc = finish_out(*c, WS, dWS, n_WS))) return rc;
  return check_status(*c);
}

int cb2_leg_fwd(cb2_ctx *c, const cb2_sph_tables *t, int ncomp, int nvector, int nscalar, size_t n_WR,
                size_t n_WS, const double *WR, double *WS) {
  if (!c || !WR || !WS) { set_error("null argument"); return CB2_ERR_ARG; }
  if (int rc = leg_args_ok(*c, ncomp, nvector, nscalar)) return rc;
  if (int rc = check_tables(*c, t, true, false)) return rc;
  if (n_WR < rtm_extent(t, ncomp) || n_WS < rlm_extent(t, ncomp)) {
    set_error("cb2_leg_fwd: n_WR or n_WS smaller than the tables' extent");
    return CB2_ERR_ARG;
  }
  DevTab dt;
  const double *dWR;
  double *dWS;
  int rc;
  if ((rc = upload_tables(*c, t, true, &dt)) || (rc = device_in(*c, WR, n_WR, 0, &dWR)) ||
      (rc = device_out(*c, WS, n_WS, 1, &dWS)))
    return rc;
  CB2_CUDA(cudaMemsetAsync(dWS, 0, n_WS * sizeof(double), c->stream));
  const int nj = t->nidx_rlm[1];
  for (const Chunk &ch : chunks(c->prec, nvector, nscalar)) {
    const int nc = ch.nc();
    int slots[13];
    for (int g = 0; g < ch.nv; g++) slots[g] = MADV + 3 * g;
    for (int s = 0; s < ch.ns; s++) slots[ch.nv + s] = MADV + 3 * ch.nv + s;
    CB2_CUDA(cudaMemsetAsync(c->d_four, 0, four_bytes(*c), c->stream));
    k_rtm_to_four<<<dim3(cdiv((long)c->nth * c->nr, kBnd), t->nidx_rtm[2]), kBnd, 0, c->stream>>>(
        four_view(*c, ch.nv, ch.ns), c->nth, c->nr, ncomp, t->istep_rtm[0], t->istep_rtm[1], t->istep_rtm[2],
        ch.comp0, dt.mq, dWR);
    if (c->prec == CB2_PREC_FP64) {
      leg_fwd_f64(*c, ch.nv, ch.ns, (const double *)c->d_four, slots);
    } else {
      const MLayout l = mlayout(*c, c->d_four, ch.nv, ch.ns);
      if ((rc = leg_fwd_mixed(*c, l, slots))) return rc;
    }
    k_slots_to_rlm<<<dim3(cdiv(nj, kBnd), c->nr), kBnd, 0, c->stream>>>(
        nj, c->nr, ncomp, t->istep_rlm[0], t->istep_rlm[1], ch.comp0, nc, MADV, dt.jj, c->d_f, c->fsize(),
        c->jmax, dWS);
  }
  CB2_CUDA(cudaGetLastError());
  if ((rc = finish_out(*c, WS, dWS, n_WS))) return rc;
  return check_status(*c);
}

int cb2_fft_bwd(cb2_ctx *c, const cb2_sph_tables *t, int ncomp, size_t n_WR, const double *WR, double *fld_rtp) {
  if (!c || !WR || !fld_rtp || ncomp < 1) { set_error("null argument or ncomp < 1"); return CB2_ERR_ARG; }
  if (int rc = check_tables(*c, t, false, true)) return rc;
  if (n_WR < rtm_extent(t, ncomp)) { set_error("cb2_fft_bwd: n_WR smaller than the tables' extent"); return CB2_ERR_ARG; }
  const size_t nnod = (size_t)c->nr * c->nth * c->nph, nout = nnod * ncomp;
  DevTab dt;
  const double *dWR;
  double *dF;
  int rc;
  if ((rc = upload_tables(*c, t, false, &dt)) || (rc = device_in(*c, WR, n_WR, 0, &dWR)) ||
      (rc = device_out(*c, fld_rtp, nout, 1, &dF)))
    return rc;
  if ((rc = grow((void **)&c->d_bnd_grid, &c->bnd_grid_bytes, 13 * nnod * sizeof(double)))) return rc;
  for (int c0 = 0; c0 < ncomp; c0 += 13) {
    const int nc = std::min(13, ncomp - c0);
    CB2_CUDA(cudaMemsetAsync(c->d_four, 0, four_bytes(*c), c->stream));
    FourView fv = four_view(*c, 0, nc);
    k_rtm_to_four<<<dim3(cdiv((long)c->nth * c->nr, kBnd), t->nidx_rtm[2]), kBnd, 0, c->stream>>>(
        fv, c->nth, c->nr, ncomp, t->istep_rtm[0], t->istep_rtm[1], t->istep_rtm[2], c0, dt.mq, dWR);
    if (c->prec == CB2_PREC_FP64) fft_backward_grid<double>(*c, nc, (const double *)c->d_four, c->d_bnd_grid);
    else fft_backward_grid_m(*c, fv.ml, c->d_bnd_grid);
    k_grid_to_rtp<<<cdiv((long)nnod, kBnd), kBnd, 0, c->stream>>>(nc, c->nr, c->nth, c->nph, t->istep_rtp[0],
                                                                  t->istep_rtp[1], t->istep_rtp[2], c0, nnod,
                                                                  c->d_bnd_grid, dF);
  }
  CB2_CUDA(cudaGetLastError());
  return finish_out(*c, fld_rtp, dF, nout);
}

int cb2_fft_products(cb2_ctx *c, const cb2_sph_tables *t, size_t n_WR, const double *WR, size_t n_WS,
                     double *WS) {
  if (!c || !WR || !WS) { set_error("null argument"); return CB2_ERR_ARG; }
  if (int rc = check_tables(*c, t, false, false)) return rc;
  if (n_WR < rtm_extent(t, 13) || n_WS < rtm_extent(t, 12)) {
    set_error("cb2_fft_products: n_WR (13 components) or n_WS (12) smaller than the tables' extent");
    return CB2_ERR_ARG;
  }
  DevTab dt;
  const double *dWR;
  double *dWS;
  int rc;
  if ((rc = upload_tables(*c, t, false, &dt)) || (rc = device_in(*c, WR, n_WR, 0, &dWR)) ||
      (rc = device_out(*c, WS, n_WS, 1, &dWS)))
    return rc;
  CB2_CUDA(cudaMemsetAsync(dWS, 0, n_WS * sizeof(double), c->stream));
  CB2_CUDA(cudaMemsetAsync(c->d_four, 0, four_bytes(*c), c->stream));
  const FourView fin = four_view(*c, 4, 1), fout = four_view(*c, 4, 0, c->d_four2);
  const dim3 grid(cdiv((long)c->nth * c->nr, kBnd), t->nidx_rtm[2]);
  k_rtm_to_four<<<grid, kBnd, 0, c->stream>>>(fin, c->nth, c->nr, 13, t->istep_rtm[0], t->istep_rtm[1],
                                             t->istep_rtm[2], 0, dt.mq, dWR);
  if (c->prec == CB2_PREC_FP64) fft_products<double>(*c, (const double *)c->d_four, (double *)c->d_four2);
  else fft_products_m(*c, fin.ml, fout.ml);
  k_four_to_rtm<<<grid, kBnd, 0, c->stream>>>(fout, c->nth, c->nr, 12, t->istep_rtm[0], t->istep_rtm[1],
                                             t->istep_rtm[2], 0, dt.mq, dWS);
  CB2_CUDA(cudaGetLastError());
  return finish_out(*c, WS, dWS, n_WS);
}

int cb2_fft_fwd(cb2_ctx *c, const cb2_sph_tables *t, int ncomp, const double *frc_rtp, size_t n_WS, double *WS) {
  if (!c || !WS || !frc_rtp || ncomp < 1) { set_error("null argument or ncomp < 1"); return CB2_ERR_ARG; }
  if (int rc = check_tables(*c, t, false, true)) return rc;
  if (n_WS < rtm_extent(t, ncomp)) { set_error("cb2_fft_fwd: n_WS smaller than the tables' extent"); return CB2_ERR_ARG; }
  const size_t nnod = (size_t)c->nr * c->nth * c->nph, nin = nnod * ncomp;
  DevTab dt;
  const double *dF;
  double *dWS;
  int rc;
  if ((rc = upload_tables(*c, t, false, &dt)) || (rc = device_in(*c, frc_rtp, nin, 0, &dF)) ||
      (rc = device_out(*c, WS, n_WS, 1, &dWS)))
    return rc;
  if ((rc = grow((void **)&c->d_bnd_grid, &c->bnd_grid_bytes, 13 * nnod * sizeof(double)))) return rc;
  CB2_CUDA(cudaMemsetAsync(dWS, 0, n_WS * sizeof(double), c->stream));
  for (int c0 = 0; c0 < ncomp; c0 += 13) {
    const int nc = std::min(13, ncomp - c0);
    k_rtp_to_grid<<<cdiv((long)nnod, kBnd), kBnd, 0, c->stream>>>(nc, c->nr, c->nth, c->nph, t->istep_rtp[0],
                                                                  t->istep_rtp[1], t->istep_rtp[2], c0, nnod, dF,
                                                                  c->d_bnd_grid);
    FourView fv = four_view(*c, 0, nc);
    if (c->prec == CB2_PREC_FP64) fft_forward_grid<double>(*c, nc, c->d_bnd_grid, (double *)c->d_four);
    else fft_forward_grid_m(*c, c->d_bnd_grid, fv.ml);
    k_four_to_rtm<<<dim3(cdiv((long)c->nth * c->nr, kBnd), t->nidx_rtm[2]), kBnd, 0, c->stream>>>(
        fv, c->nth, c->nr, ncomp, t->istep_rtm[0], t->istep_rtm[1], t->istep_rtm[2], c0, dt.mq, dWS);
  }
  CB2_CUDA(cudaGetLastError());
  return finish_out(*c, WS, dWS, n_WS);
}

}  // extern "C"
