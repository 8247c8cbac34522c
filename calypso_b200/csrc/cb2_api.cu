// cb2_api.cu -- the C ABI of libcalypso_b200 (see include/calypso_b200.h).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int cuda_fail(cudaError_t e, const char *what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return CB2_ERR_CUDA;
}

// l = 0 part of the temperature: (T + T_ref) - T_ref each step, as the
// reference's trans_per_temp_to_temp_sph / sync_temp_by_per_temp_sph pair
__global__ void k_temp_roundtrip(int nr, size_t jmax, const double *reft0, double *T) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nr) return;
  double v = T[(size_t)k * jmax] + reft0[k];
  T[(size_t)k * jmax] = v - reft0[k];
}

// host j = l(l+1)+m  <->  device m-major jj
__global__ void k_to_device_order(int nr, int jmax, const int *perm, const double *src, double *dst) {
  size_t n = (size_t)nr * jmax;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = (int)(i / jmax), jj = (int)(i % jmax);
  dst[i] = src[(size_t)k * jmax + perm[jj]];
}

__global__ void k_to_host_order(int nr, int jmax, const int *perm, const double *src, double *dst) {
  size_t n = (size_t)nr * jmax;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = (int)(i / jmax), jj = (int)(i % jmax);
  dst[(size_t)k * jmax + perm[jj]] = src[i];
}

__global__ void k_fill(size_t n, double *x, double v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

// initial state (set_initial_sph_dynamo.f90, initial_magne_dynamobench.f90)
__global__ void k_init_dbench1(RJArgs a, double *f, size_t fs, int jj44, int js, int jt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nr) return;
  double pi = 4.0 * atan(1.0);
  double ri = a.r[a.kin], ro = a.r[a.kout], shell = ro - ri;
  size_t at = (size_t)k * a.jmax;
  double *T = f + (size_t)TEMP * fs;
  if (a.use_ref_temp) T[at] = a.reft0[k];
  if (k < a.kin || k > a.kout) return;
  if (jj44 >= 0) {
    double xr = 2.0 * a.r[k] - 1.0 * (ro + ri) / shell;
    double x2 = xr * xr, x4 = x2 * x2, x6 = x4 * x2;
    T[at + jj44] = (1.0 - 3.0 * x2 + 3.0 * x4 - x6) * 0.1 * 3.0 / sqrt(2.0 * pi);
  }
  double rr = a.r[k];
  if (js >= 0) {
    f[(size_t)MAGNE * fs + at + js] = (5.0 / 8.0) * (-3.0 * rr * rr * rr + 4.0 * ro * rr * rr - ri * ri * ri * ri / rr);
    f[(size_t)(MAGNE + 1) * fs + at + js] = (5.0 / 8.0) * (-9.0 * rr * rr + 8.0 * ro * rr + ri * ri * ri * ri / (rr * rr));
    f[(size_t)(CURRENT + 2) * fs + at + js] = (5.0 * 3.0 / 2.0) * rr;
  }
  if (jt >= 0) {
    double bt = (10.0 / 3.0) * rr * sin(pi * (rr - ri));
    f[(size_t)(MAGNE + 2) * fs + at + jt] = bt;
    f[(size_t)CURRENT * fs + at + jt] = bt;
    f[(size_t)(CURRENT + 1) * fs + at + jt] = (10.0 / 3.0) * (sin(pi * (rr - ri)) + pi * rr * cos(pi * (rr - ri)));
  }
}

__global__ void k_init_seeded(RJArgs a, double *f, size_t fs, const int *jjs, const double *amp, int nmode,
                              int mode_b0) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nr) return;
  double ri = a.r[a.kin], ro = a.r[a.kout], shell = ro - ri;
  size_t at = (size_t)k * a.jmax;
  double *T = f + (size_t)TEMP * fs;
  if (a.use_ref_temp) T[at] = a.reft0[k];
  if (k < a.kin || k > a.kout) return;
  double xr = 2.0 * a.r[k] - 1.0 * (ro + ri) / shell;
  double x2 = xr * xr, x4 = x2 * x2, x6 = x4 * x2;
  double rr = a.r[k];
  for (int q = 0; q < nmode; q++) {
    if (q < mode_b0) T[at + jjs[q]] = amp[q] * (1.0 - 3.0 * x2 + 3.0 * x4 - x6);
    else f[(size_t)MAGNE * fs + at + jjs[q]] = amp[q] * (-3.0 * rr * rr * rr + 4.0 * ro * rr * rr - ri * ri * ri * ri / rr);
  }
}

__global__ void k_temp_shift(int nr, size_t jmax, const double *reft0, double *T, double sign) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nr) return;
  T[(size_t)k * jmax] += sign * reft0[k];
}

static unsigned long long rng_next(unsigned long long *s) {
  unsigned long long z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double rng_uniform(unsigned long long *s) {
  return (double)(rng_next(s) >> 11) * (1.0 / 9007199254740992.0);
}

static int jj_of(const Ctx &c, int l, int m) {
  int am = std::abs(m);
  return c.h_moff[am] + ((m < 0) ? (c.L + 1 - am) : 0) + (l - am);
}

static const int kBwdSlots[5] = {VELO, VORT, MAGNE, CURRENT, TEMP};
static const int kFwdSlots[4] = {MADV, LOR, VPIND, HFLUX};

// The nonlinear terms in three parts around the mixed path's two
// tensor-core Legendre GEMMs:
//   head: mixed: the spectra packed for the backward GEMM
//   grid: mixed: FFT + grid products, the forward GEMM's row scales
//   tail: rj operators after the forward transform (with the Coriolis
//         term), closure
// nonlinear() launches this shell's GEMMs between them; an ensemble
// launches each GEMM once for all its shells (step_phase).
static int nl_head(Ctx &c) {
  if (c.timers) cudaEventRecord(c.ev[10], c.stream);
  if (c.timers) cudaEventRecord(c.ev[11], c.stream);
  if (c.prec == CB2_PREC_MIXED) return leg_bwd_pack(c, kBwdSlots, mlayout(c, c.d_four, 4, 1));
  return 0;
}

static int nl_grid(Ctx &c) {
  if (c.timers) cudaEventRecord(c.ev[12], c.stream);
  const MLayout fin = mlayout(c, c.d_four, 4, 1), fout = mlayout(c, c.d_four2, 4, 0);
  const bool maxima = fft_products_m(c, fin, fout, mixed_fwd_pmax(c));
  if (c.timers) cudaEventRecord(c.ev[13], c.stream);
  leg_fwd_rowmax(c, fout, maxima);
  return 0;
}

static int nl_tail(Ctx &c) {
  if (c.timers) cudaEventRecord(c.ev[14], c.stream);
  rj_after_transform(c);
  if (c.closure) {
    int rc = closure_apply(c);
    if (rc) return rc;
  }
  if (c.timers) cudaEventRecord(c.ev[15], c.stream);
  return 0;
}

static int nonlinear(Ctx &c) {
  int rc = nl_head(c);
  if (rc) return rc;
  if (c.prec == CB2_PREC_FP64) {
    leg_bwd_f64(c, 4, 1, kBwdSlots, (double *)c.d_four);
    if (c.timers) cudaEventRecord(c.ev[12], c.stream);
    fft_products<double>(c, (const double *)c.d_four, (double *)c.d_four2);
    if (c.timers) cudaEventRecord(c.ev[13], c.stream);
    leg_fwd_f64(c, 4, 0, (const double *)c.d_four2, kFwdSlots);
  } else {
    if ((rc = leg_bwd_gemm(c, mlayout(c, c.d_four, 4, 1)))) return rc;
    if ((rc = nl_grid(c))) return rc;
    if ((rc = leg_fwd_gemm(c, mlayout(c, c.d_four2, 4, 0), kFwdSlots))) return rc;
  }
  return nl_tail(c);
}

static void temp_roundtrip(Ctx &c) {
  if (!c.p.use_ref_temp) return;
  k_temp_roundtrip<<<cdiv(c.nr, 128), 128, 0, c.stream>>>(c.nr, (size_t)c.jmax, c.d_reft0, c.fld(TEMP));
}

// explicit update and radial solves of a step
static void solve(Ctx &c) {
  c.istep += 1;
  if (c.timers) cudaEventRecord(c.ev[0], c.stream);
  if (c.cn_ready && c.tune[TUNE_CN] == 1) {
    // explicit update, solves and derived fields in one kernel
    if (c.timers) cudaEventRecord(c.ev[1], c.stream);
    cn_step(c, c.istep == 1);
  } else {
    rj_explicit(c, c.istep == 1);
    if (c.timers) cudaEventRecord(c.ev[1], c.stream);
    rj_implicit(c);
  }
  if (c.timers) cudaEventRecord(c.ev[2], c.stream);
}

int step_once(Ctx &c) {
  solve(c);
  int rc = nonlinear(c);
  temp_roundtrip(c);
  if (c.timers) cudaEventRecord(c.ev[3], c.stream);
  return rc;
}

int step_phase(Ctx &c, int phase) {
  if (c.prec != CB2_PREC_MIXED) {
    set_error("step_phase: mixed-precision contexts only");
    return CB2_ERR_ARG;
  }
  if (phase == 0) {
    solve(c);
    return nl_head(c);
  }
  if (phase == 1) return nl_grid(c);
  const int rc = nl_tail(c);
  temp_roundtrip(c);
  if (c.timers) cudaEventRecord(c.ev[3], c.stream);
  return rc;
}

int step_gemms_setup(const std::vector<Ctx *> &shells, MultiLeg **out) {
  return multi_leg_setup(shells, 4, 1, kFwdSlots, 4, 0, out);
}

static void accumulate_timers(Ctx &c) {
  if (!c.timers) return;
  cudaEventSynchronize(c.ev[3]);
  auto el = [&](int a, int b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev[a], c.ev[b]);
    return (double)ms;
  };
  c.stage_ms[6] += el(0, 1);
  c.stage_ms[7] += el(1, 2);
  c.stage_ms[13] += el(10, 11);
  c.stage_ms[22] += el(11, 12);
  c.stage_ms[24] += el(12, 13);
  c.stage_ms[23] += el(13, 14);
  c.stage_ms[17] += el(14, 15);
  c.stage_ms[0] += el(0, 3);
}

int check_status(Ctx &c) {
  int st = 0;
  CB2_CUDA(cudaMemcpyAsync(&st, c.d_status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  if (st & CB2_STATUS_PIPE_TIMEOUT) {
    set_error("a tensor-core Legendre pipeline wait ran out of time; the state is void");
    return CB2_ERR_TIMEOUT;
  }
  return 0;
}

static int host_stage(Ctx &c, size_t bytes) {
  if (c.h_stage_bytes >= bytes) return 0;
  if (c.h_stage) cudaFreeHost(c.h_stage);
  c.h_stage = nullptr;
  CB2_CUDA(cudaMallocHost(&c.h_stage, bytes));
  c.h_stage_bytes = bytes;
  return 0;
}

}  // namespace cb2

using namespace cb2;

extern "C" {

const char *cb2_last_error(void) { return g_err.c_str(); }

int cb2_create(const cb2_params *p, int precision, int device, cb2_ctx **out) {
  if (!p || !out) { set_error("null argument"); return CB2_ERR_ARG; }
  *out = nullptr;
  if (p->ltr < 1 || p->nr < 5 || p->nth < 4 || (p->nth & 1) || p->nph < 4 ||
      p->nth < p->ltr + 1 || p->nph < 2 * (p->ltr + 1)) {
    set_error("unsupported grid: need nr >= 5, even nth >= L+1, nph >= 2(L+1)");
    return CB2_ERR_ARG;
  }
  if (precision != CB2_PREC_FP64 && precision != CB2_PREC_MIXED) {
    set_error("unknown precision");
    return CB2_ERR_ARG;
  }
  if (device >= 0) CB2_CUDA(cudaSetDevice(device));
  cb2_ctx *c = new cb2_ctx();
  CB2_CUDA(cudaGetDevice(&c->device));
  c->p = *p;
  c->prec = precision;
  c->L = p->ltr; c->nth = p->nth; c->nph = p->nph; c->nr = p->nr;
  c->jmax = (p->ltr + 1) * (p->ltr + 1);
  c->nh = p->nth / 2;
  c->NS = 2 * (p->ltr + 1);
  c->kin = 0; c->kout = p->nr - 1;
  const char *tm = getenv("CB2_TIMERS");
  c->timers = tm && tm[0] == '1';
  if (const char *pw = getenv("CB2_PIPE_WAIT_NS")) c->pipe_wait_ns = strtoull(pw, nullptr, 10);
  int rc;
  auto fail = [&](int code) { cb2_destroy(c); return code; };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    delete c;
    return CB2_ERR_CUDA;
  }
  for (int i = 0; i < 64; i++) c->ev[i] = nullptr;
  if (c->timers)
    for (int i = 0; i < 16; i++) cudaEventCreate(&c->ev[i]);
  if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "cudaMalloc(status)"));
  if ((rc = setup_tables(*c))) return fail(rc);
  if ((rc = rj_lu_factorise(*c))) return fail(rc);
  if ((rc = cn_setup(*c))) return fail(rc);
  if ((rc = fft_setup(*c))) return fail(rc);
  size_t fs = c->fsize();
  if (cudaMalloc(&c->d_f, (size_t)NSLOT * fs * sizeof(double)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaMalloc(fields)"));
  cudaMemsetAsync(c->d_f, 0, (size_t)NSLOT * fs * sizeof(double), c->stream);
  size_t rows = (size_t)c->nth * c->nr * c->NS;
  // float64 rows [theta][k][c][s] (13 and 12 components), or the padded
  // order-major float32 layout of the mixed path
  const size_t b1 = (precision == CB2_PREC_FP64) ? rows * 13 * sizeof(double) : mlayout_floats(*c) * sizeof(float);
  const size_t b2 = (precision == CB2_PREC_FP64) ? rows * 12 * sizeof(double) : mlayout_floats(*c) * sizeof(float);
  if (cudaMalloc(&c->d_four, b1) != cudaSuccess ||
      cudaMalloc(&c->d_four2, b2) != cudaSuccess ||
      cudaMalloc(&c->d_ene, (7 * (size_t)c->jmax + 16) * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_tmp, fs * sizeof(double)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaMalloc(work)"));
  if (precision == CB2_PREC_MIXED && (rc = mixed_setup(*c))) return fail(rc);
  if ((rc = static_scratch_setup(c->device))) return fail(rc);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "set-up"));
  *out = c;
  return 0;
}

int cb2_destroy(cb2_ctx *c) {
  if (!c) return 0;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->prec == CB2_PREC_MIXED) mixed_free(*c);
  closure_free(*c);
  cn_free(*c);
  free_tables(*c);
  void *ptrs[] = {c->d_lu_vp, c->d_lu_vt, c->d_lu_bs, c->d_lu_bt, c->d_lu_t, c->d_pv_vp, c->d_pv_vt,
                  c->d_pv_bs, c->d_pv_bt, c->d_pv_t, c->d_status, c->d_tw_fft, c->d_tw_fft32, c->d_twp32, c->d_twf4, c->d_twf4_64, c->d_imp_map,
                  c->d_cn_lu, c->d_cn_tiles, c->d_f, c->d_four, c->d_four2, c->d_ene, c->d_tmp, c->d_host_state,
                  c->d_bnd_a, c->d_bnd_b, c->d_bnd_grid, c->d_bnd_tab};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  for (int i = 0; i < 64; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  for (cudaEvent_t e : c->copy_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

int cb2_init_fields(cb2_ctx *c, int kind, unsigned seed) {
  if (!c) return CB2_ERR_ARG;
  size_t fs = c->fsize();
  CB2_CUDA(cudaMemsetAsync(c->d_f, 0, (size_t)NSLOT * fs * sizeof(double), c->stream));
  RJArgs a = c->rj_args();
  if (kind == 1) {
    int jj44 = (c->L >= 4) ? jj_of(*c, 4, 4) : -1;
    int js = jj_of(*c, 1, 0), jt = (c->L >= 2) ? jj_of(*c, 2, 0) : -1;
    k_init_dbench1<<<cdiv(c->nr, 128), 128, 0, c->stream>>>(a, c->d_f, fs, jj44, js, jt);
  } else if (kind == 2) {
    // the same generator and draw order as the oracle's seeded state
    unsigned long long st = 0x5DEECE66DULL ^ ((unsigned long long)seed << 17);
    std::vector<int> jjs;
    std::vector<double> amp;
    int lmax = std::min(c->L, 8);
    for (int l = 1; l <= lmax; l++)
      for (int m = -l; m <= l; m++) {
        amp.push_back(0.1 * (2.0 * rng_uniform(&st) - 1.0) / sqrt((double)(2 * l + 1)));
        jjs.push_back(jj_of(*c, l, m));
      }
    int nb0 = (int)jjs.size();
    int lb = std::min(c->L, 3);
    for (int l = 1; l <= lb; l++)
      for (int m = -l; m <= l; m++) {
        amp.push_back((l == 1 && m == 0 ? 1.0e-2 : 1.0e-3) * (2.0 * rng_uniform(&st) - 1.0));
        jjs.push_back(jj_of(*c, l, m));
      }
    int *d_j = nullptr;
    double *d_a = nullptr;
    CB2_CUDA(cudaMalloc(&d_j, jjs.size() * sizeof(int)));
    CB2_CUDA(cudaMalloc(&d_a, amp.size() * sizeof(double)));
    CB2_CUDA(cudaMemcpyAsync(d_j, jjs.data(), jjs.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CB2_CUDA(cudaMemcpyAsync(d_a, amp.data(), amp.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_init_seeded<<<cdiv(c->nr, 128), 128, 0, c->stream>>>(a, c->d_f, fs, d_j, d_a, (int)jjs.size(), nb0);
    CB2_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(d_j);
    cudaFree(d_a);
  } else {
    set_error("unknown initial field kind");
    return CB2_ERR_ARG;
  }
  // perturbation temperature (sync_temp_by_per_temp_sph)
  if (c->p.use_ref_temp)
    k_temp_shift<<<cdiv(c->nr, 128), 128, 0, c->stream>>>(c->nr, (size_t)c->jmax, c->d_reft0, c->fld(TEMP), -1.0);
  CB2_CUDA(cudaGetLastError());
  return cb2_start(c);
}

int cb2_start(cb2_ctx *c) {
  if (!c) return CB2_ERR_ARG;
  c->terms_stale = false;
  rj_start_derived(*c);
  int rc = nonlinear(*c);
  if (rc) return rc;
  CB2_CUDA(cudaGetLastError());
  if ((rc = check_status(*c))) return rc;
  c->istep = 0;
  c->started = true;
  return 0;
}

// the nonlinear terms of the current state, when the last call left them out
static int fresh_terms(Ctx &c) {
  if (!c.terms_stale) return 0;
  int rc = nonlinear(c);
  if (rc) return rc;
  temp_roundtrip(c);
  c.terms_stale = false;
  return 0;
}

int cb2_step(cb2_ctx *c, int nsteps) {
  if (!c) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_step before cb2_start / cb2_init_fields"); return CB2_ERR_STATE; }
  if (int rc = fresh_terms(*c)) return rc;
  if (c->timers) for (int i = 0; i < 32; i++) c->stage_ms[i] = 0.0;
  for (int s = 0; s < nsteps; s++) {
    int rc = step_once(*c);
    if (rc) return rc;
    if (c->timers) accumulate_timers(*c);
  }
  CB2_CUDA(cudaGetLastError());
  return 0;
}

int cb2_step_graph(cb2_ctx *c, int nsteps) {
  if (!c) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_step_graph before cb2_start"); return CB2_ERR_STATE; }
  if (int rc = fresh_terms(*c)) return rc;
  // the first step is an Euler step and not captured
  int done = 0;
  if (c->istep == 0 && nsteps > 0) {
    int rc = step_once(*c);
    if (rc) return rc;
    done = 1;
  }
  if (done == nsteps) return 0;
  if (!c->graph_exec) {
    bool tm = c->timers;
    c->timers = false;
    cudaGraph_t g;
    CB2_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int save = c->istep;
    int rc = step_once(*c);
    c->istep = save;
    cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
    if (rc) {
      if (ec == cudaSuccess) cudaGraphDestroy(g);
      c->timers = tm;
      return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture");
    CB2_CUDA(cudaGraphInstantiate(&c->graph_exec, g, 0));
    cudaGraphDestroy(g);
    c->timers = tm;
  }
  for (int s = done; s < nsteps; s++) {
    CB2_CUDA(cudaGraphLaunch(c->graph_exec, c->stream));
    c->istep += 1;
  }
  return 0;
}

int cb2_time_steps(cb2_ctx *c, int nsteps, int use_graph, double *ms) {
  if (!c || !ms) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_time_steps before cb2_start"); return CB2_ERR_STATE; }
  cudaEvent_t e0, e1;
  CB2_CUDA(cudaEventCreate(&e0));
  CB2_CUDA(cudaEventCreate(&e1));
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  CB2_CUDA(cudaEventRecord(e0, c->stream));
  int rc = use_graph ? cb2_step_graph(c, nsteps) : cb2_step(c, nsteps);
  CB2_CUDA(cudaEventRecord(e1, c->stream));
  CB2_CUDA(cudaEventSynchronize(e1));
  float t = 0.0f;
  CB2_CUDA(cudaEventElapsedTime(&t, e0, e1));
  *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc ? rc : check_status(*c);
}

int cb2_sync(cb2_ctx *c) {
  if (!c) return CB2_ERR_ARG;
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(*c);
}

int cb2_istep(const cb2_ctx *c) { return c ? c->istep : -1; }

int cb2_energies(cb2_ctx *c, double out[7]) {
  if (!c || !out) return CB2_ERR_ARG;
  int rc = check_status(*c);
  return rc ? rc : rj_energies(*c, out);
}

int cb2_energy_spectra(cb2_ctx *c, double *out_l, double *out_m, double *out_lm) {
  if (!c || !out_l || !out_m || !out_lm) return CB2_ERR_ARG;
  int rc = check_status(*c);
  return rc ? rc : rj_energy_spectra(*c, out_l, out_m, out_lm);
}

int cb2_get_field_device(cb2_ctx *c, int slot, double *dev) {
  if (!c || slot < 0 || slot >= NSLOT || !dev) return CB2_ERR_ARG;
  size_t n = c->fsize();
  k_to_host_order<<<cdiv(n, 256), 256, 0, c->stream>>>(c->nr, c->jmax, c->d_perm, c->fld(slot), dev);
  CB2_CUDA(cudaGetLastError());
  return 0;
}

int cb2_set_field_device(cb2_ctx *c, int slot, const double *dev) {
  if (!c || slot < 0 || slot >= NSLOT || !dev) return CB2_ERR_ARG;
  size_t n = c->fsize();
  k_to_device_order<<<cdiv(n, 256), 256, 0, c->stream>>>(c->nr, c->jmax, c->d_perm, dev, c->fld(slot));
  CB2_CUDA(cudaGetLastError());
  return 0;
}

int cb2_get_field(cb2_ctx *c, int slot, double *host) {
  if (!c || !host) return CB2_ERR_ARG;
  size_t n = c->fsize();
  int rc = host_stage(*c, n * sizeof(double));
  if (rc) return rc;
  if ((rc = cb2_get_field_device(c, slot, c->d_tmp))) return rc;
  CB2_CUDA(cudaMemcpyAsync(c->h_stage, c->d_tmp, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(host, c->h_stage, n * sizeof(double));
  return 0;
}

int cb2_set_field(cb2_ctx *c, int slot, const double *host) {
  if (!c || !host) return CB2_ERR_ARG;
  size_t n = c->fsize();
  int rc = host_stage(*c, n * sizeof(double));
  if (rc) return rc;
  memcpy(c->h_stage, host, n * sizeof(double));
  CB2_CUDA(cudaMemcpyAsync(c->d_tmp, c->h_stage, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((rc = cb2_set_field_device(c, slot, c->d_tmp))) return rc;
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

// the fields one step reads and rewrites (explicit terms, Adams-Bashforth
// history and the evolved fields); everything else is derived inside the step
static const int kHostStateSlots[20] = {
    VORT, VORT + 2, WDIFF, WDIFF + 2, FORCES, FORCES + 2, PREMOM, PREMOM + 2,
    MAGNE, MAGNE + 2, BDIFF, BDIFF + 2, INDUCT, INDUCT + 2, PREUXB, PREUXB + 2,
    TEMP, TDIFF, HADV, PREHEAT};

int cb2_step_host_state(cb2_ctx *c, double *state, double out_energies[7]) {
  if (!c || !state) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_step_host_state before cb2_start"); return CB2_ERR_STATE; }
  size_t n = c->fsize(), bytes = 20 * n * sizeof(double);
  if (!c->d_host_state) CB2_CUDA(cudaMalloc(&c->d_host_state, bytes));
  // pinned caller buffers are copied directly, pageable ones through staging
  cudaPointerAttributes pa;
  bool pinned = cudaPointerGetAttributes(&pa, state) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (!pinned) {
    int rc = host_stage(*c, bytes);
    if (rc) return rc;
  }
  double *src = pinned ? state : c->h_stage;
  if (!pinned) memcpy(c->h_stage, state, bytes);
  CB2_CUDA(cudaMemcpyAsync(c->d_host_state, src, bytes, cudaMemcpyHostToDevice, c->stream));
  for (int q = 0; q < 20; q++)
    k_to_device_order<<<cdiv(n, 256), 256, 0, c->stream>>>(c->nr, c->jmax, c->d_perm,
                                                             c->d_host_state + q * n, c->fld(kHostStateSlots[q]));
  if (c->istep == 0) c->istep = 1;   // the loaded history makes this an Adams-Bashforth step
  c->terms_stale = false;            // the state carries its own nonlinear terms
  if (int rc = step_once(*c)) return rc;
  for (int q = 0; q < 20; q++)
    k_to_host_order<<<cdiv(n, 256), 256, 0, c->stream>>>(c->nr, c->jmax, c->d_perm,
                                                         c->fld(kHostStateSlots[q]), c->d_host_state + q * n);
  CB2_CUDA(cudaMemcpyAsync(src, c->d_host_state, bytes, cudaMemcpyDeviceToHost, c->stream));
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  if (!pinned) memcpy(state, c->h_stage, bytes);
  if (out_energies) return cb2_energies(c, out_energies);
  return 0;
}

// The reference's restart set (MHD_src/sph_MHD/set_sph_restart_IO.f90:62-142,
// written after trans_per_temp_to_temp_sph, so the temperature is the total
// one): velocity (S, dS/dr, T), temperature, magnetic field (S, dS/dr, T),
// previous_momentum (3), previous_induction (3), previous_heat (1).
static const int kRestartSlots[14] = {VELO, VELO + 1, VELO + 2, TEMP, MAGNE, MAGNE + 1, MAGNE + 2,
                                      PREMOM, PREMOM + 1, PREMOM + 2, PREUXB, PREUXB + 1, PREUXB + 2, PREHEAT};

__global__ void k_add_l0(int nr, size_t jmax, const double *reft0, double *T, double sign) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nr) T[(size_t)k * jmax] += sign * reft0[k];   // host order: j = 0 is l = m = 0
}

// Restart entries a step never writes: the dS/dr components of
// previous_momentum and previous_induction (entries 8 and 11; the explicit
// update keeps only the poloidal and toroidal history).  A host that keeps
// the restart set already holds their values after the step.
static bool restart_entry_kept(int q) { return q == 8 || q == 11; }

// consecutive runs [run[i][0], run[i][1]) of restart entries in [lo, hi)
// that a step reads (kept = false) or keeps (kept = true), for one copy per
// run; returns the number of runs
static int restart_runs(int lo, int hi, bool kept, int (&run)[14][2]) {
  int nrun = 0;
  for (int q = lo; q < hi;) {
    if (restart_entry_kept(q) != kept) { q++; continue; }
    int q1 = q;
    while (q1 < hi && restart_entry_kept(q1) == kept) q1++;
    run[nrun][0] = q;
    run[nrun++][1] = q1;
    q = q1;
  }
  return nrun;
}

// host restart state -> field slots (through the device staging
// d_host_state).  The first 7 entries are the state (velocity, temperature,
// magnetic field), the last 7 the Adams-Bashforth history.  Two halves: the
// state on the compute stream, and the history, which only the explicit
// update reads, on the copy stream after it (started by
// load_restart_state, placed in its slots by load_restart_history), so the
// history crosses PCIe while the nonlinear terms of the state are computed.
// Within the history the five entries the step reads go first (copy_ev[1]),
// the two it keeps after them (copy_ev[2]).
static int load_restart_state(Ctx &c, const double *state) {
  const size_t n = c.fsize(), half = 7 * n * sizeof(double);
  if (!c.d_host_state) CB2_CUDA(cudaMalloc(&c.d_host_state, 20 * n * sizeof(double)));
  if (!c.copy_stream) {
    CB2_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t &e : c.copy_ev) CB2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  CB2_CUDA(cudaMemcpyAsync(c.d_host_state, state, half, cudaMemcpyHostToDevice, c.stream));
  // the history after the state (so the two do not share the link), and
  // after this context's earlier work on the staging buffer
  CB2_CUDA(cudaEventRecord(c.copy_ev[0], c.stream));
  CB2_CUDA(cudaStreamWaitEvent(c.copy_stream, c.copy_ev[0], 0));
  int run[14][2];
  for (int kept = 0; kept < 2; kept++) {
    for (int i = 0, nrun = restart_runs(7, 14, kept, run); i < nrun; i++)
      CB2_CUDA(cudaMemcpyAsync(c.d_host_state + run[i][0] * n, state + run[i][0] * n,
                               (run[i][1] - run[i][0]) * n * sizeof(double), cudaMemcpyHostToDevice,
                               c.copy_stream));
    CB2_CUDA(cudaEventRecord(c.copy_ev[1 + kept], c.copy_stream));
  }
  // the total temperature back to the perturbation (sync_temp_by_per_temp_sph)
  if (c.p.use_ref_temp)
    k_add_l0<<<cdiv(c.nr, 128), 128, 0, c.stream>>>(c.nr, (size_t)c.jmax, c.d_reft0, c.d_host_state + 3 * n, -1.0);
  for (int q = 0; q < 7; q++)
    k_to_device_order<<<cdiv(n, 256), 256, 0, c.stream>>>(c.nr, c.jmax, c.d_perm, c.d_host_state + q * n,
                                                          c.fld(kRestartSlots[q]));
  CB2_CUDA(cudaGetLastError());
  return 0;
}

// the history entries the step reads (kept = false, after copy_ev[1]) or
// keeps (kept = true, after copy_ev[2]) into their slots
static int load_restart_history(Ctx &c, bool kept) {
  const size_t n = c.fsize();
  CB2_CUDA(cudaStreamWaitEvent(c.stream, c.copy_ev[kept ? 2 : 1], 0));
  for (int q = 7; q < 14; q++)
    if (restart_entry_kept(q) == kept)
      k_to_device_order<<<cdiv(n, 256), 256, 0, c.stream>>>(c.nr, c.jmax, c.d_perm, c.d_host_state + q * n,
                                                            c.fld(kRestartSlots[q]));
  CB2_CUDA(cudaGetLastError());
  return 0;
}

static int load_restart(Ctx &c, const double *state) {
  int rc = load_restart_state(c, state);
  if (!rc) rc = load_restart_history(c, false);
  return rc ? rc : load_restart_history(c, true);
}

// field slots -> host restart state.  After a cb2_step_restart_state step
// (after_step) the two entries the step keeps are not copied back (the host
// holds them already); their upload, which trails the rest of the history,
// is placed in its slots while the other twelve come down.
static int store_restart(Ctx &c, double *state, bool after_step = false) {
  const size_t n = c.fsize();
  if (!c.d_host_state) CB2_CUDA(cudaMalloc(&c.d_host_state, 20 * n * sizeof(double)));
  for (int q = 0; q < 14; q++)
    if (!after_step || !restart_entry_kept(q))
      k_to_host_order<<<cdiv(n, 256), 256, 0, c.stream>>>(c.nr, c.jmax, c.d_perm, c.fld(kRestartSlots[q]),
                                                          c.d_host_state + q * n);
  if (c.p.use_ref_temp)
    k_add_l0<<<cdiv(c.nr, 128), 128, 0, c.stream>>>(c.nr, (size_t)c.jmax, c.d_reft0, c.d_host_state + 3 * n, 1.0);
  CB2_CUDA(cudaGetLastError());
  int run[14][2] = {{0, 14}};
  const int nrun = after_step ? restart_runs(0, 14, false, run) : 1;
  for (int i = 0; i < nrun; i++)
    CB2_CUDA(cudaMemcpyAsync(state + run[i][0] * n, c.d_host_state + run[i][0] * n,
                             (run[i][1] - run[i][0]) * n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (after_step)
    if (int rc = load_restart_history(c, true)) return rc;
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  return check_status(c);
}

static int sht_common(cb2_ctx *c, int nvec, int nscal) {
  if (!c || nvec < 0 || nscal < 0 || nvec + nscal == 0 || 3 * nvec + nscal > 13) {
    set_error("sht: need 1..13 components");
    return CB2_ERR_ARG;
  }
  if (c->prec == CB2_PREC_MIXED && nvec + nscal > 8) {
    set_error("sht: the mixed precision path takes at most 8 vectors + scalars");
    return CB2_ERR_ARG;
  }
  return 0;
}

int cb2_sht_backward(cb2_ctx *c, int nvec, int nscal, const double *spec, double *grid) {
  int rc = sht_common(c, nvec, nscal);
  if (rc) return rc;
  int nc = 3 * nvec + nscal;
  size_t n = c->fsize(), gsz = (size_t)nc * c->nr * c->nth * c->nph;
  // spectra go to the work slots 20.. of the field array
  int slots[13];
  for (int g = 0; g < nvec; g++) slots[g] = MADV + 3 * g;
  for (int s = 0; s < nscal; s++) slots[nvec + s] = MADV + 3 * nvec + s;
  for (int q = 0; q < nc; q++)
    if ((rc = cb2_set_field(c, MADV + q, spec + q * n))) return rc;
  double *dgrid = nullptr;
  CB2_CUDA(cudaMalloc(&dgrid, gsz * sizeof(double)));
  if (c->prec == CB2_PREC_FP64) {
    leg_bwd_f64(*c, nvec, nscal, slots, (double *)c->d_four);
    fft_backward_grid<double>(*c, nc, (const double *)c->d_four, dgrid);
  } else {
    const MLayout l = mlayout(*c, c->d_four, nvec, nscal);
    if ((rc = leg_bwd_mixed(*c, slots, l))) { cudaFree(dgrid); return rc; }
    fft_backward_grid_m(*c, l, dgrid);
  }
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaMemcpyAsync(grid, dgrid, gsz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(dgrid);
  return check_status(*c);
}

int cb2_sht_forward(cb2_ctx *c, int nvec, int nscal, const double *grid, double *spec) {
  int rc = sht_common(c, nvec, nscal);
  if (rc) return rc;
  int nc = 3 * nvec + nscal;
  size_t n = c->fsize(), gsz = (size_t)nc * c->nr * c->nth * c->nph;
  int slots[13];
  for (int g = 0; g < nvec; g++) slots[g] = MADV + 3 * g;
  for (int s = 0; s < nscal; s++) slots[nvec + s] = MADV + 3 * nvec + s;
  double *dgrid = nullptr;
  CB2_CUDA(cudaMalloc(&dgrid, gsz * sizeof(double)));
  CB2_CUDA(cudaMemcpyAsync(dgrid, grid, gsz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (c->prec == CB2_PREC_FP64) {
    fft_forward_grid<double>(*c, nc, dgrid, (double *)c->d_four);
    leg_fwd_f64(*c, nvec, nscal, (const double *)c->d_four, slots);
  } else {
    const MLayout l = mlayout(*c, c->d_four, nvec, nscal);
    fft_forward_grid_m(*c, dgrid, l);
    if ((rc = leg_fwd_mixed(*c, l, slots))) { cudaFree(dgrid); return rc; }
  }
  CB2_CUDA(cudaGetLastError());
  CB2_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(dgrid);
  if ((rc = check_status(*c))) return rc;
  for (int q = 0; q < nc; q++)
    if ((rc = cb2_get_field(c, MADV + q, spec + q * n))) return rc;
  return 0;
}

int cb2_get_restart_state(cb2_ctx *c, double *state) {
  if (!c || !state) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_get_restart_state before cb2_start"); return CB2_ERR_STATE; }
  return store_restart(*c, state);
}

int cb2_set_restart_state(cb2_ctx *c, const double *state, int istep) {
  if (!c || !state || istep < 0) return CB2_ERR_ARG;
  int rc = load_restart(*c, state);
  if (rc) return rc;
  // set_sph_field_to_start + the first nonlinear terms
  if ((rc = cb2_start(c))) return rc;
  c->istep = istep;
  c->terms_stale = false;
  return 0;
}

int cb2_step_restart_state(cb2_ctx *c, double *state, double out_energies[7]) {
  if (!c || !state) return CB2_ERR_ARG;
  if (!c->started) { set_error("cb2_step_restart_state before cb2_start"); return CB2_ERR_STATE; }
  int rc = load_restart_state(*c, state);
  if (rc) return rc;
  rj_start_derived(*c);
  if ((rc = nonlinear(*c))) return rc;
  if ((rc = load_restart_history(*c, false))) return rc;   // the history has crossed meanwhile
  c->istep = std::max(c->istep, 1) + 1;     // the loaded history makes this an Adams-Bashforth step
  cn_stage(*c, false);
  // the nonlinear terms of the new state are left to the next call (or to
  // the next cb2_step, which computes them first)
  c->terms_stale = true;
  if ((rc = store_restart(*c, state, true))) return rc;
  return out_energies ? cb2_energies(c, out_energies) : 0;
}

int cb2_get_gauss(cb2_ctx *c, double *colat, double *weight) {
  if (!c) return CB2_ERR_ARG;
  memcpy(colat, c->h_colat.data(), c->nth * sizeof(double));
  memcpy(weight, c->h_wgt.data(), c->nth * sizeof(double));
  return 0;
}

int cb2_get_plm(cb2_ctx *c, int l, int m, double *p, double *dp) {
  if (!c || m < 0 || m > l || l > c->L) return CB2_ERR_ARG;
  int nh = c->nh;
  std::vector<double> a(nh), b(nh);
  size_t off = c->h_poff[m] + (size_t)(l - m) * nh;
  CB2_CUDA(cudaMemcpy(a.data(), c->d_Plt + off, nh * sizeof(double), cudaMemcpyDeviceToHost));
  CB2_CUDA(cudaMemcpy(b.data(), c->d_dPlt + off, nh * sizeof(double), cudaMemcpyDeviceToHost));
  double sg = ((l - m) % 2 == 0) ? 1.0 : -1.0;
  for (int i = 0; i < nh; i++) {
    p[i] = a[i];
    dp[i] = b[i];
    p[c->nth - 1 - i] = sg * a[i];
    dp[c->nth - 1 - i] = -sg * b[i];
  }
  return 0;
}

int cb2_alloc_pinned(size_t bytes, void **out) {
  if (!out) return CB2_ERR_ARG;
  CB2_CUDA(cudaMallocHost(out, bytes));
  return 0;
}

int cb2_free_pinned(void *p) {
  if (p) CB2_CUDA(cudaFreeHost(p));
  return 0;
}

static bool same_nocase(const char *a, const char *b) {
  for (; *a && *b; a++, b++)
    if (std::tolower((unsigned char)*a) != std::tolower((unsigned char)*b)) return false;
  return *a == 0 && *b == 0;
}

// trailing blanks of a Fortran character value are not part of the name
static std::string trimmed(const char *s) {
  std::string t(s);
  while (!t.empty() && (t.back() == ' ' || t.back() == '\t' || t.back() == '\0')) t.pop_back();
  return t;
}

int cb2_legendre_trans_mode(const char *ctl) {
  if (!ctl) return CB2_PREC_FP64;
  const std::string v = trimmed(ctl);
  if (same_nocase(v.c_str(), "B200_mixed") || same_nocase(v.c_str(), "B200_tcgen05")) return CB2_PREC_MIXED;
  return CB2_PREC_FP64;
}

int cb2_fft_library_known(const char *ctl) {
  if (!ctl) return 0;
  const std::string v = trimmed(ctl);
  static const char *known[] = {"fftpack", "ispack", "fftw", "fftw3", "fftw_single", "fftw3_single",
                                "fftw_field", "fftw3_field", "B200"};
  for (const char *k : known)
    if (same_nocase(v.c_str(), k)) return 1;
  return 0;
}

int cb2_stage_times(cb2_ctx *c, double ms[32]) {
  if (!c || !ms) return CB2_ERR_ARG;
  for (int i = 0; i < 32; i++) ms[i] = c->stage_ms[i];
  return 0;
}

}  // extern "C"
