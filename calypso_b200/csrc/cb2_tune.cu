// cb2_tune.cu -- kernel-variant autotuner and the batched ensemble of shells.
//
// Autotuner.  The reference chooses among its Legendre loop variants by
// timing each on the actual grid at start-up (select_legendre_transform,
// MHD_src/sph_MHD/sph_transforms_4_MHD.f90:309-426).  Here the variants are
// compile-time tile shapes and launch shapes of the GPU kernels (Tune in
// cb2_internal.cuh); cb2_autotune times every candidate of every tunable on
// the context's own buffers with CUDA events (one warm-up, best of three)
// and keeps the fastest.  It runs the transform stages, which overwrite the
// work fields, so it is only allowed before the fields are initialised.
//
// Ensemble.  Independent shells (any mix of truncations and parameters) are
// advanced together: each shell keeps its own context and stream, and one
// CUDA graph holds one time step of every shell as parallel branches
// (fork/join on events), so a single graph launch advances all shells and
// the small shells run concurrently instead of one after another.  Shells
// of one shape share one autotuning.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cb2_internal.cuh"

namespace cb2 {

static int time_stage(Ctx &c, int (*stage)(Ctx &), float *best_ms) {
  cudaEvent_t e0, e1;
  CB2_CUDA(cudaEventCreate(&e0));
  CB2_CUDA(cudaEventCreate(&e1));
  int rc = stage(c);   // warm-up (also first-launch set-up)
  float best = 1e30f;
  for (int it = 0; it < 3 && !rc; it++) {
    cudaEventRecord(e0, c.stream);
    rc = stage(c);
    cudaEventRecord(e1, c.stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = cuda_fail(cudaGetLastError(), "autotune timing"); break; }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = check_status(c);
  *best_ms = best;
  return rc;
}

static const int kBwdSlots[5] = {VELO, VORT, MAGNE, CURRENT, TEMP};
static const int kFwdSlots[4] = {MADV, LOR, VPIND, HFLUX};

static int stage_bwd_f64(Ctx &c) {
  leg_bwd_f64(c, 4, 1, kBwdSlots, (double *)c.d_four);
  CB2_CUDA(cudaGetLastError());
  return 0;
}
static int stage_fwd_f64(Ctx &c) {
  leg_fwd_f64(c, 4, 0, (const double *)c.d_four2, kFwdSlots);
  CB2_CUDA(cudaGetLastError());
  return 0;
}
static int stage_fft_f64(Ctx &c) {
  fft_products<double>(c, (const double *)c.d_four, (double *)c.d_four2);
  CB2_CUDA(cudaGetLastError());
  return 0;
}
static int stage_bwd_mixed(Ctx &c) {
  int rc = leg_bwd_mixed(c, kBwdSlots, mlayout(c, c.d_four, 4, 1));
  if (!rc) CB2_CUDA(cudaGetLastError());
  return rc;
}
static int stage_fft_mixed(Ctx &c) {
  fft_products_m(c, mlayout(c, c.d_four, 4, 1), mlayout(c, c.d_four2, 4, 0));
  CB2_CUDA(cudaGetLastError());
  return 0;
}

// the Crank-Nicolson stage of an Adams-Bashforth step, as the step runs it
static int stage_cn(Ctx &c) {
  cn_stage(c, false);
  CB2_CUDA(cudaGetLastError());
  return 0;
}

int autotune(Ctx &c) {
  struct Item {
    int which;
    std::vector<int> cand;
    int (*stage)(Ctx &);
  };
  std::vector<Item> items;
  if (c.prec == CB2_PREC_FP64) {
    items.push_back({TUNE_BWD_KT, {1, 2, 4}, stage_bwd_f64});
    items.push_back({TUNE_FWD_KT, {1, 2, 3}, stage_fwd_f64});
    // 384: the float64 four-step kernel (where nphi = 3 (L + 1)), 512: Stockham
    items.push_back({TUNE_FFT_THREADS, {384, 512}, stage_fft_f64});
  } else {
    items.push_back({TUNE_PACK_KC, {1, 2, 4}, stage_bwd_mixed});
    items.push_back({TUNE_FFT_THREADS, {384, 512, 256, 128}, stage_fft_mixed});
  }
  if (c.cn_ready) items.push_back({TUNE_CN, {0, 1}, stage_cn});
  for (const Item &it : items) {
    int best = c.tune[it.which];
    float best_ms = 1e30f;
    for (int v : it.cand) {
      c.tune[it.which] = v;
      float ms;
      int rc = time_stage(c, it.stage, &ms);
      if (rc) return rc;
      if (ms < best_ms) { best_ms = ms; best = v; }
    }
    c.tune[it.which] = best;
  }
  // the transforms above wrote the work fields: clear them again
  CB2_CUDA(cudaMemsetAsync(c.d_f, 0, (size_t)NSLOT * c.fsize() * sizeof(double), c.stream));
  CB2_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

}  // namespace cb2

using namespace cb2;

struct cb2_ensemble {
  std::vector<cb2_ctx *> shells;
  cudaStream_t stream = nullptr;         // fork / join stream of the graph
  cudaEvent_t fork[3] = {nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> join[3];      // per phase and shell
  cudaGraphExec_t graph = nullptr;
  int device = 0;
  // mixed-precision shells: each Legendre GEMM launched once for all shells
  // (between the shells' step phases) instead of once per shell.  Off by
  // default: on the 48-shell and 64-shell ensembles measured the joins
  // around the two launches cost more (3-4 % of the step) than the single
  // launches save in GEMM time (6 %)
  int batched = 0;
  MultiLeg *ml = nullptr;
};

extern "C" {

int cb2_autotune(cb2_ctx *c) {
  if (!c) { set_error("cb2_autotune: null context"); return CB2_ERR_ARG; }
  if (c->started) {
    set_error("cb2_autotune: call it before cb2_init_fields / cb2_start (it overwrites the work fields)");
    return CB2_ERR_STATE;
  }
  return autotune(*c);
}

int cb2_get_tuning(const cb2_ctx *c, int out[TUNE_N]) {
  if (!c || !out) { set_error("cb2_get_tuning: null argument"); return CB2_ERR_ARG; }
  for (int q = 0; q < TUNE_N; q++) out[q] = c->tune[q];
  return 0;
}

const char *cb2_tuning_note(const cb2_ctx *c) { return c ? c->cn_off_reason : ""; }

int cb2_set_tuning(cb2_ctx *c, const int in[TUNE_N]) {
  if (!c || !in) { set_error("cb2_set_tuning: null argument"); return CB2_ERR_ARG; }
  if (c->graph_exec) {
    set_error("cb2_set_tuning: the step graph is already captured");
    return CB2_ERR_STATE;
  }
  for (int q = 0; q < TUNE_N; q++)
    if (q != TUNE_CN || c->cn_ready) c->tune[q] = in[q];
  return 0;
}

int cb2_ensemble_destroy(cb2_ensemble *e) {
  if (!e) return 0;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  multi_leg_free(e->ml);
  for (cb2_ctx *c : e->shells) cb2_destroy(c);
  for (int ph = 0; ph < 3; ph++) {
    for (cudaEvent_t ev : e->join[ph])
      if (ev) cudaEventDestroy(ev);
    if (e->fork[ph]) cudaEventDestroy(e->fork[ph]);
  }
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return 0;
}

int cb2_ensemble_create(const cb2_params *ps, int n, int precision, int device, int autotune_shapes,
                        cb2_ensemble **out) {
  if (!ps || n <= 0 || !out) { set_error("cb2_ensemble_create: bad argument"); return CB2_ERR_ARG; }
  *out = nullptr;
  cb2_ensemble *e = new cb2_ensemble();
  auto fail = [&](int rc) { cb2_ensemble_destroy(e); return rc; };
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "cudaSetDevice"));
  cudaGetDevice(&e->device);
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "ensemble stream"));
  for (int ph = 0; ph < 3; ph++)
    if (cudaEventCreateWithFlags(&e->fork[ph], cudaEventDisableTiming) != cudaSuccess)
      return fail(cuda_fail(cudaGetLastError(), "ensemble event"));
  // shells of one shape (L, nr, nth, nph) share the first one's autotuning
  std::vector<int> first_of(n, -1);
  for (int i = 0; i < n; i++) {
    cb2_ctx *c = nullptr;
    int rc = cb2_create(&ps[i], precision, e->device, &c);
    if (rc) return fail(rc);
    e->shells.push_back(c);
    // small shells take a few SMs each (about eight tiles per CTA of the
    // persistent Legendre kernels), so the graph's branches run side by side
    if (n > 1) c->ws_tiles_per_cta = 8;
    for (int ph = 0; ph < 3; ph++) {
      cudaEvent_t ev;
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "ensemble event"));
      e->join[ph].push_back(ev);
    }
    for (int j = 0; j < i; j++)
      if (ps[j].ltr == ps[i].ltr && ps[j].nr == ps[i].nr && ps[j].nth == ps[i].nth && ps[j].nph == ps[i].nph) {
        first_of[i] = j;
        break;
      }
    if (autotune_shapes) {
      if (first_of[i] < 0) {
        if ((rc = autotune(*c))) return fail(rc);
      } else {
        // the kernel shapes, and the fused Crank-Nicolson choice where this
        // shell's factors allow it (same shape, possibly other operators)
        const int cn = c->tune[TUNE_CN];
        std::memcpy(c->tune, e->shells[first_of[i]]->tune, sizeof(c->tune));
        if (!c->cn_ready) c->tune[TUNE_CN] = cn;
      }
    }
  }
  *out = e;
  return 0;
}

int cb2_ensemble_set_batched(cb2_ensemble *e, int on) {
  if (!e) { set_error("cb2_ensemble_set_batched: null ensemble"); return CB2_ERR_ARG; }
  if ((on != 0) != (e->batched != 0) && e->graph) {
    // the step graph is captured again at the next cb2_ensemble_step
    CB2_CUDA(cudaStreamSynchronize(e->stream));
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  e->batched = on ? 1 : 0;
  return 0;
}

int cb2_ensemble_size(const cb2_ensemble *e) { return e ? (int)e->shells.size() : -1; }

cb2_ctx *cb2_ensemble_shell(cb2_ensemble *e, int i) {
  if (!e || i < 0 || i >= (int)e->shells.size()) return nullptr;
  return e->shells[i];
}

int cb2_ensemble_init_fields(cb2_ensemble *e, int kind, unsigned seed0) {
  if (!e) return CB2_ERR_ARG;
  for (size_t i = 0; i < e->shells.size(); i++) {
    int rc = cb2_init_fields(e->shells[i], kind, seed0 + (unsigned)i);
    if (rc) return rc;
  }
  return 0;
}

// nsteps steps of every shell: the first (Euler) step of a shell runs
// eagerly; the Adams-Bashforth steps replay one graph that holds a step of
// every shell as parallel branches
int cb2_ensemble_step(cb2_ensemble *e, int nsteps) {
  if (!e) return CB2_ERR_ARG;
  int done = 0;
  for (cb2_ctx *c : e->shells) {
    if (!c->started) { set_error("cb2_ensemble_step before cb2_ensemble_init_fields"); return CB2_ERR_STATE; }
  }
  if (nsteps <= 0) return 0;
  bool any_first = false;
  for (cb2_ctx *c : e->shells) any_first |= (c->istep == 0);
  if (any_first) {   // one eager step of every shell (Euler where it is a shell's first)
    for (cb2_ctx *c : e->shells) {
      int rc = step_once(*c);
      if (rc) return rc;
    }
    done = 1;
  }
  if (done == nsteps) return 0;
  if (!e->graph) {
    bool batched = e->batched != 0;
    for (cb2_ctx *c : e->shells) batched &= (c->prec == CB2_PREC_MIXED);
    if (batched && !e->ml) {
      std::vector<Ctx *> v(e->shells.begin(), e->shells.end());
      int rc = step_gemms_setup(v, &e->ml);
      if (rc) return rc;
    }
    cudaGraph_t g;
    CB2_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    std::vector<int> save(e->shells.size());
    std::vector<bool> tm(e->shells.size());
    for (size_t i = 0; i < e->shells.size(); i++) {
      save[i] = e->shells[i]->istep;
      tm[i] = e->shells[i]->timers;
      e->shells[i]->timers = false;
    }
    // batched: phase 0 of every shell, the backward GEMM of all, phase 1 of
    // every shell, the forward GEMM of all, phase 2 of every shell; else one
    // branch per shell holding its whole step
    const int nph = batched ? 3 : 1;
    // branches in order of decreasing work per step (L^3 nr), so the longest
    // chains start first and the joins wait less on a late start
    std::vector<size_t> order(e->shells.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    auto work = [&](size_t i) {
      const double l1 = e->shells[i]->L + 1.0;
      return l1 * l1 * l1 * e->shells[i]->nr;
    };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return work(x) > work(y); });
    for (int ph = 0; ph < nph && !rc; ph++) {
      cudaEventRecord(e->fork[ph], e->stream);
      for (size_t i : order) {
        if (rc) break;
        cb2_ctx *c = e->shells[i];
        cudaStreamWaitEvent(c->stream, e->fork[ph], 0);
        rc = batched ? step_phase(*c, ph) : step_once(*c);
        cudaEventRecord(e->join[ph][i], c->stream);
        cudaStreamWaitEvent(e->stream, e->join[ph][i], 0);
      }
      if (batched && ph == 0) multi_leg_bwd(e->ml, e->stream);
      if (batched && ph == 1) multi_leg_fwd(e->ml, e->stream);
    }
    for (size_t i = 0; i < e->shells.size(); i++) {
      e->shells[i]->istep = save[i];
      e->shells[i]->timers = tm[i];
    }
    cudaError_t ec = cudaStreamEndCapture(e->stream, &g);
    if (rc) {
      if (ec == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture (ensemble)");
    ec = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaGraphInstantiate (ensemble)");
  }
  // the shells' own streams must be idle before the graph runs
  for (cb2_ctx *c : e->shells) CB2_CUDA(cudaStreamSynchronize(c->stream));
  for (int s = done; s < nsteps; s++) {
    CB2_CUDA(cudaGraphLaunch(e->graph, e->stream));
    for (cb2_ctx *c : e->shells) c->istep += 1;
  }
  return 0;
}

int cb2_ensemble_sync(cb2_ensemble *e) {
  if (!e) return CB2_ERR_ARG;
  CB2_CUDA(cudaStreamSynchronize(e->stream));
  for (cb2_ctx *c : e->shells) {
    int rc = cb2_sync(c);
    if (rc) return rc;
  }
  return 0;
}

int cb2_ensemble_time_steps(cb2_ensemble *e, int nsteps, double *ms) {
  if (!e || !ms) return CB2_ERR_ARG;
  int rc = cb2_ensemble_sync(e);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  CB2_CUDA(cudaEventCreate(&e0));
  CB2_CUDA(cudaEventCreate(&e1));
  CB2_CUDA(cudaEventRecord(e0, e->stream));
  rc = cb2_ensemble_step(e, nsteps);
  CB2_CUDA(cudaEventRecord(e1, e->stream));
  CB2_CUDA(cudaEventSynchronize(e1));
  float t = 0.0f;
  cudaEventElapsedTime(&t, e0, e1);
  *ms = t;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc ? rc : cb2_ensemble_sync(e);
}

int cb2_ensemble_energies(cb2_ensemble *e, double *out) {
  if (!e || !out) return CB2_ERR_ARG;
  int rc = cb2_ensemble_sync(e);
  if (rc) return rc;
  for (size_t i = 0; i < e->shells.size(); i++)
    if ((rc = cb2_energies(e->shells[i], out + 7 * i))) return rc;
  return 0;
}

}  // extern "C"
