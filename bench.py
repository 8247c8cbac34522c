#!/usr/bin/env python
"""Benchmark of the time-step hot path: simulated steps/s at L255 / Nr129.

Workload (named in config.workload): the full MHD time step of a spherical
shell at L=255, Nr=129, 384 Gauss nodes x 768 longitudes, E=1e-4, modified
Ra=300, Pr=1, Pm=5, dt=5e-6, seeded thermal perturbation on random l<=8
modes plus a weak dipole-dominated seed field (synthetic; the same generator
feeds the CPU oracle).  One "step" is one SPH_analyze_MHD call.

Arms
  (default)          this library on N GPUs (one replica shell per GPU, no
                     collective in the data path; launched by torchrun for N>1),
                     mixed precision unless --precision fp64.  The FP64 plain
                     path is timed beside it on the same GPU, and both paths
                     run --compare-steps steps (500) from the same seeded start
                     to report the relative energy error of the mixed path.
  --impl reference   the reference's algorithm restated on the CPU (the
                     oracle; the reference's Fortran build is unavailable in
                     this image), timed on the host cores, rank 0 only.

Extra keys of the default arm (rank 0, one GPU; each can be skipped):
fp64_plain (config 2 on the FP64 path), sht_roundtrip (config 1, per-field
errors), ensemble (config 3, 48 shells) and closure (config 4, the network
trained on filtered L255 runs and applied at L63).

Timing: W untimed warm-up steps, then K steps captured as a CUDA graph and
timed with CUDA events on the library's stream, bracketed by barriers and
device synchronisation; the max over ranks is reported.  The model state
(58 fields x 8.45e6 modes, 3.9 GB) is larger than L2, so no L2 flush is
needed between steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "steps/s at L255 Nr129: mixed-precision vs FP64 plain, same B200, rel err"
WORKLOAD = "full_step_L255_Nr129"


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def legendre_flops(L, nr, nth, nvec_b=4, nscal_b=1, nvec_f=4, nscal_f=0):
    """Algorithmic flops of the backward and forward Legendre transforms:
    U = 2 (Nth/2) Nr (L+1)^2 per scalar-equivalent column with the
    equatorial symmetry; a vector is 5 U, a scalar 1 U."""
    U = 2.0 * (nth / 2) * nr * (L + 1) ** 2
    return (5 * nvec_b + nscal_b) * U, (5 * nvec_f + nscal_f) * U


def max_over_ranks(ms, dist, device):
    """The job's time: the largest per-rank device time (replicas that share
    no data still finish together only when the slowest does)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(ms, steps, world):
    """Whole-job steps/s: every replica advances its own shell `steps` times."""
    return world * steps / (ms / 1000.0)


# the reference arm times at most this many steps (and warm-up steps): one
# oracle step at L255 / Nr129 takes about 5 s on 16 host cores
REF_MAX_STEPS, REF_MAX_WARMUP = 30, 5
DATA = "synthetic: seeded thermal perturbation (l<=8) + dipole seed field"


def workload_config(params, workload):
    """The workload both arms run (identical in both JSON lines)."""
    E = 2.0 / params["coef_cor"]
    return {"workload": workload, "L": params["ltr"], "Nr": params["nr"], "Ntheta": params["nth"],
            "Nphi": params["nph"], "dt": params["dt"], "E": E,
            "Ra": params["coef_buo"] * E / (1.0 - params["r_icb"] / params["r_cmb"]),
            "Pr": 1.0 / params["coef_d_temp"], "Pm": 1.0 / params["coef_d_magne"],
            "start": "seeded (kind 2, seed 1 + rank)",
            "l2": "state 3.9 GB > 126 MB L2, no flush needed"}


def oracle_steps(params, cores, n_warm, n_timed):
    """Wall time of n_timed oracle steps after n_warm (the first is the
    Euler step, so timed steps are Adams-Bashforth steps when n_warm >= 1)."""
    from oracle.calypso_oracle import Oracle
    p = dict(params)
    p["nthreads"] = cores
    o = Oracle(p)
    o.init_fields(2, 1)
    o.step(n_warm)
    t0 = time.perf_counter()
    o.step(n_timed)
    dt = time.perf_counter() - t0
    o.close()
    return dt


def run_reference(args, params):
    """The reference's algorithm on the host cores (oracle port), rank 0 only."""
    rank, _, world = env_rank()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    nw = max(1, min(args.warmup, REF_MAX_WARMUP))
    nt = max(1, min(args.steps, REF_MAX_STEPS))
    dt = oracle_steps(params, cores, nw, nt)
    v = nt / dt
    line = {
        "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world, "steps": nt,
        "warmup": nw, "ms_per_step": 1000.0 * dt / nt, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": workload_config(params, args.workload),
        "impl_config": {"precision": "fp64 (CPU)", "parallelism": f"openmp x{cores}"},
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{nt} Adams-Bashforth steps after {nw} warm-up steps "
                                   "(the first an Euler step), host wall clock"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's Fortran build is unavailable in this image (no Fortran "
                "compiler); this arm runs the oracle, its C restatement pinned to the "
                "reference's Dynamobench golden energies",
    }
    print(json.dumps(line), flush=True)


def stage_times(params, prec, tuning, rank, local_rank, nst=3):
    """Per-stage CUDA-event times (ms per step) of nst eager Adams-Bashforth
    steps on a fresh context (CB2_TIMERS), outside the timed run."""
    from calypso_b200 import SphMHD
    os.environ["CB2_TIMERS"] = "1"
    try:
        gt = SphMHD(params, prec, device=local_rank)
        gt.tuning = tuning
        gt.init_fields(2, seed=1 + rank)
        gt.step(1)
        gt.step(nst)
        st = gt.stage_times() / nst
        gt.close()
    finally:
        os.environ.pop("CB2_TIMERS", None)
    return st


def stage_dict(st, tuning):
    """Stage names of cb2_stage_times ids (the reference's timer labels)."""
    d = ({"cn_step": st[6] + st[7]} if tuning[4] == 1 else
         {"explicit": st[6], "implicit+rj_derived": st[7]})
    # (the Coriolis term is evaluated inside rj_after_transform)
    d.update({"legendre_bwd": st[22], "fft_products": st[24],
              "legendre_fwd": st[23], "rj_after_transform": st[17], "step": st[0]})
    return d


def dgemm_peak(local_rank):
    """Measured float64 GEMM throughput (cuBLAS through torch.matmul, 8192^3,
    best of 5), TFLOP/s: the yardstick of the FP64 Legendre stages."""
    try:
        import torch
        dev = f"cuda:{local_rank}"
        a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
        b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
        torch.matmul(a, b)
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def sht_roundtrip_extras(local_rank, with_oracle=True):
    """The isolated SHT round trip at L255 / 384 x 768 / Nr65, 3 vectors + 2
    scalars, seeded spectra with power falling as l^-2: wall time of the
    four routine-level calls (backward Legendre, backward FFT, forward FFT,
    forward Legendre; reference layouts, device buffers, each call
    synchronous) per precision, and the error of each field against the
    float64 GPU path and, when with_oracle, against the oracle (whose round
    trip is timed on the host cores too)."""
    import torch
    from calypso_b200 import PREC_FP64, PREC_MIXED, SphMHD, configs, sph_tables
    from calypso_b200.sph_mhd import rlm_size, rtm_size
    p = configs.sht_roundtrip()
    L, nr, nth, nph = p["ltr"], p["nr"], p["nth"], p["nph"]
    nvec, nscal = 3, 2
    nc = 3 * nvec + nscal
    spec = configs.sht_roundtrip_spectra(L, nr, nvec, nscal)
    t = sph_tables(L, nr, nth, nph)
    jg = np.array([l * (l + 1) + m for (l, m) in t.j_order])
    WR = np.zeros(rlm_size(t, nc))
    for c in range(nc):
        idx = c + nc * (np.arange(nr)[:, None] * t.istep_rlm[0] + np.arange(len(jg))[None, :] * t.istep_rlm[1])
        WR[idx] = spec[c][:, jg]
    dev = f"cuda:{local_rank}"
    dWR = torch.from_numpy(WR).to(dev)
    nnod = nr * nth * nph
    out = {"workload": "sht_roundtrip_L255_Nr65", "fields": "3 vectors + 2 scalars",
           "timer": "host wall clock around the four synchronous calls (device buffers), best of 3"}
    grids, backs = {}, {}
    for prec, name in ((PREC_FP64, "fp64"), (PREC_MIXED, "mixed")):
        g = SphMHD(p, prec, device=local_rank)
        four = torch.zeros(rtm_size(t, nc), dtype=torch.float64, device=dev)
        grid = torch.zeros(nnod * nc, dtype=torch.float64, device=dev)
        four2 = torch.zeros_like(four)
        back = torch.zeros(rlm_size(t, nc), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            g.sel_backward_legendre_trans(nc, nvec, nscal, dWR.data_ptr(), t, WS=four.data_ptr())
            g.back_MHD_FFT_sel_from_recv(nc, four.data_ptr(), t, fld_rtp=grid.data_ptr())
            g.fwd_MHD_FFT_sel_from_recv(nc, grid.data_ptr(), t, WS=four2.data_ptr())
            g.sel_forward_legendre_trans(nc, nvec, nscal, four2.data_ptr(), t, WS=back.data_ptr())
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[f"roundtrip_ms_{name}"] = 1e3 * best
        grids[name] = grid.view(nc, nnod).cpu().numpy()
        backs[name] = back.cpu().numpy()
        g.close()
        del four, grid, four2, back
    torch.cuda.empty_cache()
    fields = [list(range(3 * v, 3 * v + 3)) for v in range(nvec)] + [[3 * nvec + s] for s in range(nscal)]

    def err(a, b):
        return [float(np.linalg.norm(a[f] - b[f]) / np.linalg.norm(b[f])) for f in fields]
    out["grid_err_mixed_vs_fp64"] = err(grids["mixed"], grids["fp64"])
    rb = {k: v.reshape(-1, nc).T for k, v in backs.items()}
    out["roundtrip_err_mixed_vs_fp64"] = err(rb["mixed"], rb["fp64"])
    out["roundtrip_err_fp64_vs_input"] = err(rb["fp64"], WR.reshape(-1, nc).T)
    if with_oracle:
        from oracle.calypso_oracle import Oracle
        cores = os.cpu_count() or 1
        o = Oracle(dict(p, nthreads=cores))
        t0 = time.perf_counter()
        go = o.sht_backward(nvec, nscal, spec)
        so = o.sht_forward(nvec, nscal, go)
        out["cpu_roundtrip_s"] = time.perf_counter() - t0
        out["cpu_cores"] = cores
        o.close()
        # the library's grid in its default rtp layout: phi fastest, then theta, k
        gk = go.reshape(nc, -1)
        out["grid_err_fp64_vs_oracle"] = err(grids["fp64"], gk)
        out["grid_err_mixed_vs_oracle"] = err(grids["mixed"], gk)
        del go, so
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-sht", action="store_true", help="skip the SHT round-trip extra key")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 48-shell ensemble extra key")
    ap.add_argument("--no-closure", action="store_true", help="skip the learned-closure extra key")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel variants")
    ap.add_argument("--compare-steps", type=int, default=500,
                    help="steps of the mixed and FP64 runs whose energies are compared")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    from calypso_b200 import configs
    params = configs.CONFIGS[args.workload]()
    if args.impl == "reference":
        run_reference(args, params)
        return

    rank, local_rank, world = env_rank()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist

    from calypso_b200 import PREC_FP64, PREC_MIXED, SphMHD
    from calypso_b200.sph_mhd import RESTART_FIELDS_COMPS, PinnedArray

    prec = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    g = SphMHD(params, prec, device=local_rank)
    # the library's start-up autotuner picks the kernel variants (before the
    # fields exist); the stage-timer context and the FP64 context reuse it
    tuning = g.autotune() if not args.no_autotune else g.tuning
    tuning_note = g.tuning_note
    g.init_fields(2, seed=1 + rank)
    g.step(1)                                    # Euler first step
    g.step(args.warmup, graph=True)              # warm-up (graph capture + replays)
    g.sync()

    def barrier():
        if dist is not None:
            dist.barrier()

    clock = ClockSampler(local_rank)
    clock.start()
    barrier()
    ms = g.time_steps(args.steps, graph=True)
    barrier()
    clocks = clock.stop()
    ms = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    value = job_value(ms, args.steps, world)

    # stage breakdown (eager steps with per-stage CUDA events, not the timed run)
    st = stage_times(params, prec, tuning, rank, local_rank)

    L, nr, nth, nph = params["ltr"], params["nr"], params["nth"], params["nph"]
    fb, ff = legendre_flops(L, nr, nth)
    peaks, peak_kind = load_peaks()
    fused_cn = tuning[4] == 1
    stages = stage_dict(st, tuning)
    # dominant transform stage and its roofline.  Algorithmic bytes: one read
    # of each input and one write of each output (13 spectral slots and 13
    # Fourier components backward, 12 each forward); algorithmic flops:
    # legendre_flops.  The mixed Legendre stages execute their flops several
    # times on the tensor pipe (split products): 3 backward (hi*hi' + hi*lo'
    # + lo*hi'), 4 forward (the fixed-grid split adds lo*lo').
    es = 4 if prec == PREC_MIXED else 8
    spec_b = 13 * nr * (L + 1) ** 2 * 8
    spec_f = 12 * nr * (L + 1) ** 2 * 8
    four_b = (L + 1) * nth * nr * 26 * es
    four_f = (L + 1) * nth * nr * 24 * es
    traffic = {"legendre_bwd": spec_b + four_b, "fft_products": four_b + four_f,
               "legendre_fwd": four_f + spec_f}
    flops = {"legendre_bwd": fb, "legendre_fwd": ff}
    top = max(traffic, key=lambda k: stages[k])
    t_s = stages[top] * 1e-3
    achieved = traffic[top] / t_s / 1e9
    # DRAM bytes (read + write) of the dominant kernel from one ncu capture of
    # the same kernel at L255 / Nr33 (632.0 MB per launch), scaled by the
    # (theta, k) rows processed; other shapes have no capture
    dram_per_row = {("fft_products", 255, 384, 768): (338_202_368 + 293_795_072) / (384 * 33)}
    dkey = (top, L, nth, nph)
    measured = dram_per_row[dkey] * nth * nr if (prec == PREC_MIXED and dkey in dram_per_row) else None
    roof = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": measured,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at Nr33, scaled by rows"
                              if measured else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                           else "fallback 6650 GB/s",
            "algorithmic_bytes_per_launch": traffic[top],
            "per_stage": {}}
    for k in ("legendre_bwd", "fft_products", "legendre_fwd"):
        t = stages[k] * 1e-3
        ent = {"ms": stages[k], "bytes": traffic[k], "hbm_frac": traffic[k] / t / 1e9 / peaks["hbm_gbs"]}
        if k in flops:
            ent["flops"] = flops[k]
            if prec == PREC_MIXED:
                tp = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
                terms = 4 if k == "legendre_fwd" else 3
                ent["tensor_tflops_executed"] = terms * flops[k] / t / 1e12
                ent["tensor_frac_of_measured_sustained"] = terms * flops[k] / t / 1e12 / tp
            else:
                ent["fp64_tflops"] = flops[k] / t / 1e12
        roof["per_stage"][k] = ent

    # FP64 plain path on the same GPU: speed, and the energies of both paths
    # after the same number of steps from the same seeded start (the mixed
    # run continues the timed context)
    fp64 = None
    if prec == PREC_MIXED and not args.no_fp64_compare:
        ncmp = max(args.compare_steps, 1 + args.warmup + args.steps)
        g.step(ncmp - g.istep, graph=True)
        ene_mixed = g.energies()
        g64 = SphMHD(params, PREC_FP64, device=local_rank)
        if not args.no_autotune:
            g64.autotune()
        g64.init_fields(2, seed=1 + rank)
        g64.step(1)
        g64.step(args.warmup, graph=True)
        ms64 = g64.time_steps(args.steps, graph=True)
        g64.step(ncmp - g64.istep, graph=True)
        e64 = g64.energies()
        tuning64 = g64.tuning
        g64.close()
        st64 = stage_times(params, PREC_FP64, tuning64, rank, local_rank)
        rel = np.abs(ene_mixed - e64) / np.abs(e64)
        fp64 = {"steps_per_s": args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps,
                "speedup_mixed_over_fp64": (args.steps / (ms / 1000.0)) / (args.steps / (ms64 / 1000.0)),
                "compare_steps": ncmp,
                "energy_rel_err_max": float(rel.max()),
                "energy_rel_err": dict(zip(["K_pol", "K_tor", "K", "T2", "M_pol", "M_tor", "M"],
                                           [float(x) for x in rel])),
                "tuning": list(tuning64), "stages_ms": stage_dict(st64, tuning64),
                "legendre_fp64_tflops": {"legendre_bwd": fb / (st64[22] * 1e-3) / 1e12,
                                         "legendre_fwd": ff / (st64[23] * 1e-3) / 1e12}}
        dg = dgemm_peak(local_rank)
        if dg:
            fp64["fp64_dgemm_tflops_measured"] = dg
            fp64["legendre_frac_of_dgemm"] = {k: v / dg for k, v in fp64["legendre_fp64_tflops"].items()}

    # end to end through the C ABI with a host-resident state (pinned
    # buffers): the reference's restart set (14 rj fields) goes in, one
    # Adams-Bashforth step runs, the new restart set and the energies come out
    n = g.nr * g.jmax
    st_host = PinnedArray((len(RESTART_FIELDS_COMPS), g.nr, g.jmax))
    st_host.array[:] = g.get_restart_state()
    ke = max(1, min(args.steps, 5))
    g.step_restart_state(st_host.array)          # warm-up of the copy path
    t0 = time.perf_counter()
    for _ in range(ke):
        g.step_restart_state(st_host.array, with_energies=True)
    te = time.perf_counter() - t0
    nb = len(RESTART_FIELDS_COMPS) * n * 8
    # the dS/dr entries of previous_momentum and previous_induction are not
    # written by a step, so the call leaves them in the host buffer
    nb_out = (len(RESTART_FIELDS_COMPS) - 2) * n * 8
    e2e = {"value": world * ke / te, "unit": "steps/s",
           "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb_out + 7 * 8,
           "timer": "host wall clock around cb2_step_restart_state (restart set in, step, restart set and "
                    "energies out)",
           "steps": ke}

    sht = None
    if rank == 0 and world == 1 and not args.no_sht:
        sht = sht_roundtrip_extras(local_rank, with_oracle=not args.no_cpu_baseline)

    # config 3 (48-shell ensemble, one graph launch per ensemble step) and
    # config 4 (closure trained on filtered L255 runs, applied at L63)
    ens = clo = None
    if rank == 0 and world == 1 and not args.no_ensemble:
        from calypso_b200 import ensemble_bench
        ens = ensemble_bench.run(steps=10, warmup=3, device=local_rank)
    if rank == 0 and world == 1 and not args.no_closure:
        from calypso_b200 import closure_experiment
        clo = closure_experiment.run()
        clo.pop("loss_per_epoch", None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        nc = 3
        tc = oracle_steps(params, cores, 1, nc)
        cpu = {"value": nc / tc, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"{nc} Adams-Bashforth steps at L255/Nr129 after the Euler step, host wall clock"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp16-split tensor / f32 FFT / f64 solves" if prec == PREC_MIXED else "f64",
            "data": DATA,
            "config": workload_config(params, args.workload),
            "impl_config": {"precision": args.precision, "parallelism": f"replicas x{world}",
                            "graph": True, "tuning": list(tuning),
                            **({"tuning_note": tuning_note} if tuning_note else {})},
            "roofline": roof, "stages_ms": stages, "cpu_baseline": cpu, "e2e": e2e,
            "fp64_plain": fp64, "sht_roundtrip": sht, "ensemble": ens, "closure": clo,
            # kernels per step: the Crank-Nicolson stage (one fused kernel, or
            # explicit, implicit 5-band and 3-band, two derived-field kernels);
            # Coriolis; backward Legendre (pack + GEMM when mixed); FFT +
            # products; forward Legendre (row maxima + GEMM when mixed);
            # after-transform; reference-temperature shift
            "gpu_launches": ((13 if prec == PREC_MIXED else 11) - (4 if fused_cn else 0)
                             - (0 if params.get("use_ref_temp", 0) else 1)) * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
