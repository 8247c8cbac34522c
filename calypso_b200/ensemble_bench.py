"""Throughput of the batched ensemble (48 shells: 16 x L31/Nr33, 16 x
L63/Nr65, 16 x L127/Nr97, seeded Rayleigh numbers in [80, 400]).

    python -m calypso_b200.ensemble_bench [--steps K] [--precision mixed|fp64]

prints one JSON line: shell-steps/s of the ensemble (one CUDA graph launch
per step) in its two forms -- each tensor-core Legendre GEMM as one launch
over the tiles of all 48 shells between per-shell branches of the other
kernels (batched), and each shell's whole step as one branch -- and of the
same shells stepped one after another with their own graphs, all timed with
CUDA events, and the autotuned kernel variants of each shape."""
from __future__ import annotations

import argparse
import json

from . import configs
from .sph_mhd import PREC_FP64, PREC_MIXED, Ensemble, SphMHD


def run(steps: int = 20, warmup: int = 3, per_shape: int = 16, precision: str = "mixed", device: int = 0) -> dict:
    prec = PREC_MIXED if precision == "mixed" else PREC_FP64
    params = configs.ensemble(per_shape)
    ens = Ensemble(params, prec, device=device, autotune=True)
    ens.init_fields(2, 1)
    ens.step(1 + warmup)
    ms = ens.time_steps(steps)
    ens.set_batched(False)
    ens.step(warmup)
    ms_branches = ens.time_steps(steps)
    tuning = {f"L{p['ltr']}": s.tuning for p, s in zip(params, ens.shells)}
    ens.close()
    # the same shells one after another (each its own captured graph)
    seq_ms = 0.0
    for q, p in enumerate(params):
        g = SphMHD(p, prec, device=device)
        g.tuning = tuning[f"L{p['ltr']}"]
        g.init_fields(2, 1 + q)
        g.step(1)
        g.step(warmup, graph=True)
        seq_ms += g.time_steps(steps, graph=True)
        g.close()
    n = len(params)
    return {
        "workload": f"ensemble_{n}_shells", "precision": precision, "steps": steps,
        "shell_steps_per_s": n * steps / (ms / 1000.0),
        "ms_per_ensemble_step": ms / steps,
        "legendre_launches_per_step": 2 if prec == PREC_MIXED else 2 * n,
        "branches_shell_steps_per_s": n * steps / (ms_branches / 1000.0),
        "batched_over_branches": ms_branches / ms,
        "sequential_shell_steps_per_s": n * steps / (seq_ms / 1000.0),
        "speedup_over_sequential": seq_ms / ms,
        "tuning": tuning,
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--per-shape", type=int, default=16)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    args = ap.parse_args(argv)
    print(json.dumps(run(args.steps, args.warmup, args.per_shape, args.precision)), flush=True)


if __name__ == "__main__":
    main()
