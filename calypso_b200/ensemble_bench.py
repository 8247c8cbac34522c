"""Throughput of the batched ensemble (48 shells: 16 x L31/Nr33, 16 x
L63/Nr65, 16 x L127/Nr97, seeded Rayleigh numbers in [80, 400]).

    python -m calypso_b200.ensemble_bench [--steps K] [--precision mixed|fp64] [--shells mixed48|l31x64]

prints one JSON line: shell-steps/s of the ensemble (one CUDA graph launch
per step) in its two forms -- each shell's whole step as one branch (the
default), and each tensor-core Legendre GEMM as one launch over the tiles
of all shells between per-shell branches of the other kernels (batched) --
and of the same shells stepped one after another with their own graphs, all
timed with CUDA events, and the autotuned kernel variants of each shape."""
from __future__ import annotations

import argparse
import json

from . import configs
from .sph_mhd import PREC_FP64, PREC_MIXED, Ensemble, SphMHD


def small_shells(n: int = 64, seed: int = 0) -> list:
    """n shells of the smallest ensemble shape (L31/Nr33, 48 x 96), Rayleigh
    numbers uniform in [80, 400] (seeded): an ensemble whose per-shell
    kernels are too small to fill the GPU."""
    import numpy as np
    rng = np.random.default_rng(seed)
    L, nr, nth, nph, dt = configs.ENSEMBLE_SHAPES[0]
    return [configs.shell_params(L, nr, nth, nph, E=1e-3, Ra=float(rng.uniform(80.0, 400.0)), dt=dt)
            for _ in range(n)]


def run(steps: int = 20, warmup: int = 3, per_shape: int = 16, precision: str = "mixed", device: int = 0,
        shells: str = "mixed48") -> dict:
    """shells: "mixed48" (config 3, per_shape shells of each of the three
    shapes) or "l31x64" (small_shells())."""
    prec = PREC_MIXED if precision == "mixed" else PREC_FP64
    params = configs.ensemble(per_shape) if shells == "mixed48" else small_shells()
    ens = Ensemble(params, prec, device=device, autotune=True)
    ens.init_fields(2, 1)
    ens.step(1 + warmup)
    ms = ens.time_steps(steps)          # the default form: one branch per shell
    ens.set_batched(True)
    ens.step(warmup)
    ms_batched = ens.time_steps(steps)
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
        "workload": f"ensemble_{n}_shells" + ("" if shells == "mixed48" else "_L31"), "precision": precision,
        "steps": steps,
        "shell_steps_per_s": n * steps / (ms / 1000.0),
        "ms_per_ensemble_step": ms / steps,
        "batched_shell_steps_per_s": n * steps / (ms_batched / 1000.0),
        "batched_over_branches": ms / ms_batched,
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
    ap.add_argument("--shells", default="mixed48", choices=["mixed48", "l31x64"])
    args = ap.parse_args(argv)
    print(json.dumps(run(args.steps, args.warmup, args.per_shape, args.precision, shells=args.shells)), flush=True)


if __name__ == "__main__":
    main()
