"""Learned subgrid closure experiment (the shells of the reference's
dynamo-benchmark physics at E = 1e-4, Ra = 300):

    python -m calypso_b200.closure_experiment [--small]

full:  high resolution L255 / Nr129 (mixed precision), 200 snapshots
       filtered to L63 / Nr65;
small: high resolution L63 / Nr33, 48 snapshots filtered to L31 / Nr17.
The last sixth of the snapshots is held out.  Prints one JSON line: training
loss per epoch, the fraction of the held-out subgrid tendency the network
explains, and the error of the low-resolution kinetic / magnetic energy
spectra against the filtered high-resolution run after `--horizon` steps,
plain solver vs. closure, from the last held-out snapshot."""
from __future__ import annotations

import argparse
import json
import time

from . import closure, configs
from .sph_mhd import PREC_MIXED, SphMHD


def shells(small: bool):
    if small:
        hi = configs.shell_params(63, 33, 96, 192, E=1e-4, Ra=300.0, dt=5e-6)
        lo = configs.shell_params(31, 17, 48, 96, E=1e-4, Ra=300.0, dt=5e-6)
        return hi, lo, 48, 4
    hi = configs.full_step_L255()
    lo = configs.shell_params(63, 65, 96, 192, E=1e-4, Ra=300.0, dt=5e-6)
    return hi, lo, 200, 5


def rollout_error(hi_src: SphMHD, p_lo, net, norm, alpha: float, horizon: int, ref_spectra):
    c = SphMHD(p_lo, PREC_MIXED, device=0)
    if alpha > 0:
        closure.attach(c, net, norm, alpha)
    closure.filter_fields(hi_src, c)
    c.step(horizon)
    try:
        err = closure.spectra_error(closure.energy_spectra(c), ref_spectra)
    except Exception:
        err = float("inf")
    c.close()
    return err if err == err else float("inf")


def run(small: bool = False, spin: int = 200, epochs: int = 4, horizon: int = 50, seed: int = 1,
        nhid: int = 256, batch: int = 16384, lr: float = 1e-3, alphas=(0.25, 0.5, 1.0)):
    p_hi, p_lo, n_snap, every = shells(small)
    t0 = time.time()
    hi = SphMHD(p_hi, PREC_MIXED, device=0)
    lo = SphMHD(p_lo, PREC_MIXED, device=0)
    hi.init_fields(2, seed)
    hi.step(spin, graph=True)
    xs, ys = closure.generate(hi, lo, n_snap, every)
    n_test = max(1, n_snap // 6)
    xtr, ytr, xte, yte = xs[:-n_test], ys[:-n_test], xs[-n_test:], ys[-n_test:]
    norm = closure.Normaliser(xtr, ytr, p_lo["nr"])
    net = closure.MLP(closure.NIN, nhid, closure.NOUT, seed=seed)
    t1 = time.time()
    hist = closure.train(net, xtr, ytr, norm, epochs=epochs, batch=batch, lr=lr, seed=seed)
    t2 = time.time()
    r2_train = closure.explained(net, norm, xtr[-n_test:], ytr[-n_test:])
    r2_test = closure.explained(net, norm, xte, yte)

    def errors_from_current(alist):
        """spectra errors after `horizon` steps from the current hi state:
        low-resolution rollouts from its filtered state against the filtered
        high-resolution state `horizon` steps later"""
        src = SphMHD(p_lo, PREC_MIXED, device=0)
        closure.filter_fields(hi, src)
        hi.step(horizon, graph=True)
        ref = SphMHD(p_lo, PREC_MIXED, device=0)
        closure.filter_fields(hi, ref)
        s_ref = closure.energy_spectra(ref)
        out = {a: rollout_error(src, p_lo, net, norm, a, horizon, s_ref) for a in alist}
        src.close()
        ref.close()
        return out

    # validation rollout picks the relaxation (0 = the plain solver, the fallback)
    val = errors_from_current((0.0,) + tuple(alphas))
    best = min(val, key=val.get)
    hi.step(every * 4, graph=True)
    test = errors_from_current((0.0, best) if best > 0 else (0.0,))
    return {
        "experiment": "closure_small" if small else "closure_L255_to_L63",
        "hi": {"L": p_hi["ltr"], "Nr": p_hi["nr"]}, "lo": {"L": p_lo["ltr"], "Nr": p_lo["nr"]},
        "snapshots": n_snap, "held_out": n_test, "samples_per_snapshot": int(xs[0].shape[0]),
        "net": {"layers": [closure.NIN, nhid, nhid, closure.NOUT], "weights": "bf16", "accumulate": "f32"},
        "epochs": epochs, "loss_per_epoch": hist, "explained_train": r2_train, "explained_held_out": r2_test,
        "horizon_steps": horizon, "validation_spectra_error": {str(k): v for k, v in val.items()},
        "alpha": best, "spectra_error_plain": test[0.0], "spectra_error_closure": test.get(best, test[0.0]),
        "data_s": t1 - t0, "train_s": t2 - t1,
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--small", action="store_true")
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--horizon", type=int, default=50)
    ap.add_argument("--spin", type=int, default=200)
    args = ap.parse_args(argv)
    print(json.dumps(run(args.small, spin=args.spin, epochs=args.epochs, horizon=args.horizon)), flush=True)


if __name__ == "__main__":
    main()
