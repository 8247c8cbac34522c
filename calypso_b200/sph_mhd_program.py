"""The time loop of the reference's ``sph_mhd`` program on the GPU.

    python -m calypso_b200.sph_mhd_program [DIR] [--precision fp64|mixed]
                                            [--steps N] [--graph]

reads ``DIR/control_MHD`` and ``DIR/control_sph_shell`` (the reference's
control files), sets the shell up (SPH_initialize_MHD,
src/programs/SPH_MHD/SPH_analyzer_MHD.f90:21-110), starts from the initial
field ``rst_ctl`` names, and advances from ``i_step_init_ctl`` to
``i_step_finish_ctl`` (SPH_analyze_MHD, :115-202: an Euler first step, then
Adams-Bashforth 2).  Every ``i_step_check_ctl`` steps it appends the volume
mean squares to ``DIR/sph_pwr_volume_s.dat`` (and the spectra files when
``sph_monitor_ctl`` names ``volume_pwr_spectr_prefix``), in the reference's
formats (:mod:`calypso_b200.monitor`).  The precision comes from
``Legendre_trans_loop_ctl`` unless ``--precision`` is given.

Initial fields (``rst_ctl``): ``dynamo_benchmark_1`` (the reference's
case-1 start), ``start_from_rst_file`` (the restart file of step
``i_step_init_ctl``) and ``B200_seeded`` (a seeded thermal perturbation on
l <= 8 plus a dipole-dominated seed field; no reference counterpart).
Every ``i_step_rst_ctl`` steps a restart file
``<restart_file_prefix>.<step / i_step_rst_ctl>.0.fst`` is written
(:mod:`calypso_b200.restart`).
"""
from __future__ import annotations

import argparse
import os
import time

from .control import parse_control, precision_from_control, shell_params_from_control, time_control
from .monitor import MonitorFiles
from .restart import read_restart, restart_file_name, write_restart
from .sph_mhd import PREC_FP64, PREC_MIXED, SphMHD

INIT_KINDS = {"dynamo_benchmark_1": 1, "b200_seeded": 2, "start_from_rst_file": 0}


def monitor_settings(mhd_text: str) -> dict:
    """sph_monitor_ctl (SERIAL_src/IO/m_ctl_data_4_pickup_sph.f90): the volume
    spectra prefix and the degree / order / l-m switches."""
    mon = parse_control(mhd_text).block("MHD_control", "sph_monitor_ctl")
    if mon is None:
        return {"spectra": False}

    def on(key):
        v = (mon.get(key) or "On").strip("'\"").lower()
        return v not in ("off", "no", "0")
    prefix = mon.get("volume_pwr_spectr_prefix")
    return {"spectra": prefix is not None, "volume_prefix": (prefix or "sph_pwr_volume").strip("'\""),
            "degree": on("degree_spectr_switch"), "order": on("order_spectr_switch"),
            "diff_lm": on("diff_lm_spectr_switch")}


def run(directory: str, precision: int | None = None, steps: int | None = None, graph: bool = False,
        device: int = -1, log=print) -> dict:
    with open(os.path.join(directory, "control_MHD")) as f:
        mhd = f.read()
    with open(os.path.join(directory, "control_sph_shell")) as f:
        shell = f.read()
    params = shell_params_from_control(mhd, shell)
    tc = time_control(mhd)
    prec = precision_from_control(mhd) if precision is None else precision
    rst = parse_control(mhd).block("MHD_control", "control", "restart_file_ctl")
    rst_ctl = ((rst.get("rst_ctl") if rst else None) or "dynamo_benchmark_1").strip("'\"").lower()
    if rst_ctl not in INIT_KINDS:
        raise ValueError(f"rst_ctl {rst_ctl!r} is not supported (supported: {', '.join(INIT_KINDS)})")
    mon = monitor_settings(mhd)
    files = MonitorFiles(directory, params["ltr"], params["nr"],
                         volume_prefix=mon.get("volume_prefix", "sph_pwr_volume"), spectra=mon["spectra"],
                         degree=mon.get("degree", True), order=mon.get("order", True),
                         diff_lm=mon.get("diff_lm", True))
    files_def = parse_control(mhd).block("MHD_control", "data_files_def")
    rst_prefix = ((files_def.get("restart_file_prefix") if files_def else None) or "restart/rst").strip("'\"")
    rst_prefix = os.path.join(directory, rst_prefix)
    i_rst = tc["i_step_rst"]
    g = SphMHD(params, prec, device=device)
    i0 = tc["i_step_init"]
    if INIT_KINDS[rst_ctl] == 0:
        if i_rst <= 0:
            raise ValueError("start_from_rst_file needs i_step_rst_ctl > 0")
        state, _, _, _ = read_restart(restart_file_name(rst_prefix, i0 // i_rst), g.nr, g.jmax)
        g.set_restart_state(state, i0)
    else:
        g.init_fields(INIT_KINDS[rst_ctl], 0)
    i1 = tc["i_step_finish"] if steps is None else i0 + steps
    check = tc["i_step_check"]
    dt = params["dt"]
    t0 = time.perf_counter()
    istep = i0
    while istep < i1:
        # advance to the next check or restart step (or the end) in one call
        nxt = i1
        for every in (check, i_rst):
            if every > 0:
                nxt = min(nxt, (istep // every + 1) * every)
        g.step(nxt - istep, graph=graph)
        istep = nxt
        if i_rst > 0 and istep % i_rst == 0:
            os.makedirs(os.path.dirname(rst_prefix) or ".", exist_ok=True)
            write_restart(restart_file_name(rst_prefix, istep // i_rst), g.get_restart_state(), istep,
                          istep * dt, dt)
        if check > 0 and istep % check == 0:
            e = g.energies()
            files.write(istep, istep * dt, e, g.energy_spectra() if mon["spectra"] else None)
            log(f"step {istep:8d}  time {istep * dt:.6e}  E_kin {e[2]:.8e}  E_mag {e[6]:.8e}")
    g.sync()
    wall = time.perf_counter() - t0
    out = {"steps": i1 - i0, "wall_s": wall, "precision": "mixed" if prec == PREC_MIXED else "fp64",
           "energies": g.energies().tolist()}
    g.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("directory", nargs="?", default=".")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default=None,
                    help="override Legendre_trans_loop_ctl")
    ap.add_argument("--steps", type=int, default=None, help="steps to run instead of the control file's")
    ap.add_argument("--graph", action="store_true", help="replay Adams-Bashforth steps from a CUDA graph")
    a = ap.parse_args()
    prec = None if a.precision is None else (PREC_MIXED if a.precision == "mixed" else PREC_FP64)
    r = run(a.directory, prec, a.steps, a.graph)
    print(f"{r['steps']} steps in {r['wall_s']:.3f} s ({r['precision']})")


if __name__ == "__main__":
    main()
