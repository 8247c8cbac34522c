"""Oracle pin: the CPU restatement reproduces the reference's own golden
energies of tests/Dynamobench_case1 (reference/sph_pwr_volume_s.dat) at the
reference's regression tolerance (compare_sph_mean_square.f90: 1e-9)."""
import json
import os

import numpy as np

from calypso_b200.control import shell_params_from_control

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dynamobench_case1")


def case1_params():
    with open(os.path.join(GOLD, "control_MHD")) as f:
        mhd = f.read()
    with open(os.path.join(GOLD, "control_sph_shell")) as f:
        shell = f.read()
    return shell_params_from_control(mhd, shell)


def test_oracle_reproduces_dynamobench_case1(oracle_lib):
    with open(os.path.join(GOLD, "sph_pwr_volume_s.json")) as f:
        gold = json.load(f)
    o = oracle_lib.Oracle(case1_params())
    o.init_fields(1)
    for row in gold["rows"]:
        o.step(row["step"] - o.istep)
        e = o.energies()
        ref = np.array(row["values"])
        rel = np.abs(e - ref) / np.abs(ref)
        assert rel.max() <= gold["rel_tol"], (row["step"], rel)
