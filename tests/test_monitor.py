"""Monitor files in the reference's text format: fed the golden rows, the
writer reproduces the reference's own sph_pwr_volume_s.dat byte for byte;
the column comparison follows compare_sph_mean_square.f90 (relative
tolerance per column)."""
import json
import os

import numpy as np

from calypso_b200.monitor import MonitorFiles, compare_mean_square, fortran_e, read_mean_square

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dynamobench_case1")


def test_fortran_e_format():
    assert fortran_e(2.5e-3) == "  2.50000000000000E-003"
    assert fortran_e(12.0285080867821) == "  1.20285080867821E+001"
    assert fortran_e(0.0) == "  0.00000000000000E+000"
    assert fortran_e(-9.99999999999999999e-5) == " -1.00000000000000E-004"


def test_writer_reproduces_the_reference_file(tmp_path):
    with open(os.path.join(GOLD, "sph_pwr_volume_s.json")) as f:
        gold = json.load(f)
    m = MonitorFiles(str(tmp_path), L=31, nr=49)
    for row in gold["rows"]:
        m.write(row["step"], row["time"], row["values"])
    with open(os.path.join(GOLD, "sph_pwr_volume_s.dat")) as f:
        want = f.read()
    with open(tmp_path / "sph_pwr_volume_s.dat") as f:
        got = f.read()
    assert got == want


def test_compare_mean_square(tmp_path):
    ref = os.path.join(GOLD, "sph_pwr_volume_s.dat")
    rows = read_mean_square(ref)
    assert [r[0] for r in rows] == [50, 100]
    ok, worst = compare_mean_square(ref, ref)
    assert ok and max(w for _, w in worst) == 0.0
    m = MonitorFiles(str(tmp_path), L=31, nr=49)
    for step, time, vals in rows:
        m.write(step, time, [v * (1 + 2e-9) for v in vals])
    ok, _ = compare_mean_square(str(tmp_path / "sph_pwr_volume_s.dat"), ref, 1e-9)
    assert not ok
    ok, _ = compare_mean_square(str(tmp_path / "sph_pwr_volume_s.dat"), ref, 1e-8)
    assert ok


def test_spectra_files(tmp_path):
    m = MonitorFiles(str(tmp_path), L=3, nr=9, spectra=True)
    sp = {k: np.arange(28, dtype=float).reshape(7, 4) + 1 for k in ("l", "m", "lm")}
    m.write(10, 1e-3, np.arange(7) + 1.0, sp)
    for kind, label in (("l", "degree"), ("m", "order"), ("lm", "diff_deg_order")):
        lines = open(tmp_path / f"sph_pwr_volume_{kind}.dat").read().splitlines()
        assert lines[7].startswith(f"t_step    time    {label}    K_ene_pol")
        assert len(lines) == 8 + 4
        assert lines[8].split()[:3] == ["10", "1.00000000000000E-003", "0"]
