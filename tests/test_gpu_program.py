"""The program-level driver on the reference's own regression case: the
control files of tests/Dynamobench_case1 run through
calypso_b200.sph_mhd_program, and the monitor file it writes is compared
with the reference's sph_pwr_volume_s.dat column by column, as the
reference's test does with sph_ene_check (relative 1e-9); the mixed path
within 1e-6."""
import os
import shutil

import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED
from calypso_b200.monitor import compare_mean_square, read_mean_square
from calypso_b200.sph_mhd_program import run

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dynamobench_case1")


def _case(tmp_path):
    for name in ("control_MHD", "control_sph_shell"):
        shutil.copyfile(os.path.join(GOLD, name), tmp_path / name)
    return str(tmp_path)


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, 1e-9), (PREC_MIXED, 1e-6)])
def test_program_reproduces_reference_monitor_file(tmp_path, prec, tol):
    d = _case(tmp_path)
    r = run(d, precision=prec, graph=True, log=lambda *a: None)
    assert r["steps"] == 100
    out = os.path.join(d, "sph_pwr_volume_s.dat")
    assert [row[0] for row in read_mean_square(out)] == [50, 100]
    ok, worst = compare_mean_square(out, os.path.join(GOLD, "sph_pwr_volume_s.dat"), tol)
    assert ok, worst


def test_program_writes_spectra_when_asked(tmp_path):
    d = _case(tmp_path)
    txt = open(os.path.join(d, "control_MHD")).read()
    txt = txt.replace("end MHD_control", "  begin sph_monitor_ctl\n    volume_pwr_spectr_prefix  'sph_pwr_volume'\n"
                                         "    order_spectr_switch   'Off'\n  end sph_monitor_ctl\nend MHD_control")
    open(os.path.join(d, "control_MHD"), "w").write(txt)
    run(d, precision=PREC_FP64, steps=50, log=lambda *a: None)
    assert os.path.exists(os.path.join(d, "sph_pwr_volume_l.dat"))
    assert os.path.exists(os.path.join(d, "sph_pwr_volume_lm.dat"))
    assert not os.path.exists(os.path.join(d, "sph_pwr_volume_m.dat"))
    lines = open(os.path.join(d, "sph_pwr_volume_l.dat")).read().splitlines()
    assert len(lines) == 8 + 32          # header, then degrees 0..31 of step 50
