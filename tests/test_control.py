"""The control-file reader builds the same coefficients as the reference's
construct_coefficient for the golden case, and rejects what it cannot run."""
import os

import pytest

from calypso_b200 import configs
from calypso_b200.control import (parse_control, shell_params_from_control,
                                  time_control)

GOLD = os.path.join(os.path.dirname(__file__), "golden", "dynamobench_case1")


def _read(name):
    with open(os.path.join(GOLD, name)) as f:
        return f.read()


def test_case1_params_match_named_config():
    p = shell_params_from_control(_read("control_MHD"), _read("control_sph_shell"))
    q = configs.dynamobench_case1()
    for k, v in q.items():
        if isinstance(v, float):
            assert p[k] == pytest.approx(v, rel=1e-15, abs=1e-15), k
        else:
            assert p[k] == v, k
    assert p["coef_buo"] == pytest.approx(65000.0)
    assert p["coef_cor"] == pytest.approx(2000.0)
    assert p["coef_lor"] == pytest.approx(200.0)


def test_time_control():
    t = time_control(_read("control_MHD"))
    assert t["i_step_finish"] == 100 and t["i_step_check"] == 50
    assert t["dt"] == 5e-5
    assert t["legendre_trans_loop"] == "SYMMETRIC_MATMUL"


def test_parser_blocks_and_arrays():
    txt = """
begin a_ctl
  ! comment
  key_ctl   'quoted value'   # trailing comment
  array  list_ctl  2
    list_ctl  One   1.0
    list_ctl  Two  -1.0
  end array list_ctl
  begin inner
    x_ctl 3
  end inner
end a_ctl
"""
    root = parse_control(txt)
    a = root.block("A_CTL")
    assert a.get("KEY_CTL") == "quoted value"
    assert a.array("list_ctl") == [["One", "1.0"], ["Two", "-1.0"]]
    assert a.block("inner").get("x_ctl") == "3"


def test_unbalanced_and_missing_number_rejected():
    with pytest.raises(ValueError):
        parse_control("begin a\n")
    bad = _read("control_MHD").replace("Ekman_number                     1.0e-3", "Ekmann 1.0e-3")
    with pytest.raises(ValueError):
        shell_params_from_control(bad, _read("control_sph_shell"))


def test_unsupported_boundary_rejected():
    bad = _read("control_MHD").replace("non_slip_sph  ICB", "free_slip_sph  ICB")
    with pytest.raises(ValueError):
        shell_params_from_control(bad, _read("control_sph_shell"))


def test_legendre_trans_loop_ctl_selects_the_precision():
    # the C ABI's mapping (no GPU work): the B200 names pick the mixed path,
    # every name of the reference and unknown values the float64 path (the
    # reference falls back to original_loop for an unknown value)
    from calypso_b200 import PREC_FP64, PREC_MIXED, fft_library_known, legendre_trans_mode
    assert legendre_trans_mode("B200_mixed") == PREC_MIXED
    assert legendre_trans_mode("b200_TCGEN05   ") == PREC_MIXED
    assert legendre_trans_mode("B200_fp64") == PREC_FP64
    for name in ("original_loop", "symmetric_matmul", "symmetric_BLAS_big", "test_loop", "no_such_loop", ""):
        assert legendre_trans_mode(name) == PREC_FP64, name
    for name in ("fftpack", "FFTW3", "fftw_single", "ispack", "B200"):
        assert fft_library_known(name), name
    assert not fft_library_known("cufft")


def test_precision_from_control_file():
    from calypso_b200 import PREC_FP64, PREC_MIXED
    from calypso_b200.control import precision_from_control
    txt = _read("control_MHD")
    assert precision_from_control(txt) == PREC_FP64          # 'SYMMETRIC_MATMUL'
    mixed = txt.replace("'SYMMETRIC_MATMUL'", "'B200_mixed'")
    assert mixed != txt
    assert precision_from_control(mixed) == PREC_MIXED
