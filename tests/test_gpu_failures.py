"""Failure paths, made on the host or by a wait that runs out -- no GPU
fault is caused:

  * a NaN planted in a field reaches the energy diagnostics, which return
    CB2_ERR_NAN (the reference's check_NaN_temperature,
    MHD_src/sph_MHD/cal_sol_sph_fluid_crank.f90:286-305);
  * a radial operator that cannot be factorised (a time step that is not
    finite makes every entry of the Crank-Nicolson matrix infinite) is
    rejected by the banded LU with CB2_ERR_SINGULAR (the reference's
    ludcmp_3band, SOLVER_src/direct_solver/m_ludcmp_3band.f90:118-121);
  * a tensor-core pipeline whose waits have a budget of zero (one try,
    CB2_PIPE_WAIT_NS=0) gives up at its first wait that is not complete:
    the kernels drain their copies and MMAs, free their tensor memory and
    return, and the call reports CB2_ERR_TIMEOUT.  The GPU stays usable: a
    new context afterwards steps normally."""
import math
import os

import numpy as np
import pytest

from calypso_b200 import PREC_FP64, PREC_MIXED, CalypsoError, SphMHD, configs
from calypso_b200.sph_mhd import ERR_NAN, ERR_SINGULAR, ERR_TIMEOUT, TEMP

pytestmark = pytest.mark.gpu


def test_nan_in_a_field_is_reported():
    g = SphMHD(configs.dynamobench_case1(), PREC_FP64)
    g.init_fields(1)
    g.step(2)
    assert np.all(np.isfinite(g.energies()))
    t = g.get_field(TEMP)
    t[g.nr // 2, 7] = float("nan")
    g.set_field(TEMP, t)
    with pytest.raises(CalypsoError) as e:
        g.energies()
    assert e.value.code == ERR_NAN
    # the NaN spreads through a step and is still reported
    g.step(1)
    with pytest.raises(CalypsoError) as e:
        g.energies()
    assert e.value.code == ERR_NAN


@pytest.mark.parametrize("dt", [math.inf, math.nan])
def test_operator_that_cannot_be_factorised_is_rejected(dt):
    p = configs.dynamobench_case1()
    p["dt"] = dt
    with pytest.raises(CalypsoError) as e:
        SphMHD(p, PREC_FP64)
    assert e.value.code == ERR_SINGULAR


def test_pipeline_wait_that_runs_out_is_reported(monkeypatch):
    p = configs.dynamobench_case1()
    monkeypatch.setenv("CB2_PIPE_WAIT_NS", "0")
    g = SphMHD(p, PREC_MIXED)
    monkeypatch.delenv("CB2_PIPE_WAIT_NS")
    with pytest.raises(CalypsoError) as e:
        g.init_fields(1)           # the start's nonlinear terms run the Legendre pipelines
        g.step(1)
        g.sync()
    assert e.value.code == ERR_TIMEOUT
    g.close()
    # a fresh context on the same GPU steps normally
    h = SphMHD(p, PREC_MIXED)
    h.init_fields(1)
    h.step(3)
    h.sync()
    assert np.all(np.isfinite(h.energies()))
