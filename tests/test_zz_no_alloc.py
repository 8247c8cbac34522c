"""cb2_energies_static (energies with no device allocation) against
cb2_energies, through the C ABI.  The file name sorts last so the test runs
after every other GPU test (and must also pass alone in a fresh process).

Tolerance: 1e-14 relative -- both entry points launch the same two kernels
in the same order, only the scratch buffer differs."""
import ctypes

import numpy as np
import pytest

from calypso_b200 import PREC_FP64, SphMHD, configs
from calypso_b200.sph_mhd import load_library

pytestmark = pytest.mark.gpu

TOL = 1e-14


def _static_entry():
    lib = load_library()
    f = lib.cb2_energies_static
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int
    return lib, f


def _call(f, g):
    out = np.zeros(7)
    rc = f(g._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0, load_library().cb2_last_error()
    return out


def test_energies_static_matches_energies_twice():
    _, f = _static_entry()
    g = SphMHD(configs.dynamobench_case1(), PREC_FP64)
    g.init_fields(1)
    g.step(3)
    ref = g.energies()
    for _ in range(2):                      # two calls in a row
        np.testing.assert_allclose(_call(f, g), ref, rtol=TOL, atol=0)
    g.step(2)
    ref = g.energies()
    first, second = _call(f, g), _call(f, g)
    np.testing.assert_allclose(first, ref, rtol=TOL, atol=0)
    np.testing.assert_allclose(second, ref, rtol=TOL, atol=0)
    g.close()


def _free_device_bytes():
    """cudaMemGetInfo's free bytes on the current device (the CUDA runtime
    the library itself loaded)."""
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def test_energies_static_allocates_nothing():
    # the context is created (which reserves the static scratch) and warmed
    # up first; after that, many calls leave the device's free memory as it was
    _, f = _static_entry()
    g = SphMHD(configs.dynamobench_case1(), PREC_FP64)
    g.init_fields(1)
    g.step(2)
    _call(f, g)
    before = _free_device_bytes()
    for _ in range(50):
        _call(f, g)
    assert _free_device_bytes() == before
    g.close()


def test_energies_static_rejects_truncation_beyond_scratch():
    lib, f = _static_entry()
    # L = 256: jmax = 66049 > 65536 (smallest grid the library accepts)
    p = configs.shell_params(256, 5, 258, 576, E=1e-3, Ra=100.0)
    g = SphMHD(p, PREC_FP64)
    out = np.zeros(7)
    rc = f(g._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == -1
    assert b"static scratch" in lib.cb2_last_error()
    g.close()
