"""The C-ABI library builds, loads, and exports every entry point that
include/calypso_b200.h declares (no compute call: this runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cb2_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    from calypso_b200 import build, sph_mhd
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(sph_mhd.EXPORTS) <= set(names)


def test_error_reporting_without_gpu_work():
    from calypso_b200 import sph_mhd
    lib = sph_mhd.load_library()
    p = sph_mhd.Params()
    p.ltr, p.nth, p.nph, p.nr = 31, 47, 96, 33      # odd nth: rejected before any CUDA call
    h = ctypes.c_void_p()
    rc = lib.cb2_create(ctypes.byref(p), 0, -1, ctypes.byref(h))
    assert rc == -1
    assert b"unsupported grid" in lib.cb2_last_error()
