"""calypso_b200 -- B200 (sm_100a) time-step hot path of the Calypso MHD dynamo code.

The compute runs in libcalypso_b200.so (CUDA for sm_100a behind a C ABI,
include/calypso_b200.h); this package is the host side: the control-file
reader (:mod:`calypso_b200.control`), the named workloads
(:mod:`calypso_b200.configs`) and the ctypes binding that mirrors the
reference's module procedures (:mod:`calypso_b200.sph_mhd`).
"""
from .sph_mhd import (PREC_FP64, PREC_MIXED, CalypsoError, Ensemble, SphMHD, SphTables,  # noqa: F401
                      fft_library_known, legendre_trans_mode, load_library, sph_tables)
from . import configs, control  # noqa: F401

__all__ = ["SphMHD", "Ensemble", "CalypsoError", "PREC_FP64", "PREC_MIXED", "load_library",
           "SphTables", "sph_tables", "legendre_trans_mode", "fft_library_known", "configs", "control"]
