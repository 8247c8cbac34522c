"""ctypes front of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this module; the product (``calypso_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

# field slots, mirrors calypso_oracle.h
VELO, VORT, MAGNE, CURRENT, TEMP = 0, 3, 6, 9, 12
WDIFF, BDIFF, TDIFF = 13, 16, 19
MADV, LOR, VPIND, HFLUX = 20, 23, 26, 29
ROTINERT, ROTLOR, INDUCT, HADV, ROTCOR, ROTBUO = 32, 35, 38, 41, 42, 45
FORCES, PREMOM, PREUXB, PREHEAT = 48, 51, 54, 57
NFIELD = 58


class CaloParams(ctypes.Structure):
    _fields_ = [
        ("ltr", ctypes.c_int), ("nth", ctypes.c_int), ("nph", ctypes.c_int),
        ("nr", ctypes.c_int), ("radial_grid_type", ctypes.c_int),
        ("r_icb", ctypes.c_double), ("r_cmb", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("coef_imp_v", ctypes.c_double), ("coef_imp_t", ctypes.c_double),
        ("coef_imp_b", ctypes.c_double),
        ("coef_velo", ctypes.c_double), ("coef_d_velo", ctypes.c_double),
        ("coef_buo", ctypes.c_double), ("coef_cor", ctypes.c_double),
        ("coef_lor", ctypes.c_double),
        ("coef_temp", ctypes.c_double), ("coef_d_temp", ctypes.c_double),
        ("coef_magne", ctypes.c_double), ("coef_d_magne", ctypes.c_double),
        ("coef_induct", ctypes.c_double),
        ("use_ref_temp", ctypes.c_int),
        ("depth_high_t", ctypes.c_double), ("depth_low_t", ctypes.c_double),
        ("high_temp", ctypes.c_double), ("low_temp", ctypes.c_double),
        ("temp_icb", ctypes.c_double), ("temp_cmb", ctypes.c_double),
        ("nthreads", ctypes.c_int),
    ]


def build() -> str:
    """Compile liboracle.so from oracle/*.c with the Makefile beside it."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d = ctypes.c_double
        vp = ctypes.c_void_p
        L.calo_create.restype = vp
        L.calo_create.argtypes = [P(CaloParams)]
        L.calo_destroy.argtypes = [vp]
        for name, args in [
            ("calo_jmax", [vp]), ("calo_istep", [vp]),
            ("calo_init_fields", [vp, ctypes.c_int, ctypes.c_uint]),
            ("calo_step", [vp, ctypes.c_int]),
            ("calo_start", [vp]),
            ("calo_energies", [vp, P(d)]),
            ("calo_get_field", [vp, ctypes.c_int, P(d)]),
            ("calo_set_field", [vp, ctypes.c_int, P(d)]),
            ("calo_get_gauss", [vp, P(d), P(d)]),
            ("calo_get_radius", [vp, P(d)]),
            ("calo_get_plm", [vp, ctypes.c_int, ctypes.c_int, P(d), P(d)]),
            ("calo_get_gaunt", [vp, ctypes.c_int, P(d), P(d)]),
            ("calo_sht_backward", [vp, ctypes.c_int, ctypes.c_int, P(d), P(d)]),
            ("calo_sht_forward", [vp, ctypes.c_int, ctypes.c_int, P(d), P(d)]),
            ("calo_energy_spectra", [vp, P(d), P(d), P(d)]),
            ("calo_leg_backward", [vp, ctypes.c_int, ctypes.c_int, P(d), P(d)]),
            ("calo_leg_forward", [vp, ctypes.c_int, ctypes.c_int, P(d), P(d)]),
            ("calo_fft_backward", [vp, ctypes.c_int, P(d), P(d)]),
            ("calo_fft_forward", [vp, ctypes.c_int, P(d), P(d)]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        for name in ("calo_leadki", "calo_leadli"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_int] * 6
            f.restype = ctypes.c_double
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One spherical shell advanced by the CPU restatement of the reference."""

    def __init__(self, params: dict):
        self.params = dict(params)
        p = CaloParams()
        for k, v in params.items():
            setattr(p, k, v)
        self._p = p
        self._h = lib().calo_create(ctypes.byref(p))
        if not self._h:
            raise RuntimeError("calo_create failed")
        self.L = p.ltr
        self.nr, self.nth, self.nph = p.nr, p.nth, p.nph
        self.jmax = (self.L + 1) ** 2

    def close(self):
        if self._h:
            lib().calo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_fields(self, kind: int, seed: int = 0):
        if lib().calo_init_fields(self._h, kind, seed):
            raise RuntimeError("calo_init_fields failed")

    def start(self):
        lib().calo_start(self._h)

    def step(self, n: int = 1):
        lib().calo_step(self._h, n)

    @property
    def istep(self) -> int:
        return lib().calo_istep(self._h)

    def energies(self) -> np.ndarray:
        out = np.zeros(7)
        lib().calo_energies(self._h, _ptr(out))
        return out

    def energy_spectra(self) -> dict:
        """The seven energies by degree 'l', order 'm' and 'lm' = l - |m|,
        each an array (7, L+1)."""
        out = {k: np.zeros((7, self.L + 1)) for k in ("l", "m", "lm")}
        lib().calo_energy_spectra(self._h, _ptr(out["l"]), _ptr(out["m"]), _ptr(out["lm"]))
        return out

    def get_field(self, slot: int) -> np.ndarray:
        out = np.zeros((self.nr, self.jmax))
        lib().calo_get_field(self._h, slot, _ptr(out))
        return out

    def set_field(self, slot: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.nr, self.jmax)
        lib().calo_set_field(self._h, slot, _ptr(a))

    def gauss(self):
        c, w = np.zeros(self.nth), np.zeros(self.nth)
        lib().calo_get_gauss(self._h, _ptr(c), _ptr(w))
        return c, w

    def radius(self):
        r = np.zeros(self.nr)
        lib().calo_get_radius(self._h, _ptr(r))
        return r

    def plm(self, l: int, m: int):
        p, dp = np.zeros(self.nth), np.zeros(self.nth)
        lib().calo_get_plm(self._h, l, m, _ptr(p), _ptr(dp))
        return p, dp

    def gaunt(self, j: int):
        gi, ei = np.zeros(2), np.zeros(1)
        lib().calo_get_gaunt(self._h, j, _ptr(gi), _ptr(ei))
        return gi, ei

    def sht_backward(self, nvec: int, nscal: int, spec: np.ndarray) -> np.ndarray:
        nc = 3 * nvec + nscal
        spec = np.ascontiguousarray(spec, dtype=np.float64).reshape(nc, self.nr, self.jmax)
        grid = np.zeros((nc, self.nr, self.nth, self.nph))
        lib().calo_sht_backward(self._h, nvec, nscal, _ptr(spec), _ptr(grid))
        return grid

    def sht_forward(self, nvec: int, nscal: int, grid: np.ndarray) -> np.ndarray:
        nc = 3 * nvec + nscal
        grid = np.ascontiguousarray(grid, dtype=np.float64).reshape(nc, self.nr, self.nth, self.nph)
        spec = np.zeros((nc, self.nr, self.jmax))
        lib().calo_sht_forward(self._h, nvec, nscal, _ptr(grid), _ptr(spec))
        return spec


    # Legendre-only / FFT-only halves: Fourier arrays [c][k][theta][m + L]
    def leg_backward(self, nvec: int, nscal: int, spec: np.ndarray) -> np.ndarray:
        nc = 3 * nvec + nscal
        spec = np.ascontiguousarray(spec, dtype=np.float64).reshape(nc, self.nr, self.jmax)
        four = np.zeros((nc, self.nr, self.nth, 2 * self.L + 1))
        lib().calo_leg_backward(self._h, nvec, nscal, _ptr(spec), _ptr(four))
        return four

    def leg_forward(self, nvec: int, nscal: int, four: np.ndarray) -> np.ndarray:
        nc = 3 * nvec + nscal
        four = np.ascontiguousarray(four, dtype=np.float64).reshape(nc, self.nr, self.nth, 2 * self.L + 1)
        spec = np.zeros((nc, self.nr, self.jmax))
        lib().calo_leg_forward(self._h, nvec, nscal, _ptr(four), _ptr(spec))
        return spec

    def fft_backward(self, four: np.ndarray) -> np.ndarray:
        four = np.ascontiguousarray(four, dtype=np.float64)
        nc = four.shape[0]
        grid = np.zeros((nc, self.nr, self.nth, self.nph))
        lib().calo_fft_backward(self._h, nc, _ptr(four), _ptr(grid))
        return grid

    def fft_forward(self, grid: np.ndarray) -> np.ndarray:
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        nc = grid.shape[0]
        four = np.zeros((nc, self.nr, self.nth, 2 * self.L + 1))
        lib().calo_fft_forward(self._h, nc, _ptr(grid), _ptr(four))
        return four


def leadki(l1, m1, l2, m2, l3, m3) -> float:
    return lib().calo_leadki(l1, m1, l2, m2, l3, m3)


def leadli(l1, m1, l2, m2, l3, m3) -> float:
    return lib().calo_leadli(l1, m1, l2, m2, l3, m3)
