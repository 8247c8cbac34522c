"""Host side of the B200 time-step hot path (ctypes over libcalypso_b200.so).

The class names and methods mirror the reference's module procedures so a
caller of the reference finds the same operations:

=============================  ==============================================
this module                    reference (src/Fortran_libraries/...)
=============================  ==============================================
``SphMHD(params)``             ``SPH_initialize_MHD`` set-up part
                               (programs/SPH_MHD/SPH_analyzer_MHD.f90:21-110)
``init_fields(kind, seed)``    ``sph_initial_data_control`` + ``set_sph_field_to_start``
                               + first ``nonlinear``
``SPH_analyze_MHD(n)``         ``SPH_analyze_MHD`` (SPH_analyzer_MHD.f90:115-202)
``energies()``                 ``cal_rms_sph_outer_core`` -> sph_pwr_volume_s.dat row
``sel_backward_legendre_trans``  the backward Legendre transform alone on the
                               reference's rlm / rtm buffers
                               (legendre_transform_select.f90:309-317)
``sel_forward_legendre_trans``   the forward Legendre transform alone
                               (legendre_transform_select.f90:375-383)
``back_MHD_FFT_sel_from_recv``   the backward FFT alone, rtm -> rtp
                               (MHD_FFT_selector.F90:219-249)
``fwd_MHD_FFT_sel_from_recv``    the forward FFT alone, rtp -> rtm
                               (MHD_FFT_selector.F90:185-215)
``sph_back_trans``             the whole backward transform, spectra (rj) to
                               grid (the Legendre and FFT stages of
                               sph_back_trans_4_MHD, sph_transforms_4_MHD.f90:152-172)
``sph_forward_trans``          the whole forward transform, grid to spectra
                               (sph_forward_trans_4_MHD, :176-195)
=============================  ==============================================

Errors come back as :class:`CalypsoError` (the reference aborts through
``calypso_MPI_abort``; the library never aborts the process).  There is no
CPU fallback: without the CUDA library this module raises on import of the
library, and every call runs on the GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcalypso_b200.so")

PREC_FP64 = 0
PREC_MIXED = 1

# d_rj slots of the evolved fields
VELO, VORT, MAGNE, CURRENT, TEMP = 0, 3, 6, 9, 12

# the reference's restart file: field names and components, in the order of
# the restart state (cb2_get_restart_state)
RESTART_FIELDS = [("velocity", 3), ("temperature", 1), ("magnetic_field", 3),
                  ("previous_momentum", 3), ("previous_induction", 3), ("previous_heat", 1)]
RESTART_FIELDS_COMPS = [(n, c) for n, nc in RESTART_FIELDS for c in range(nc)]

# kernel-variant tuning entries (cb2_get_tuning / cb2_set_tuning): float64
# backward radial tile, float64 forward radial tile, mixed pack radial tile,
# FFT kernel (384 four-step, else Stockham threads), fused Crank-Nicolson
# step (1) or separate kernels (0)
TUNE_BWD_KT, TUNE_FWD_KT, TUNE_PACK_KC, TUNE_FFT_THREADS, TUNE_CN = range(5)
TUNE_N = 5


# status codes of the C ABI (include/calypso_b200.h)
ERR_ARG, ERR_CUDA, ERR_SINGULAR, ERR_NAN, ERR_STATE, ERR_TIMEOUT = -1, -2, -3, -4, -5, -6


class CalypsoError(RuntimeError):
    """A failed library call; `code` is its CB2_ERR_* status."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


class SphTables(ctypes.Structure):
    """cb2_sph_tables: index tables of a single-domain grid in the form the
    reference's module m_spheric_parameter holds them (1-based values,
    column-major index arrays).  Build one with :func:`sph_tables`."""
    _fields_ = [
        ("nidx_rlm", ctypes.c_int * 2), ("istep_rlm", ctypes.c_int * 2),
        ("idx_gl_1d_rlm_j", ctypes.POINTER(ctypes.c_int)),
        ("nidx_rtm", ctypes.c_int * 3), ("istep_rtm", ctypes.c_int * 3),
        ("idx_gl_1d_rtm_m", ctypes.POINTER(ctypes.c_int)),
        ("nidx_rtp", ctypes.c_int * 3), ("istep_rtp", ctypes.c_int * 3),
    ]


def sph_tables(L: int, nr: int, nth: int, nph: int, j_order=None, m_order=None,
               istep_rlm=None, istep_rtm=None, istep_rtp=None) -> SphTables:
    """Index tables of a single-domain grid.  j_order: the (l, m) pairs of
    the rlm index j_rlm = 1.. (default: l(l+1)+m order); m_order: the orders
    of the rtm index mp = 1.. (default -L..L, so mp and nidx_rtm(3)-mp+1
    are the orders +-m as the reference's transforms pair them); strides
    default to the innermost index running fastest (j, then k; k, theta, m;
    phi, theta, k).  The arrays stay referenced by the returned object."""
    if j_order is None:
        j_order = [(l, m) for l in range(L + 1) for m in range(-l, l + 1)]
    if m_order is None:
        m_order = list(range(-L, L + 1))
    nj, nm = len(j_order), len(m_order)
    jt = np.zeros((3, nj), dtype=np.int32)          # column-major nj x 3
    for q, (l, m) in enumerate(j_order):
        jt[:, q] = (l * (l + 1) + m + 1, l, m)
    mt = np.zeros((2, nm), dtype=np.int32)
    for q, m in enumerate(m_order):
        mt[:, q] = (q + 1, m)
    t = SphTables()
    t.nidx_rlm[:] = (nr, nj)
    t.istep_rlm[:] = istep_rlm or (nj, 1)
    t.nidx_rtm[:] = (nr, nth, nm)
    t.istep_rtm[:] = istep_rtm or (1, nr, nr * nth)
    t.nidx_rtp[:] = (nr, nth, nph)
    t.istep_rtp[:] = istep_rtp or (nth * nph, nph, 1)
    t._jt, t._mt = np.ascontiguousarray(jt.reshape(-1)), np.ascontiguousarray(mt.reshape(-1))
    t.idx_gl_1d_rlm_j = t._jt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    t.idx_gl_1d_rtm_m = t._mt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    t.j_order, t.m_order = list(j_order), list(m_order)
    return t


def rlm_size(t: SphTables, ncomp: int) -> int:
    return ncomp * ((t.nidx_rlm[0] - 1) * t.istep_rlm[0] + (t.nidx_rlm[1] - 1) * t.istep_rlm[1] + 1)


def rtm_size(t: SphTables, ncomp: int) -> int:
    return ncomp * ((t.nidx_rtm[0] - 1) * t.istep_rtm[0] + (t.nidx_rtm[1] - 1) * t.istep_rtm[1]
                    + (t.nidx_rtm[2] - 1) * t.istep_rtm[2] + 1)


class Params(ctypes.Structure):
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


_lib = None

EXPORTS = [
    "cb2_last_error", "cb2_create", "cb2_destroy", "cb2_init_fields", "cb2_start",
    "cb2_step", "cb2_step_graph", "cb2_sync", "cb2_istep", "cb2_energies",
    "cb2_get_field", "cb2_set_field", "cb2_get_field_device", "cb2_set_field_device",
    "cb2_step_host_state", "cb2_sht_backward", "cb2_sht_forward", "cb2_get_gauss",
    "cb2_get_plm", "cb2_stage_times", "cb2_time_steps", "cb2_alloc_pinned", "cb2_free_pinned",
    "cb2_energies_static", "cb2_autotune", "cb2_get_tuning", "cb2_set_tuning",
    "cb2_ensemble_create", "cb2_ensemble_destroy", "cb2_ensemble_size", "cb2_ensemble_shell",
    "cb2_ensemble_init_fields", "cb2_ensemble_step", "cb2_ensemble_set_batched", "cb2_ensemble_sync", "cb2_ensemble_time_steps",
    "cb2_ensemble_energies", "cb2_leg_bwd", "cb2_leg_fwd", "cb2_fft_bwd", "cb2_fft_fwd",
    "cb2_legendre_trans_mode", "cb2_fft_library_known", "cb2_energy_spectra", "cb2_fft_products",
    "cb2_get_restart_state", "cb2_set_restart_state", "cb2_step_restart_state", "cb2_tuning_note",
]


def load_library(path: str = LIB_PATH):
    """Load libcalypso_b200.so and declare its C ABI; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CalypsoError(
            f"{path} is missing: build it with `python -m calypso_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(path)
    P, d, vp, i = ctypes.POINTER, ctypes.c_double, ctypes.c_void_p, ctypes.c_int
    pd = P(d)
    sig = {
        "cb2_last_error": ([], ctypes.c_char_p),
        "cb2_create": ([P(Params), i, i, P(vp)], i),
        "cb2_destroy": ([vp], i),
        "cb2_init_fields": ([vp, i, ctypes.c_uint], i),
        "cb2_start": ([vp], i),
        "cb2_step": ([vp, i], i),
        "cb2_step_graph": ([vp, i], i),
        "cb2_sync": ([vp], i),
        "cb2_istep": ([vp], i),
        "cb2_energies": ([vp, pd], i),
        "cb2_get_field": ([vp, i, pd], i),
        "cb2_set_field": ([vp, i, pd], i),
        "cb2_get_field_device": ([vp, i, vp], i),
        "cb2_set_field_device": ([vp, i, vp], i),
        "cb2_step_host_state": ([vp, pd, pd], i),
        "cb2_sht_backward": ([vp, i, i, pd, pd], i),
        "cb2_sht_forward": ([vp, i, i, pd, pd], i),
        "cb2_get_gauss": ([vp, pd, pd], i),
        "cb2_get_plm": ([vp, i, i, pd, pd], i),
        "cb2_stage_times": ([vp, pd], i),
        "cb2_time_steps": ([vp, i, i, pd], i),
        "cb2_alloc_pinned": ([ctypes.c_size_t, P(vp)], i),
        "cb2_free_pinned": ([vp], i),
        "cb2_energies_static": ([vp, pd], i),
        "cb2_autotune": ([vp], i),
        "cb2_get_tuning": ([vp, P(i)], i),
        "cb2_tuning_note": ([vp], ctypes.c_char_p),
        "cb2_set_tuning": ([vp, P(i)], i),
        "cb2_ensemble_create": ([P(Params), i, i, i, i, P(vp)], i),
        "cb2_ensemble_destroy": ([vp], i),
        "cb2_ensemble_size": ([vp], i),
        "cb2_ensemble_shell": ([vp, i], vp),
        "cb2_ensemble_init_fields": ([vp, i, ctypes.c_uint], i),
        "cb2_ensemble_step": ([vp, i], i),
        "cb2_ensemble_set_batched": ([vp, i], i),
        "cb2_ensemble_sync": ([vp], i),
        "cb2_ensemble_time_steps": ([vp, i, pd], i),
        "cb2_ensemble_energies": ([vp, pd], i),
        "cb2_leg_bwd": ([vp, P(SphTables), i, i, i, ctypes.c_size_t, ctypes.c_size_t, vp, vp], i),
        "cb2_leg_fwd": ([vp, P(SphTables), i, i, i, ctypes.c_size_t, ctypes.c_size_t, vp, vp], i),
        "cb2_fft_bwd": ([vp, P(SphTables), i, ctypes.c_size_t, vp, vp], i),
        "cb2_fft_fwd": ([vp, P(SphTables), i, vp, ctypes.c_size_t, vp], i),
        "cb2_legendre_trans_mode": ([ctypes.c_char_p], i),
        "cb2_fft_library_known": ([ctypes.c_char_p], i),
        "cb2_energy_spectra": ([vp, pd, pd, pd], i),
        "cb2_fft_products": ([vp, P(SphTables), ctypes.c_size_t, vp, ctypes.c_size_t, vp], i),
        "cb2_get_restart_state": ([vp, pd], i),
        "cb2_set_restart_state": ([vp, pd, i], i),
        "cb2_step_restart_state": ([vp, pd, pd], i),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise CalypsoError("arrays passed to the library must be C-contiguous float64")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc: int, what: str):
    if rc != 0:
        msg = load_library().cb2_last_error().decode(errors="replace")
        raise CalypsoError(f"{what} failed ({rc}): {msg}", rc)


class SphMHD:
    """One spherical shell advanced on the GPU (device-resident state)."""

    def __init__(self, params: dict, precision: int = PREC_FP64, device: int = -1):
        lib = load_library()
        p = Params()
        for k, v in params.items():
            setattr(p, k, v)
        h = ctypes.c_void_p()
        _check(lib.cb2_create(ctypes.byref(p), precision, device, ctypes.byref(h)), "cb2_create")
        self._h = h
        self.params = dict(params)
        self.precision = precision
        self.L, self.nr, self.nth, self.nph = p.ltr, p.nr, p.nth, p.nph
        self.jmax = (self.L + 1) ** 2

    @classmethod
    def _wrap(cls, handle, params: dict, precision: int):
        """A non-owning view of a context that belongs to an Ensemble."""
        self = cls.__new__(cls)
        self._h = ctypes.c_void_p(handle)
        self._owned = False
        self.params = dict(params)
        self.precision = precision
        self.L, self.nr, self.nth, self.nph = params["ltr"], params["nr"], params["nth"], params["nph"]
        self.jmax = (self.L + 1) ** 2
        return self

    # --- lifetime -----------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value and getattr(self, "_owned", True):
            load_library().cb2_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- time stepping ------------------------------------------------
    def init_fields(self, kind: int = 1, seed: int = 0):
        _check(load_library().cb2_init_fields(self._h, kind, seed), "cb2_init_fields")

    def start(self):
        _check(load_library().cb2_start(self._h), "cb2_start")

    def SPH_analyze_MHD(self, nsteps: int = 1, graph: bool = False):
        f = load_library().cb2_step_graph if graph else load_library().cb2_step
        _check(f(self._h, nsteps), "cb2_step")

    step = SPH_analyze_MHD

    def time_steps(self, nsteps: int, graph: bool = True) -> float:
        """Device time (ms) of nsteps, CUDA events on the library's stream."""
        ms = ctypes.c_double()
        _check(load_library().cb2_time_steps(self._h, nsteps, 1 if graph else 0, ctypes.byref(ms)),
               "cb2_time_steps")
        return ms.value

    def sync(self):
        _check(load_library().cb2_sync(self._h), "cb2_sync")

    # --- kernel-variant autotuning (before init_fields) -----------------
    def autotune(self) -> list:
        _check(load_library().cb2_autotune(self._h), "cb2_autotune")
        return self.tuning

    @property
    def tuning(self) -> list:
        out = (ctypes.c_int * TUNE_N)()
        _check(load_library().cb2_get_tuning(self._h, out), "cb2_get_tuning")
        return list(out)

    @property
    def tuning_note(self) -> str:
        """Why the one-kernel Crank-Nicolson step is off ('' when available)."""
        return load_library().cb2_tuning_note(self._h).decode(errors="replace")

    @tuning.setter
    def tuning(self, values):
        # entries not given keep their current values
        vals = list(values)
        vals += self.tuning[len(vals):]
        arr = (ctypes.c_int * TUNE_N)(*vals[:TUNE_N])
        _check(load_library().cb2_set_tuning(self._h, arr), "cb2_set_tuning")

    @property
    def istep(self) -> int:
        return load_library().cb2_istep(self._h)

    def energies(self) -> np.ndarray:
        out = np.zeros(7)
        _check(load_library().cb2_energies(self._h, _ptr(out)), "cb2_energies")
        return out

    def energy_spectra(self) -> dict:
        """The seven energies of energies() by degree 'l', order 'm' and
        'lm' = l - |m|: arrays (7, L+1) (sph_pwr_volume_l/_m/_lm.dat)."""
        out = {k: np.zeros((7, self.L + 1)) for k in ("l", "m", "lm")}
        _check(load_library().cb2_energy_spectra(self._h, _ptr(out["l"]), _ptr(out["m"]), _ptr(out["lm"])),
               "cb2_energy_spectra")
        return out

    def stage_times(self) -> np.ndarray:
        out = np.zeros(32)
        _check(load_library().cb2_stage_times(self._h, _ptr(out)), "cb2_stage_times")
        return out

    # --- fields -------------------------------------------------------
    def get_field(self, slot: int) -> np.ndarray:
        out = np.zeros((self.nr, self.jmax))
        _check(load_library().cb2_get_field(self._h, slot, _ptr(out)), "cb2_get_field")
        return out

    def set_field(self, slot: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.nr, self.jmax)
        _check(load_library().cb2_set_field(self._h, slot, _ptr(a)), "cb2_set_field")

    def step_host_state(self, state: np.ndarray, with_energies: bool = True):
        """One step with the 20-field host-resident state (cb2_step_host_state)."""
        ene = np.zeros(7)
        _check(load_library().cb2_step_host_state(
            self._h, _ptr(state), _ptr(ene) if with_energies else None), "cb2_step_host_state")
        return ene

    # --- restart state (the fields of the reference's restart file) ---------
    def get_restart_state(self) -> np.ndarray:
        """(14, nr, jmax): velocity (3), total temperature, magnetic field
        (3), previous_momentum (3), previous_induction (3), previous_heat."""
        out = np.zeros((len(RESTART_FIELDS_COMPS), self.nr, self.jmax))
        _check(load_library().cb2_get_restart_state(self._h, _ptr(out)), "cb2_get_restart_state")
        return out

    def set_restart_state(self, state: np.ndarray, istep: int):
        state = np.ascontiguousarray(state, dtype=np.float64).reshape(len(RESTART_FIELDS_COMPS), self.nr, self.jmax)
        _check(load_library().cb2_set_restart_state(self._h, _ptr(state), istep), "cb2_set_restart_state")

    def step_restart_state(self, state: np.ndarray, with_energies: bool = True):
        """One Adams-Bashforth step of a host-resident restart state (in place)."""
        ene = np.zeros(7)
        _check(load_library().cb2_step_restart_state(self._h, _ptr(state), _ptr(ene) if with_energies else None),
               "cb2_step_restart_state")
        return ene

    # --- transforms -----------------------------------------------------
    def sph_back_trans(self, nvec: int, nscal: int, spec: np.ndarray) -> np.ndarray:
        """Spectra (nc x nr x jmax, j = l(l+1)+m) -> grid (nc x nr x nth x nph)."""
        nc = 3 * nvec + nscal
        spec = np.ascontiguousarray(spec, dtype=np.float64).reshape(nc, self.nr, self.jmax)
        grid = np.zeros((nc, self.nr, self.nth, self.nph))
        _check(load_library().cb2_sht_backward(self._h, nvec, nscal, _ptr(spec), _ptr(grid)),
               "cb2_sht_backward")
        return grid

    def sph_forward_trans(self, nvec: int, nscal: int, grid: np.ndarray) -> np.ndarray:
        """Grid (nc x nr x nth x nph) -> spectra (nc x nr x jmax)."""
        nc = 3 * nvec + nscal
        grid = np.ascontiguousarray(grid, dtype=np.float64).reshape(nc, self.nr, self.nth, self.nph)
        spec = np.zeros((nc, self.nr, self.jmax))
        _check(load_library().cb2_sht_forward(self._h, nvec, nscal, _ptr(grid), _ptr(spec)),
               "cb2_sht_forward")
        return spec

    # the reference's routine-level entry points on its transposed buffers
    # (host numpy arrays or device addresses as ints; see cb2_sph_tables)
    @staticmethod
    def _buf(a, n):
        if isinstance(a, int):
            return ctypes.c_void_p(a), None
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if a.size < n:
            raise CalypsoError(f"buffer of {a.size} values, the tables need {n}")
        return ctypes.c_void_p(a.ctypes.data), a

    def sel_backward_legendre_trans(self, ncomp: int, nvector: int, nscalar: int, WR, tables: SphTables,
                                    WS=None):
        """sp_rlm (WR) -> vr_rtm (WS), Legendre transform only."""
        n_wr, n_ws = rlm_size(tables, ncomp), rtm_size(tables, ncomp)
        pr, keep = self._buf(WR, n_wr)
        if WS is None:
            WS = np.zeros(n_ws)
        pw, out = self._buf(WS, n_ws)
        _check(load_library().cb2_leg_bwd(self._h, ctypes.byref(tables), ncomp, nvector, nscalar,
                                          keep.size if keep is not None else n_wr,
                                          out.size if out is not None else n_ws, pr, pw), "cb2_leg_bwd")
        return WS

    def sel_forward_legendre_trans(self, ncomp: int, nvector: int, nscalar: int, WR, tables: SphTables,
                                   WS=None):
        """vr_rtm (WR) -> sp_rlm (WS), Legendre transform only."""
        n_wr, n_ws = rtm_size(tables, ncomp), rlm_size(tables, ncomp)
        pr, keep = self._buf(WR, n_wr)
        if WS is None:
            WS = np.zeros(n_ws)
        pw, out = self._buf(WS, n_ws)
        _check(load_library().cb2_leg_fwd(self._h, ctypes.byref(tables), ncomp, nvector, nscalar,
                                          keep.size if keep is not None else n_wr,
                                          out.size if out is not None else n_ws, pr, pw), "cb2_leg_fwd")
        return WS

    def back_MHD_FFT_sel_from_recv(self, ncomp: int, WR, tables: SphTables, fld_rtp=None):
        """vr_rtm (WR) -> fld_rtp (nnod_rtp x ncomp, Fortran order), FFT only."""
        n_wr = rtm_size(tables, ncomp)
        nnod = self.nr * self.nth * self.nph
        pr, keep = self._buf(WR, n_wr)
        if fld_rtp is None:
            fld_rtp = np.zeros(nnod * ncomp)
        pf, _ = self._buf(fld_rtp, nnod * ncomp)
        _check(load_library().cb2_fft_bwd(self._h, ctypes.byref(tables), ncomp,
                                          keep.size if keep is not None else n_wr, pr, pf), "cb2_fft_bwd")
        return fld_rtp

    def fft_products(self, WR, tables: SphTables, WS=None):
        """13 Fourier components (u, w, B, J, T) in the rtm layout -> the 12
        product components (w x u, J x B, u x B, u T with their
        coefficients): FFT, grid products and FFT of the time step."""
        n_wr, n_ws = rtm_size(tables, 13), rtm_size(tables, 12)
        pr, keep = self._buf(WR, n_wr)
        if WS is None:
            WS = np.zeros(n_ws)
        pw, out = self._buf(WS, n_ws)
        _check(load_library().cb2_fft_products(self._h, ctypes.byref(tables),
                                               keep.size if keep is not None else n_wr, pr,
                                               out.size if out is not None else n_ws, pw), "cb2_fft_products")
        return WS

    def fwd_MHD_FFT_sel_from_recv(self, ncomp: int, frc_rtp, tables: SphTables, WS=None):
        """frc_rtp (nnod_rtp x ncomp, Fortran order) -> vr_rtm (WS), FFT only."""
        n_ws = rtm_size(tables, ncomp)
        nnod = self.nr * self.nth * self.nph
        pf, keep = self._buf(frc_rtp, nnod * ncomp)
        if WS is None:
            WS = np.zeros(n_ws)
        pw, out = self._buf(WS, n_ws)
        _check(load_library().cb2_fft_fwd(self._h, ctypes.byref(tables), ncomp, pf,
                                          out.size if out is not None else n_ws, pw), "cb2_fft_fwd")
        return WS

    def gauss(self):
        c, w = np.zeros(self.nth), np.zeros(self.nth)
        _check(load_library().cb2_get_gauss(self._h, _ptr(c), _ptr(w)), "cb2_get_gauss")
        return c, w

    def plm(self, l: int, m: int):
        p, dp = np.zeros(self.nth), np.zeros(self.nth)
        _check(load_library().cb2_get_plm(self._h, l, m, _ptr(p), _ptr(dp)), "cb2_get_plm")
        return p, dp


def legendre_trans_mode(legendre_trans_loop_ctl: str) -> int:
    """Precision a Legendre_trans_loop_ctl value selects (cb2_legendre_trans_mode)."""
    return load_library().cb2_legendre_trans_mode((legendre_trans_loop_ctl or "").encode())


def fft_library_known(fft_library_ctl: str) -> bool:
    return bool(load_library().cb2_fft_library_known((fft_library_ctl or "").encode()))


class Ensemble:
    """Independent shells advanced together, one CUDA graph launch per step
    (cb2_ensemble_*); set_batched(True) makes mixed-precision shells share
    one launch of each Legendre GEMM.  `shells[i]` is a view of shell i (do
    not close it)."""

    def __init__(self, params_list, precision: int = PREC_MIXED, device: int = -1, autotune: bool = True):
        lib = load_library()
        n = len(params_list)
        arr = (Params * n)()
        for q, prm in enumerate(params_list):
            for k, v in prm.items():
                setattr(arr[q], k, v)
        h = ctypes.c_void_p()
        _check(lib.cb2_ensemble_create(arr, n, precision, device, 1 if autotune else 0, ctypes.byref(h)),
               "cb2_ensemble_create")
        self._h = h
        self.params = [dict(p) for p in params_list]
        self.shells = [SphMHD._wrap(lib.cb2_ensemble_shell(h, q), self.params[q], precision) for q in range(n)]

    def __len__(self):
        return len(self.shells)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            load_library().cb2_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()
            self.shells = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_fields(self, kind: int = 2, seed0: int = 0):
        _check(load_library().cb2_ensemble_init_fields(self._h, kind, seed0), "cb2_ensemble_init_fields")

    def step(self, nsteps: int = 1):
        _check(load_library().cb2_ensemble_step(self._h, nsteps), "cb2_ensemble_step")

    def set_batched(self, on: bool):
        """Mixed-precision shells: each Legendre GEMM as one launch over all
        shells (True) or one launch per shell (False, the default)."""
        _check(load_library().cb2_ensemble_set_batched(self._h, 1 if on else 0), "cb2_ensemble_set_batched")

    def sync(self):
        _check(load_library().cb2_ensemble_sync(self._h), "cb2_ensemble_sync")

    def time_steps(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        _check(load_library().cb2_ensemble_time_steps(self._h, nsteps, ctypes.byref(ms)), "cb2_ensemble_time_steps")
        return ms.value

    def energies(self) -> np.ndarray:
        out = np.zeros((len(self.shells), 7))
        _check(load_library().cb2_ensemble_energies(self._h, _ptr(out)), "cb2_ensemble_energies")
        return out


class PinnedArray:
    """Page-locked float64 array from cb2_alloc_pinned (freed with the object)."""

    def __init__(self, shape):
        n = int(np.prod(shape))
        p = ctypes.c_void_p()
        _check(load_library().cb2_alloc_pinned(n * 8, ctypes.byref(p)), "cb2_alloc_pinned")
        self._p = p
        buf = (ctypes.c_double * n).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=np.float64).reshape(shape)

    def __del__(self):
        try:
            if self._p.value:
                load_library().cb2_free_pinned(self._p)
        except Exception:
            pass
