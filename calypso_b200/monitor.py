"""Monitor files of the time loop in the reference's text formats.

* ``sph_pwr_volume_s.dat``: volume mean squares after every check step
  (output_sph_m_square_file.f90 write_sph_vol_ms_file, format
  ``(i16,1pe23.14e3,1p200e23.14e3)``), header as write_sph_mean_sq_header
  (m_rms_4_sph_spectr.f90:226-279);
* ``sph_pwr_volume_l.dat`` / ``_m.dat`` / ``_lm.dat``: the same by degree,
  order and l - |m| (write_sph_volume_data, ``(i16,1pe23.14e3,i16,
  N(1pe23.14e3))``), written when the control file's ``sph_monitor_ctl``
  names a ``volume_pwr_spectr_prefix``;
* :func:`compare_mean_square` checks two such files column by column with a
  relative tolerance, as the reference's ``sph_ene_check``
  (src/programs/data_utilities/TIME_HISTORIES/compare_sph_mean_square.f90:96-117).

The seven columns are the energies of :meth:`SphMHD.energies`: kinetic
(poloidal, toroidal, total), the mean square temperature, magnetic
(poloidal, toroidal, total).
"""
from __future__ import annotations

import math
import os

LABELS = ["K_ene_pol", "K_ene_tor", "K_ene", "temperature", "M_ene_pol", "M_ene_tor", "M_ene"]
COMPS = [3, 1, 3]          # velocity, temperature, magnetic_field


def fortran_e(x: float, digits: int = 14, width: int = 23, edigits: int = 3) -> str:
    """One value as Fortran's 1pE<width>.<digits>e<edigits> edit descriptor writes it."""
    if not math.isfinite(x):
        return f"{'NaN' if math.isnan(x) else ('Infinity' if x > 0 else '-Infinity'):>{width}}"
    if x == 0.0:
        mant, ex = 0.0, 0
    else:
        ex = math.floor(math.log10(abs(x)))
        mant = x / 10.0 ** ex
        # rounding can carry the mantissa to 10
        if round(abs(mant), digits) >= 10.0:
            ex += 1
            mant = x / 10.0 ** ex
    s = f"{mant:.{digits}f}E{'-' if ex < 0 else '+'}{abs(ex):0{edigits}d}"
    return f"{s:>{width}}"


def _header(f, L: int, nlayer_icb: int, nlayer_cmb: int, mode_label: str | None):
    f.write("radial_layers, truncation\n")
    f.write(f"{0:16d}{L:16d}\n")
    f.write("ICB_id, CMB_id\n")
    f.write(f"{nlayer_icb:16d}{nlayer_cmb:16d}\n")
    f.write("number of components\n")
    f.write(f"{len(COMPS):16d}{sum(COMPS):16d}\n")
    f.write("".join(f"{c:5d}" for c in COMPS) + "\n")
    f.write("t_step    time    ")
    if mode_label:
        f.write(f"{mode_label}    ")
    f.write("".join(f"{lab}    " for lab in LABELS) + "\n")


class MonitorFiles:
    """Appends the check-step rows of one run (a file and its header are
    written with its first row, as open_sph_mean_sq_file does for a file that
    does not exist yet)."""

    def __init__(self, directory: str, L: int, nr: int, volume_prefix: str = "sph_pwr_volume",
                 spectra: bool = False, degree: bool = True, order: bool = True, diff_lm: bool = True):
        self.dir, self.L, self.nr = directory, L, nr
        self.prefix = volume_prefix
        self.spectra = spectra
        self.kinds = [k for k, on in (("l", degree), ("m", order), ("lm", diff_lm)) if on]

    def _path(self, suffix: str) -> str:
        return os.path.join(self.dir, f"{self.prefix}{suffix}")

    def write(self, step: int, time: float, energies, spectra: dict | None = None):
        path = self._path("_s.dat")
        new = not os.path.exists(path)
        with open(path, "a") as f:
            if new:
                _header(f, self.L, 1, self.nr, None)
            f.write(f"{step:16d}" + fortran_e(time) + "".join(fortran_e(float(v)) for v in energies) + "\n")
        if not (self.spectra and spectra):
            return
        labels = {"l": "degree", "m": "order", "lm": "diff_deg_order"}
        for kind in self.kinds:
            path = self._path(f"_{kind}.dat")
            new = not os.path.exists(path)
            with open(path, "a") as f:
                if new:
                    _header(f, self.L, 1, self.nr, labels[kind])
                sp = spectra[kind]
                for g in range(self.L + 1):
                    f.write(f"{step:16d}" + fortran_e(time) + f"{g:16d}"
                            + "".join(fortran_e(float(sp[q][g])) for q in range(len(LABELS))) + "\n")


def read_mean_square(path: str):
    """Rows (step, time, values) of a volume mean-square file."""
    rows = []
    with open(path) as f:
        lines = f.read().splitlines()
    start = next(i for i, ln in enumerate(lines) if ln.startswith("t_step")) + 1
    for ln in lines[start:]:
        v = ln.split()
        if v:
            rows.append((int(v[0]), float(v[1]), [float(x) for x in v[2:]]))
    return rows


def compare_mean_square(path_a: str, path_b: str, rel_tol: float = 1e-9):
    """Rows of path_a against the rows of path_b with the same step: the
    largest relative difference per row, and whether every column of every
    common row is within rel_tol (|a - b| <= rel_tol |b|, the check of
    compare_sph_mean_square.f90)."""
    b = {r[0]: r for r in read_mean_square(path_b)}
    worst, ok = [], True
    for step, _, va in read_mean_square(path_a):
        if step not in b:
            continue
        vb = b[step][2]
        rel = max(abs(x - y) / abs(y) if y != 0.0 else abs(x) for x, y in zip(va, vb))
        worst.append((step, rel))
        ok = ok and rel <= rel_tol and len(va) == len(vb)
    return ok and bool(worst), worst
