"""Restart files in the reference's ascii spectral field format.

A restart file (MHD_src/IO/sph_mhd_rst_IO_control.f90:89-145, written by
SERIAL_src/IO/field_file_IO.f90 write_step_field_file) holds one domain's
rj spectra of the restart fields (MHD_src/sph_MHD/set_sph_restart_IO.f90):
velocity, temperature (total), magnetic_field, previous_momentum,
previous_induction and previous_heat, after a step header
(SERIAL_src/IO/m_time_data_IO.f90 write_step_data):

    !  domain ID
                   0
    !  time step number
                 100
    !  time, Delta t
      5.000000000000000E-003  5.000000000000000E-005
    ! Number of field and component
              139264               6
        3    1    3    3    3    1
    velocity
      <S>  <dS/dr>  <T>                 (one row per node, 1pE25.15e3 each)
    ...

The nodes run j fastest (inod = j + (k-1) jmax, j = l(l+1)+m+1), one file
per domain named ``<prefix>.<istep / i_step_rst_ctl>.<rank>.fst``
(SERIAL_src/IO/set_field_file_names.f90 set_SPH_fld_file_name).  This
library runs one domain, rank 0.
"""
from __future__ import annotations

import re

import numpy as np

from .monitor import fortran_e
from .sph_mhd import RESTART_FIELDS

TIME_HD1, TIME_HD2, TIME_HD3 = "!  domain ID", "!  time step number", "!  time, Delta t"
FLD_HD1 = "! Number of field and component"

_EXP2 = re.compile(rb"E([+-])(\d\d)(?=\s|$)")


def restart_file_name(prefix: str, istep_fld: int, rank: int = 0) -> str:
    return f"{prefix}.{istep_fld}.{rank}.fst"


def _rows(values: np.ndarray) -> bytes:
    """Rows of 1pE25.15e3 values (values: nnod x ncomp)."""
    ncomp = values.shape[1]
    fmt = "".join(["%24.15E"] * ncomp)
    txt = "\n".join(fmt % tuple(r) for r in values).encode()
    # three exponent digits, as the Fortran edit descriptor writes them
    return _EXP2.sub(rb"E\g<1>0\2", txt) + b"\n"


def write_restart(path: str, state: np.ndarray, istep: int, time: float, dt: float, rank: int = 0):
    """state: (14, nr, jmax) from SphMHD.get_restart_state()."""
    nc, nr, jmax = state.shape
    nnod = nr * jmax
    with open(path, "wb") as f:
        f.write(f"{TIME_HD1}\n{rank:16d}\n{TIME_HD2}\n{istep:16d}\n{TIME_HD3}\n".encode())
        f.write((fortran_e(time, 15, 25) + fortran_e(dt, 15, 25) + "\n").encode())
        f.write(f"{FLD_HD1}\n{nnod:16d}{len(RESTART_FIELDS):16d}\n".encode())
        comps = [c for _, c in RESTART_FIELDS]
        for i in range(0, len(comps), 10):
            f.write(("".join(f"{c:5d}" for c in comps[i:i + 10]) + "\n").encode())
        q = 0
        for name, ncomp in RESTART_FIELDS:
            f.write(f"{name}\n".encode())
            f.write(_rows(state[q:q + ncomp].reshape(ncomp, nnod).T))
            q += ncomp


def read_restart(path: str, nr: int, jmax: int):
    """(state (14, nr, jmax), istep, time, dt) from a restart file; fields
    are found by name (set_sph_restart_from_IO), others are skipped."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0

    def nxt():
        nonlocal pos
        while lines[pos].strip().startswith("!") or not lines[pos].strip():
            pos += 1
        ln = lines[pos]
        pos += 1
        return ln
    nxt()                                   # domain ID
    istep = int(nxt().split()[0])
    t = nxt().split()
    time, dt = float(t[0]), float(t[1])
    hd = nxt().split()
    nnod, nfield = int(hd[0]), int(hd[1])
    if nnod != nr * jmax:
        raise ValueError(f"restart file has {nnod} nodes, the shell {nr * jmax}")
    comps = []
    while len(comps) < nfield:
        comps += [int(x) for x in nxt().split()]
    found = {}
    for ncomp in comps:
        name = nxt().strip()
        block = np.loadtxt(lines[pos:pos + nnod], ndmin=2).reshape(nnod, ncomp)
        pos += nnod
        found[name] = block.T.reshape(ncomp, nr, jmax)
    state = np.zeros((sum(c for _, c in RESTART_FIELDS), nr, jmax))
    q = 0
    for name, ncomp in RESTART_FIELDS:
        if name not in found:
            raise ValueError(f"restart file has no field {name}")
        state[q:q + ncomp] = found[name]
        q += ncomp
    return state, istep, time, dt
