"""Restart files in the reference's ascii spectral field format (step
header, field/component table, one row per rj node): a written state reads
back to 1e-15 (16 significant digits in the file), the header and field
table have the reference's layout, and missing fields are an error."""
import numpy as np
import pytest

from calypso_b200.restart import read_restart, restart_file_name, write_restart


def test_restart_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(3)
    nr, jmax = 5, 16
    state = rng.standard_normal((14, nr, jmax)) * np.logspace(-9, 3, 14)[:, None, None]
    path = tmp_path / restart_file_name("rst", 2)
    assert path.name == "rst.2.0.fst"
    write_restart(str(path), state, 100, 5e-3, 5e-5)
    lines = path.read_text().splitlines()
    assert lines[:6] == ["!  domain ID", f"{0:16d}", "!  time step number", f"{100:16d}", "!  time, Delta t",
                         "   5.000000000000000E-003   5.000000000000000E-005"]
    assert lines[6] == "! Number of field and component"
    assert lines[7] == f"{nr * jmax:16d}{6:16d}"
    assert lines[8] == "    3    1    3    3    3    1"
    assert lines[9] == "velocity"
    assert len(lines[10]) == 75 and lines[10].count("E") == 3
    back, istep, time, dt = read_restart(str(path), nr, jmax)
    assert (istep, time, dt) == (100, 5e-3, 5e-5)
    np.testing.assert_allclose(back, state, rtol=1e-15, atol=0)


def test_restart_missing_field_rejected(tmp_path):
    nr, jmax = 3, 4
    path = tmp_path / "r.fst"
    write_restart(str(path), np.ones((14, nr, jmax)), 1, 0.1, 0.1)
    txt = path.read_text().replace("previous_heat", "some_other_field")
    path.write_text(txt)
    with pytest.raises(ValueError):
        read_restart(str(path), nr, jmax)
    with pytest.raises(ValueError):
        read_restart(str(path), nr + 1, jmax)
