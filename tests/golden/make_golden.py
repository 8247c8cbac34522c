"""Generate the golden fixtures of the Dynamobench case 1 parity pin.

Reads, from the reference tree (hlokavarapu/calypso, read-only), the test
case tests/Dynamobench_case1: its two control files (inputs of the run) and
reference/sph_pwr_volume_s.dat (the energies the reference's own regression
test compares at 1e-9).  Writes them under tests/golden/dynamobench_case1/:
  control_MHD, control_sph_shell   -- the run's input files, verbatim
  sph_pwr_volume_s.dat             -- the reference's monitor file, verbatim
                                      (its text format is pinned too)
  sph_pwr_volume_s.json            -- steps, times and the 7 energy columns
Run:  python tests/golden/make_golden.py /path/to/the/reference/checkout
"""
import json
import os
import shutil
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dynamobench_case1")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/the/reference/checkout")
    CASE = os.path.join(sys.argv[1], "tests", "Dynamobench_case1")
    os.makedirs(OUT, exist_ok=True)
    for name in ("control_MHD", "control_sph_shell"):
        shutil.copyfile(os.path.join(CASE, name), os.path.join(OUT, name))
    shutil.copyfile(os.path.join(CASE, "reference", "sph_pwr_volume_s.dat"),
                    os.path.join(OUT, "sph_pwr_volume_s.dat"))
    rows, names = [], None
    with open(os.path.join(CASE, "reference", "sph_pwr_volume_s.dat")) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] == "t_step":
                names = tok[2:]
                continue
            if names and len(tok) == len(names) + 2:
                rows.append({"step": int(tok[0]), "time": float(tok[1]),
                             "values": [float(v) for v in tok[2:]]})
    doc = {"source": "tests/Dynamobench_case1/reference/sph_pwr_volume_s.dat",
           "columns": names, "rows": rows, "rel_tol": 1.0e-9}
    with open(os.path.join(OUT, "sph_pwr_volume_s.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
