"""Writes tests/golden/reference_pins.json: values the reference printed in a
run of its own, with the inputs needed to recompute them, read from the
reference's files.

The reference ships one run log, doc/images/echo-qgp-output.txt (a 51^3
viscous optical-Glauber Au+Au run at b = 5 fm on [-9, 9]^3 fm).  Two of its
lines are outputs of routines on or beside the step path:

  - line 98, "check nucleus mass 196.94642": the thickness table of the
    optical Glauber initial state (init.f90:1164-1219, printed at :1219),
    from the nucleus of nuclear_data.dat line 1 (Au) and the printed table
    steps and accuracy (lines 61-63) over the reach of the printed grid and
    impact parameter (lines 16-18, 40; init.f90:1100-1104);
  - line 109, the pressure and energy density of the viscosity smoothing
    threshold (evolve.f90:1181): the energy is get_energy (eos.f90:468-523)
    of the printed pressure in the default table qcdIEOS0.dat
    (common.f90:649).  The two table rows that bracket the pressure are
    stored here as the file holds them (text), with their 1-based indices.

Run from the repository root with the reference's files present; the tests
read only the JSON.
"""
from __future__ import annotations

import json
import math
import os
import sys

REF = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))
HC3 = 0.00768351  # eos.f90:275


def main():
    log = open(os.path.join(REF, "doc/images/echo-qgp-output.txt")).read().splitlines()
    mass_line = log[97]
    thr_line = log[108]
    assert mass_line.startswith("check nucleus mass"), mass_line
    assert "Pressure treshold" in thr_line, thr_line
    check_printed = mass_line.split()[-1]
    f = thr_line.split()
    p_golden = float(f[3])
    e_golden = float(f[-1])
    nuc = open(os.path.join(REF, "nuclear_data.dat")).readline()

    def field(key):
        return float(nuc.split(key + "=")[1].split()[0])

    nucleus = {"name": nuc.split()[0], "projmass": field("projmass"), "radius": field("radius"),
               "delta": field("delta"), "roze": field("roze")}
    # the table rows around p_golden, located as get_energy's bisection would
    rows = open(os.path.join(REF, "eos_data/qcdIEOS0.dat")).read().splitlines()
    n = int(rows[0].split()[0])
    body = rows[1:1 + n]
    p = []
    for r in body:
        T, _, c3, _ = (float(x) for x in r.split()[:4])
        p.append(c3 / HC3 * math.pow(T, 4.0))
    lo, hi = 1, n
    mid = (lo + hi) // 2
    while lo + 1 != hi:
        if p_golden > p[mid - 1]:
            lo = mid
        else:
            hi = mid
        mid = (lo + hi) // 2
    out = {
        "source": "doc/images/echo-qgp-output.txt (the reference's own run log)",
        "check_nucleus_mass": {
            "printed": check_printed, "format": "f10.5", "log_line": 98,
            "printed_by": "init.f90:1219", "nucleus": nucleus, "nuclear_data_line": 1,
            "grid": {"x1": -9.0, "x2": 9.0, "y1": -9.0, "y2": 9.0, "log_lines": [17, 18]},
            "bimpact": 5.0, "bimpact_log_line": 40,
            "dr": 0.001, "dz1": 0.001, "acc": 1e-7, "steps_log_lines": [61, 62, 63],
        },
        "eos_get_energy": {
            "pressure": p_golden, "energy": e_golden, "log_line": 109, "printed_by": "evolve.f90:1181",
            "table": "eos_data/qcdIEOS0.dat", "entries": n, "row_lo": lo, "row_hi": hi,
            "rows_text": [body[lo - 1], body[hi - 1]],
        },
        "generated_by": "tests/golden/make_reference_pins.py",
    }
    path = os.path.join(HERE, "reference_pins.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {path}: check mass {check_printed}, p {p_golden!r} -> e {e_golden!r} in rows {lo}, {hi}")


if __name__ == "__main__":
    sys.exit(main())
