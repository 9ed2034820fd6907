"""The oracle against values the reference printed in its own run log
(doc/images/echo-qgp-output.txt, via tests/golden/reference_pins.json,
written by tests/golden/make_reference_pins.py from the reference's files).

  - the optical Glauber thickness table (init.f90:1164-1219): the
    reference printed "check nucleus mass 196.94642" (f10.5) for Au on its
    [-9, 9]^2 fm grid at b = 5 fm with 0.001 fm steps and accuracy 1e-7;
  - the tabulated EoS interpolation get_energy (eos.f90:468-523): for the
    printed smoothing-threshold pressure the reference printed the energy
    density 1.3051308079431541E-002 from qcdIEOS0.dat; the oracle, reading
    the same two table rows with the reference's conversion (eos.f90:322-327),
    must give the same double, bit for bit.
"""
import json
import math
import os

import numpy as np

import pyoracle as O
from echo_gpu import initial as I
from echo_gpu import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
PINS = json.load(open(os.path.join(HERE, "golden", "reference_pins.json")))


def test_check_nucleus_mass_matches_the_reference_log():
    c = PINS["check_nucleus_mass"]
    nuc, g = c["nucleus"], c["grid"]
    largestx = max(abs(g["x1"]), abs(g["x2"])) + c["bimpact"]
    largesty = max(abs(g["y1"]), abs(g["y2"]))
    nmax = int(math.sqrt(largestx**2 + largesty**2) / c["dr"]) + 1  # init.f90:1101-1104
    chk, thick = O.thickness(nuc["radius"], nuc["delta"], nuc["roze"], c["dr"], c["dz1"], c["acc"], nmax)
    assert f"{chk:10.5f}".strip() == c["printed"], chk
    assert thick[0] > thick[-1] > 0


def test_eos_energy_matches_the_reference_log():
    e = PINS["eos_get_energy"]
    rows = []
    for r in e["rows_text"]:
        T, c2, c3, cs = (float(x) for x in r.split()[:4])
        t4 = math.pow(T, 4.0)
        rows.append((T, c2 / I.HC3 * t4, c3 / I.HC3 * t4, cs))
    tab = np.array(rows)
    pc = P.config1().to_c(przero=0.0)
    pc.eqstate = P.EOS_TABLE
    err, en = O.eos_energy(pc, tab, e["pressure"])
    assert err == 0
    assert en == e["energy"], (en, e["energy"])
