"""The optical Glauber initial state on the device (echo_gpu_optical_glauber)
against the oracle's restatement of init.f90:852-1242, and against the
reference's own printed check of its thickness table.

Tolerances: the device integrates each thickness with CUDA's exp and pow
(the oracle with libm), so the table and e agree to 1e-12 relative, not
bit for bit; the check mass, summed in the reference's order on both sides,
prints the reference's f10.5 digits."""
import json
import math
import os

import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu.lib import Evolve, optical_glauber_params
from helpers import eos_table

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _grid_params(cfg, eqstate=P.EOS_CONFORMAL, tab=None):
    pc = cfg.to_c(przero=cfg.enezero / 3.0 if tab is None else 0.0)
    return pc


@pytest.mark.parametrize("where", ["workload_101_b7", "reference_log_b5", "rmhd_3d_cut"])
def test_device_glauber_matches_oracle(where):
    tab = None
    if where == "workload_101_b7":
        cfg, b = P.config0(), 7.0
    elif where == "reference_log_b5":
        cfg, b = P.config0().replace(nx=51, ny=51, x1=-9.0, x2=9.0, y1=-9.0, y2=9.0), 5.0
    else:
        cfg, b = P.small(P.config1(), 33, nz=27), 7.0
        tab = eos_table()
    przero = cfg.enezero / 3.0 if tab is None else 0.0
    if tab is not None:
        from echo_gpu import initial as I
        przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0])
    pc = cfg.to_c(przero=przero)
    g = optical_glauber_params("Au", b=b, ecenter=20.0, rhocenter=0.1)
    ev = Evolve(pc, tab, exact=True)
    chk_d, emax = ev.optical_glauber(g, cfg.tstart)
    v, _ = ev.download()
    ev.close()
    chk_o, e_o = O.optical_glauber(g, cfg.nx, cfg.ny, cfg.nz, cfg.x1, cfg.x2, cfg.y1, cfg.y2, cfg.z1, cfg.z2)
    assert chk_o > 0 and abs(chk_d - chk_o) <= 1e-12 * chk_o
    assert abs(emax - e_o.max()) <= 1e-12 * e_o.max()
    nc = cfg.ncell
    pr = v[4 * nc:5 * nc]
    if tab is None:  # p = e/3 + przero (conformal, initio init.f90:874-880)
        assert np.max(np.abs(pr - (e_o / 3.0 + przero))) <= 1e-12 * e_o.max()
    else:
        from echo_gpu import initial as I
        assert np.max(np.abs(pr - (I.table_pressure(tab, e_o) + przero))) <= 1e-12 * pr.max()
    assert np.all(v[:nc] == 0.1)
    if where == "reference_log_b5":
        pins = json.load(open(os.path.join(HERE, "golden", "reference_pins.json")))
        assert f"{chk_d:10.5f}".strip() == pins["check_nucleus_mass"]["printed"]


def test_device_glauber_peak_normalisation_and_step():
    """The workload's normalisation (peak e = 30 GeV/fm^3 at b = 7 fm) and a
    few steps from the device initial state."""
    cfg = P.config0()
    pc = cfg.to_c(przero=cfg.enezero / 3.0)
    ev = Evolve(pc, None)
    chk, emax = ev.optical_glauber(optical_glauber_params("Au", b=7.0), cfg.tstart, peak=30.0)
    assert abs(emax - 30.0) <= 1e-12 * 30.0
    ev.run(5)
    ev.sync()
    assert ev.stats().errcode == 0
