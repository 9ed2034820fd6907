"""Host side of the learned seed, on the oracle (no GPU): the six
invariants and two targets of each equation set's states, and the weight
layout the C-ABI declares (include/echo_gpu.h ECHO_MLP_*)."""
import os
import re

import numpy as np

import pyoracle as O
from echo_gpu import initial as I
from echo_gpu import seed as S
from helpers import CASES, przero_of, setup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _state(case, v=None, steps=2, tab=None):
    cfg = CASES[case]()
    pc, tab0, v0 = setup(cfg)
    tab = tab0 if tab is None else tab
    o = O.Oracle(cfg.to_c(przero=przero_of(cfg)) if v is not None else pc, tab)
    o.set_state(v0 if v is None else v, None, cfg.tstart)
    for _ in range(steps):
        o.step()
    v, u = o.state()
    return cfg, v, u, o.t - o.dt


def test_header_layout_matches_the_host():
    with open(os.path.join(ROOT, "include", "echo_gpu.h")) as f:
        h = f.read()
    val = {k: int(re.search(rf"#define {k} (\d+)", h).group(1)) for k in
           ("ECHO_MLP_NIN", "ECHO_MLP_NWEIGHTS", "ECHO_MLP_NNORM")}
    nin = val["ECHO_MLP_NIN"]
    assert nin == S.NIN and val["ECHO_MLP_NWEIGHTS"] == S.NW and val["ECHO_MLP_NNORM"] == S.NNORM
    # 4 x 64 tanh: (nin, 64), (64, 64) x 3, (64, 2), each followed by its biases
    assert S.NW == nin * 64 + 64 + 3 * (64 * 64 + 64) + 64 * 2 + 2
    assert S.NNORM == 2 * nin + 4


def _check_common(cfg, v, u, t, X, T):
    n = cfg.nx * cfg.ny * cfg.nz
    assert X.shape == (n, S.NIN) and T.shape == (n, 2)
    assert np.isfinite(X).all() and np.isfinite(T).all()
    uu = u.reshape(cfg.nv, -1) / t
    vv = v.reshape(cfg.nv, -1)
    assert np.allclose(X[:, 0], np.log(uu[4]), rtol=1e-6)
    assert np.allclose(X[:, 1], uu[0] / uu[4], rtol=1e-6)
    assert np.allclose(T[:, 1], vv[4] / uu[4], rtol=1e-6)
    assert (T[:, 0] >= 0).all() and (T[:, 0] < 1).all()


def test_ideal_rmhd_invariants():
    cfg, v, u, t = _state("rmhd3d")
    X, T = S.invariants_targets(u, v, t, cfg)
    _check_common(cfg, v, u, t, X, T)
    assert (X[:, 3] > 0).all() and (X[:, 5] == 0).all()  # B, no E


def test_viscous_invariants_have_no_field():
    cfg, v, u, t = _state("visc2d")
    X, T = S.invariants_targets(u, v, t, cfg)
    _check_common(cfg, v, u, t, X, T)
    assert (X[:, 3:] == 0).all()


def test_resistive_invariants_carry_e():
    cfg = CASES["res3d"]()
    _, tab, _ = setup(cfg)
    cfg, v, u, t = _state("res3d", v=I.resistive_flow(cfg, tab, amp=0.2, ideal=0.7), tab=tab)
    X, T = S.invariants_targets(u, v, t, cfg)
    _check_common(cfg, v, u, t, X, T)
    uu = u.reshape(cfg.nv, -1) / t
    e2 = uu[8] ** 2 + uu[9] ** 2 + t * t * uu[10] ** 2
    assert np.allclose(X[:, 5], e2 / uu[4], rtol=1e-6) and (X[:, 5] > 0).mean() > 0.9
