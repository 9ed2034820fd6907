"""The viscous inversion (system.f90:564-666) on the oracle: the
reference's nested loop ends after one outer pass, so its primitives keep
pi^{t mu} of the guess's velocities; ECHO_C2P_NEWTON iterates the passes to
the fixed point.  Residual = max over the conserved fields of
|prim2cons(v) - u| / max|u| at the metric of the inversion."""
import numpy as np

import pyoracle as O
from echo_gpu import params as P
from helpers import CASES, rel_linf, setup


def _cells(steps=6):
    cfg = CASES["visc2d"]()
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    for _ in range(steps):
        o.step()
    v, u = o.state()
    t = o.t - o.dt  # the last inversion used the metric of the step's start
    return cfg, pc, tab, v.reshape(cfg.nv, -1).T.copy(), u.reshape(cfg.nv, -1).T.copy(), t


def _residual(pc, tab, t, v, u):
    _, u2, bad = O.prim2cons(pc, tab, t * t, t, v.copy())
    assert bad == 0
    return float((np.abs(u2 - u)[:, :5].max(0) / np.maximum(np.abs(u)[:, :5].max(0), 1e-300)).max())


def test_reference_loop_stops_after_one_pass():
    cfg, pc, tab, v, u, t = _cells()
    guess = v.copy()
    guess[:, 1:4] *= 0.99  # velocities 1 % off
    vr, err, it = O.c2p(pc, tab, t * t, t, u, guess)
    assert (err == 0).all()
    # the Newton ran once: the 1 % shows up in the answer through pi^{t mu}
    assert rel_linf(vr.T.copy(), v.T.copy(), cfg.nv) > 1e-6
    assert _residual(pc, tab, t, vr, u) > 1e-7


def test_newton_mode_reaches_the_fixed_point():
    cfg, pc, tab, v, u, t = _cells()
    pn = cfg.replace(algo_solver=P.C2P_NEWTON).to_c(przero=pc.przero)
    answers = []
    for scale in (1.0, 0.99, 0.9):
        guess = v.copy()
        guess[:, 1:4] *= scale
        guess[:, 4] *= 2.0 - scale
        vn, err, it = O.c2p(pn, tab, t * t, t, u, guess)
        assert (err == 0).all()
        assert _residual(pn, tab, t, vn, u) < 1e-12
        answers.append(vn)
    # every start meets the same root, to the Newton's 1e-12 step tolerance
    for a in answers[1:]:
        assert rel_linf(a.T.copy(), answers[0].T.copy(), cfg.nv) < 1e-12
