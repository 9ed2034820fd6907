"""The product build's cell-centred face sweep (faces_seg_kernel: one lane per
cell, both face states of a cell from one set of WENO5 smoothness
indicators, the state of the cell below taken from the neighbouring lane),
in both segment lengths, against the oracle and against the
one-thread-per-face sweep.  For every
equation set, on grids whose extents leave partial segments and partial
lane groups, and with the boundary codes that take the general ghost path
(extrapolation, mixed codes).  Bar: the product build's 1e-12 relative
L-inf per field group."""
import os
import sys

import pytest

from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, RES_GROUPS, rel_linf, resistive_state, setup

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import pyoracle as O  # noqa: E402  (the checker)

pytestmark = pytest.mark.gpu

RUNS = {
    "hd2d": (lambda: CASES["hd2d"](), 8),
    "rmhd3d": (lambda: CASES["rmhd3d"](), 5),
    "rmhd3d_odd": (lambda: P.small(P.config1(), 13, nz=9), 3),
    "visc2d_imex": (lambda: CASES["visc2d"]().replace(imex=1), 6),
    "res3d": (lambda: CASES["res3d"]().replace(sigma_el=500.0), 3),
}


def _run(pc, tab, v0, u0, t0, steps, mode):
    g = Evolve(pc, tab, exact=False)
    g.set_faces(mode)
    g.upload(v0, u0, t0)
    g.run(steps)
    g.sync()
    st = g.stats()
    v, u = g.download()
    g.close()
    return v, u, st


def _oracle(pc, tab, v, t0, steps):
    o = O.Oracle(pc, tab)
    o.set_state(v, None, t0)
    v0, u0 = o.state()
    for _ in range(steps):
        o.step()
    vo, _ = o.state()
    return v0, u0, vo


@pytest.mark.parametrize("name", list(RUNS))
def test_face_modes_match_oracle_and_face_sweep(name):
    mk, steps = RUNS[name]
    cfg = mk()
    pc, tab, v = setup(cfg)
    groups = None
    if name.startswith("res"):
        v = resistive_state(cfg, tab)
        groups = RES_GROUPS
    v0, u0, vo = _oracle(pc, tab, v, cfg.tstart, steps)
    vf, _, sf = _run(pc, tab, v0, u0, cfg.tstart, steps, 0)
    assert sf.errcode == 0 and rel_linf(vf, vo, cfg.nv, groups) <= 1e-12
    for mode in (8, 16):
        vs, _, ss = _run(pc, tab, v0, u0, cfg.tstart, steps, mode)
        assert ss.errcode == 0, (mode, ss.errcode)
        assert ss.t == sf.t
        e = rel_linf(vs, vo, cfg.nv, groups)
        print(f"{name} faces mode {mode}: vs oracle {e:.2e}, vs face sweep {rel_linf(vs, vf, cfg.nv, groups):.2e}")
        assert e <= 1e-12, (mode, e)


def test_face_modes_general_boundaries():
    """Extrapolation (code 3) along x and reflecting along y with v^y odd:
    the general ghost path."""
    cfg = CASES["rmhd3d"]()
    pc, tab, v = setup(cfg)
    for k in range(16):
        for s in range(2):
            pc.ibc[k][s][0] = 3
            pc.ibc[k][s][1] = -1 if k == 2 else 1
    v0, u0, vo = _oracle(pc, tab, v, cfg.tstart, 3)
    for mode in (0, 8, 16):
        vs, _, ss = _run(pc, tab, v0, u0, cfg.tstart, 3, mode)
        assert ss.errcode == 0
        assert rel_linf(vs, vo, cfg.nv) <= 1e-12, (mode, rel_linf(vs, vo, cfg.nv))


def test_face_mode_is_checked():
    cfg = CASES["hd2d"]()
    pc, tab, _ = setup(cfg)
    g = Evolve(pc, tab, exact=False)
    for bad in (-1, 1, 2, 7, 32):
        with pytest.raises(RuntimeError):
            g.set_faces(bad)
    g.close()
