"""The fused stage kernel (stage.cuh) against the sweep kernels and the oracle.

The fused stage computes every face flux from the same stencils with the
same arithmetic as the sweep kernels, so in the parity build (no FMA
contraction) a run through it is bit-identical to the same run through the
sweeps, and both equal the oracle within the parity bar.  Checked for every
equation set: ideal hydro (RK2: its first stage runs the sweeps, the second
the fused kernel), ideal RMHD with GLM (RK3, every stage fused), viscous
(explicit and IMEX RK2), resistive RMHD (IMEX-SSP3(4,3,3): the fused kernel
writes the stage right-hand sides); with the tile chosen for the grid and
with small forced tiles and eta segments, so that partial tiles, tile edges
and segment starts occur everywhere on these small grids.
"""
import os
import sys

import numpy as np
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
    "visc2d": (lambda: CASES["visc2d"](), 6),
    "visc2d_imex": (lambda: CASES["visc2d"]().replace(imex=1), 6),
    "res3d": (lambda: CASES["res3d"]().replace(sigma_el=500.0), 3),
    "rmhd3d_newton": (lambda: CASES["rmhd3d"]().replace(algo_solver=P.C2P_NEWTON), 5),
}


def _state(name, cfg):
    pc, tab, v = setup(cfg)
    if name.startswith("res"):
        v = resistive_state(cfg, tab)
    return pc, tab, v


def _run(pc, tab, v0, u0, t0, steps, exact, stage):
    g = Evolve(pc, tab, exact=exact)
    info = g.set_stage(**stage)
    g.upload(v0, u0, t0)
    g.run(steps)
    g.sync()
    st = g.stats()
    v, u = g.download()
    g.close()
    return v, u, st, info


@pytest.mark.parametrize("name", list(RUNS))
def test_fused_stage_matches_sweeps_and_oracle(name):
    mk, steps = RUNS[name]
    cfg = mk()
    pc, tab, v = _state(name, cfg)
    groups = RES_GROUPS if name.startswith("res") else None
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    for _ in range(steps):
        o.step()
    vo, uo = o.state()
    vs, us, ss, _ = _run(pc, tab, v0, u0, cfg.tstart, steps, True, {"fused": False})
    assert ss.errcode == 0
    tiles = [{"fused": True}, {"fused": True, "tx": 6, "ty": 5, "zseg": 3}, {"fused": True, "tx": 7, "ty": 9, "zseg": 2}]
    for stage in tiles:
        vf, uf, sf, info = _run(pc, tab, v0, u0, cfg.tstart, steps, True, stage)
        assert info["fused"] == 1, info
        assert sf.errcode == 0
        # parity build: the same arithmetic, so the same bits as the sweeps
        assert np.array_equal(vf, vs), (stage, rel_linf(vf, vs, cfg.nv, groups))
        assert np.array_equal(uf, us), (stage, rel_linf(uf, us, cfg.nv, groups))
        assert sf.t == ss.t and sf.dt == ss.dt
        # Newton con2prim meets the oracle's BRENTM root at the product bar
        bar = 1e-12 if cfg.algo_solver == P.C2P_NEWTON else 1e-13
        assert rel_linf(vf, vo, cfg.nv, groups) <= bar
    # product build, fused, against the oracle
    vp, up, sp, info = _run(pc, tab, v0, u0, cfg.tstart, steps, False, {"fused": True})
    assert info["fused"] == 1 and sp.errcode == 0
    err = rel_linf(vp, vo, cfg.nv, groups)
    print(f"{name}: fused tile {info['tx']}x{info['ty']} zseg {info['zseg']} ({info['threads']} threads, "
          f"{info['ctas']} CTAs, {info['smem_bytes']} B smem): product vs oracle {err:.2e}")
    assert err <= 1e-12


def test_fused_stage_refused_where_it_cannot_run():
    cfg = CASES["rmhd3d"]().replace(recal="MPE5")
    pc, tab, v = setup(cfg)
    g = Evolve(pc, tab, exact=True)
    with pytest.raises(RuntimeError):
        g.set_stage(True)
    assert g.set_stage(False)["fused"] == 0
    g.close()
