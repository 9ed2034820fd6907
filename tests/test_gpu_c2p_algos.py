"""ALG_SOLV 2..6 on the device against the oracle: the con2prim kernel on
single cells, and whole steps of the 3+1D RMHD case (exact build 1e-13 --
algorithms 4..6 call pow/acos/cos, which may differ from libm in the last
place -- product build 1e-12)."""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu.lib import Evolve, unit_c2p
from helpers import CASES, rel_linf, setup
from test_c2p_algos import CASES_C2P, c2p_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo,eos,t,scale", CASES_C2P + [(3, P.EOS_CONFORMAL, 0.7, 1.0)])
def test_c2p_kernel(algo, eos, t, scale):
    cfg, pc, tab, cells_p, u = c2p_case(algo, eos, t, scale)
    guess = cells_p * (1 + 1e-3)
    vo, eo, io = O.c2p(pc, tab, t * t, t, u, guess)
    vg, eg, ig = unit_c2p(pc, tab, t * t, t, u, guess, exact=True)
    assert np.array_equal(eo, eg)
    ok = eo == 0
    assert rel_linf(vg[ok].T.copy(), vo[ok].T.copy(), cfg.nv) <= 1e-13


def _state(cfg, scale):
    pc, tab, v = setup(cfg)
    vv = v.reshape(cfg.nv, -1).copy()
    vv[4] *= scale
    vv[5:8] *= np.sqrt(scale)
    return pc, tab, vv.reshape(-1)


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
@pytest.mark.parametrize("algo,eos,coords,scale", [(2, P.EOS_TABLE, P.BJORKEN, 1.0), (3, P.EOS_CONFORMAL, P.BJORKEN, 0.01),
                                                   (4, P.EOS_IDEALGAS, P.BJORKEN, 1.0),
                                                   (5, P.EOS_CONFORMAL, P.BJORKEN, 1.0),
                                                   (6, P.EOS_CONFORMAL, P.MINKOWSKI, 1.0)])
def test_step_parity(exact, tol, algo, eos, coords, scale):
    cfg = CASES["rmhd3d"]().replace(algo_solver=algo, eqstate=eos, coordinates=coords)
    pc, tab, v = _state(cfg, scale)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc, tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(3):
        o.step()
        g.step()
    vo, uo = o.state()
    vg, ug = g.download()
    assert g.stats().errcode == 0
    assert rel_linf(vg, vo, cfg.nv) <= tol and rel_linf(ug, uo, cfg.nv) <= tol, (rel_linf(vg, vo, cfg.nv),)
