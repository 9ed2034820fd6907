"""Resistive RMHD (MHD = 2, IMEX-SSP3(4,3,3) with the implicit Ohm's law)
on the device against the oracle's statement of the same scheme.

Tolerances as for the other equation sets: 1e-13 exact build, 1e-12 product
build, relative L-inf per field group (rho; v; p; B, E and psi together).
"""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, RES_GROUPS, przero_of, rel_linf, resistive_state, setup
from test_resistive import cfg_box, uniform

pytestmark = pytest.mark.gpu


def _pair(cfg, v, steps, exact, use_run=False, tab=None):
    pc = cfg.to_c(przero=przero_of(cfg))
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc, tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(steps):
        o.step()
    if use_run:
        g.run(steps)
        g.sync()
    else:
        for _ in range(steps):
            g.step()
    vo, uo = o.state()
    vg, ug = g.download()
    st = g.stats()
    assert st.errcode == 0
    assert abs(st.t - o.t) <= 1e-14 * abs(o.t)
    return rel_linf(vg, vo, 12, RES_GROUPS), rel_linf(ug, uo, 12, RES_GROUPS), vo


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
@pytest.mark.parametrize("sigma", [0.0058, 500.0])
def test_step_parity(exact, tol, sigma):
    """The 3+1D workload on a 10x10x8 grid (tabulated EoS, GLM, chiral
    current) with a flow and a non-ideal E; sigma = 500 makes the implicit
    Ohm solve matter (sigma dt a_ii ~ 0.25)."""
    cfg = CASES["res3d"]().replace(sigma_el=sigma)
    _, tab, _ = setup(cfg)
    ev, eu, vo = _pair(cfg, resistive_state(cfg, tab), 6, exact, tab=tab)
    assert np.all(np.isfinite(vo))
    assert ev <= tol and eu <= tol, (ev, eu)


def test_graph_run_matches_oracle():
    cfg = CASES["res3d"]().replace(sigma_el=500.0)
    _, tab, _ = setup(cfg)
    ev, eu, _ = _pair(cfg, resistive_state(cfg, tab), 4, True, use_run=True, tab=tab)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
def test_stiff_decay_parity(exact, tol):
    """A fluid at rest in Minkowski coordinates, sigma dt = 10."""
    cfg = cfg_box(sigma_el=100.0, maxdt=0.1).replace(tstart=0.0)
    ev, eu, vo = _pair(cfg, uniform(cfg, E=(1.0, 0.0, 0.0)), 10, exact)
    assert 0.0 <= vo.reshape(12, -1)[8, 0] < 1e-10
    assert ev <= tol and eu <= tol, (ev, eu)


def test_rejected_combinations():
    base = CASES["res3d"]()
    _, tab, _ = setup(base)
    for cfg in (base.replace(nrk=P.RK3), base.replace(divclean=0)):
        with pytest.raises(RuntimeError, match="status -3"):
            Evolve(cfg.to_c(przero=przero_of(cfg)), tab)


@pytest.mark.parametrize("bc", [0, 1, 2, 3])
def test_boundaries(bc):
    """Every ghost fill (periodic, reflecting, outflow, extrapolation) in the
    faces and in the charge density's neighbours."""
    cfg = CASES["res3d"]().replace(sigma_el=500.0, boundary=bc)
    _, tab, _ = setup(cfg)
    ev, eu, _ = _pair(cfg, resistive_state(cfg, tab), 3, True, tab=tab)
    assert ev <= 1e-13 and eu <= 1e-13, (bc, ev, eu)
