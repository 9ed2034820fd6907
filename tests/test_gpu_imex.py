"""IMEX RK2 (linearly implicit Israel-Stewart relaxation per stage) on the
device against the oracle's statement of the same scheme, single grid and
batched.  Tolerances as for the explicit scheme: 1e-13 exact build, 1e-12
product build, relative L-inf per field group."""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import events as EV
from echo_gpu import initial as I
from echo_gpu.batch import DONE, Batch, event_grid
from echo_gpu.lib import Evolve
from helpers import CASES, eos_table, przero_of, rel_linf, setup, smooth_pressure_of
from test_imex import E0, T0, bjorken_visc

pytestmark = pytest.mark.gpu


def _pair(cfg, steps, exact, v=None, use_run=False):
    pc, tab, v = setup(cfg, v=v)
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
    assert g.stats().errcode == 0
    return rel_linf(vg, vo, o.nv), rel_linf(ug, uo, o.nv), vo


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
@pytest.mark.parametrize("coeff", [5.0, 0.05])
def test_imex_step_parity(exact, tol, coeff):
    """The seeded 2+1D viscous case (tabulated EoS, smoothing on) at the
    workload's tau_pi and at one 100 times shorter."""
    cfg = CASES["visc2d"]().replace(imex=1, tau_pi_coeff=coeff)
    ev, eu, vo = _pair(cfg, 8, exact)
    assert np.all(np.isfinite(vo))
    assert ev <= tol and eu <= tol, (ev, eu)


def test_imex_graph_run_matches_oracle():
    cfg = CASES["visc2d"]().replace(imex=1, tau_pi_coeff=0.05)
    ev, eu, _ = _pair(cfg, 6, True, use_run=True)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
def test_stiff_bjorken_parity(exact, tol):
    """Viscous Bjorken flow with tau_pi ~ 1e-6 dt (the Navier-Stokes limit,
    where the explicit scheme blows up): 40 steps on the device."""
    cfg = bjorken_visc(0.01, 1e-6, 1).replace(tstart=T0)
    ev, eu, vo = _pair(cfg, 40, exact, v=I.bjorken_uniform(cfg, E0))
    assert np.all(np.isfinite(vo))
    assert ev <= tol and eu <= tol, (ev, eu)


def test_batch_imex_matches_oracle_per_event():
    es = EV.small_events(base=EV.batched_viscous().cfg.replace(imex=1, tau_pi_coeff=0.5), tmax=0.7)
    tab = eos_table()
    v = EV.event_primitives(es, tab)
    pc = es.cfg.to_c(przero=przero_of(es.cfg), smooth_pressure=smooth_pressure_of(es.cfg))
    b = Batch(pc, tab, [event_grid(*es.grid(e)) for e in range(es.nev)], exact=True)
    b.upload(v, None, es.cfg.tstart, es.tmax)
    b.run_to_end(chunk=4)
    st = b.status()
    vg, ug = b.download()
    for e, (vs, us) in enumerate(zip(b.split(vg), b.split(ug))):
        cfg = es.event_config(e)
        o = O.Oracle(cfg.to_c(przero=przero_of(cfg), smooth_pressure=smooth_pressure_of(cfg)), tab)
        o.set_state(v[e], None, cfg.tstart)
        o.set_tout(es.tmax, es.tmax - cfg.tstart, es.tmax)
        n = 0
        while o.t < es.tmax:
            o.step()
            n += 1
        vo, uo = o.state()
        assert st[e]["state"] == DONE and st[e]["steps"] == n, (e, st[e], n)
        assert rel_linf(vs, vo, b.nv) <= 1e-13 and rel_linf(us, uo, b.nv) <= 1e-13, (e, rel_linf(vs, vo, b.nv))
