"""The learned con2prim seed on the viscous equations (2+1D Israel-Stewart
shear, the nested inversion of system.f90:564-666): pairs from viscous runs;
seeded explicit RK2 and IMEX RK2 steps, single grid and batched, against the
oracle's warm-started inversion iterated to the same fixed point
(ECHO_C2P_NEWTON), and that converged mode itself on the device.

Tolerances, relative L-inf per field group (rho; v; p; Pi and pi
together): the converged mode against the oracle, the plain path's bars
(1e-13 exact build, 1e-12 product build); seeded against warm-started,
1e-11: two starts of the fixed point meet within its Newton's step
tolerance (1e-12 of p) at every inversion, and the steps carry that on.
"""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import events as EV
from echo_gpu import params as P
from echo_gpu import seed as S
from echo_gpu.batch import DONE, Batch, event_grid
from echo_gpu.lib import Evolve
from helpers import CASES, eos_table, przero_of, rel_linf, setup, smooth_pressure_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    X, T = S.generate_pairs(n_target=150_000, grid=48, steps=9, every=3, viscous=True)
    w, norm, losses = S.train(X, T, steps=1500, batch=4096, lr=3e-3, report_every=100)
    return X, T, w, norm, losses


def test_pairs_and_training(trained):
    X, T, w, norm, losses = trained
    assert X.shape[1] == S.NIN and np.isfinite(X).all() and np.isfinite(T).all()
    assert np.all(X[:, 3:] == 0)  # no B, no E
    assert losses[-1] < 0.1 * losses[0], losses
    idx = np.random.default_rng(5).choice(len(X), 4000, replace=False)
    pred = S.infer(w, norm, X[idx])
    assert np.median(np.abs(pred[:, 0] - T[idx, 0])) < 0.02
    assert np.median(np.abs(pred[:, 1] / T[idx, 1] - 1)) < 0.1


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
@pytest.mark.parametrize("imex", [0, 1])
def test_converged_newton_matches_oracle(exact, tol, imex):
    cfg = CASES["visc2d"]().replace(imex=imex, algo_solver=P.C2P_NEWTON)
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc, tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(6):
        o.step()
        g.step()
    vg, ug = g.download()
    vo, uo = o.state()
    assert g.stats().errcode == 0
    ev, eu = rel_linf(vg, vo, cfg.nv), rel_linf(ug, uo, cfg.nv)
    assert ev <= tol and eu <= tol, (ev, eu)


@pytest.mark.parametrize("imex", [0, 1])
def test_seeded_steps_match_oracle(trained, imex):
    _, _, w, norm, _ = trained
    cfg = CASES["visc2d"]().replace(imex=imex, algo_solver=P.C2P_NEWTON)
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(cfg.replace(algo_solver=P.C2P_MLP).to_c(przero=pc.przero), tab)
    g.set_seed_network(w, norm)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(6):
        o.step()
        g.step()
    st = g.stats()
    assert st.errcode == 0
    vg, ug = g.download()
    vo, uo = o.state()
    ev, eu = rel_linf(vg, vo, cfg.nv), rel_linf(ug, uo, cfg.nv)
    print(f"imex={imex}: seeded vs plain oracle {ev:.2e} (v), {eu:.2e} (u); fallbacks {st.seed_fallbacks}")
    assert ev <= 1e-11 and eu <= 1e-11, (ev, eu)
    assert st.seed_fallbacks < 6 * 2 * cfg.ncell


def test_batched_seeded_events_match_oracle(trained):
    """Seeded IMEX RK2 events of uneven grids in one batch against the
    oracle's plain inversion of each event, to the end time."""
    _, _, w, norm, _ = trained
    es = EV.small_events(base=EV.batched_viscous().cfg.replace(imex=1, algo_solver=P.C2P_MLP), tmax=0.7)
    tab = eos_table()
    v = EV.event_primitives(es, tab)
    pc = es.cfg.to_c(przero=przero_of(es.cfg), smooth_pressure=smooth_pressure_of(es.cfg))
    b = Batch(pc, tab, [event_grid(*es.grid(e)) for e in range(es.nev)])
    with pytest.raises(RuntimeError):
        b.run(1)  # no network loaded
    b.set_seed_network(w, norm)
    b.upload(v, None, es.cfg.tstart, es.tmax)
    b.run_to_end(chunk=4)
    st = b.status()
    vg, ug = b.download()
    assert sum(s["seed_fallbacks"] for s in st) < sum(s["steps"] for s in st) * 2 * b.ncell
    for e, (vs, us) in enumerate(zip(b.split(vg), b.split(ug))):
        cfg = es.event_config(e).replace(algo_solver=P.C2P_NEWTON)
        o = O.Oracle(cfg.to_c(przero=przero_of(cfg), smooth_pressure=smooth_pressure_of(cfg)), tab)
        o.set_state(v[e], None, cfg.tstart)
        o.set_tout(es.tmax, es.tmax - cfg.tstart, es.tmax)
        n = 0
        while o.t < es.tmax:
            o.step()
            n += 1
        vo, uo = o.state()
        assert st[e]["state"] == DONE and st[e]["steps"] == n, (e, st[e], n)
        ev, eu = rel_linf(vs, vo, b.nv), rel_linf(us, uo, b.nv)
        assert ev <= 1e-11 and eu <= 1e-11, (e, ev, eu)
