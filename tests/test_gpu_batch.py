"""Batched event-by-event runs against the CPU oracle, event by event.

Each event of a batch must evolve exactly as the reference evolves it
alone: the oracle runs every event through its own time loop (tout = tmax,
stop at t >= tmax, echo.f90:185-262) and the batch must reach the same
state after the same number of steps.  Tolerances are those of the single
grid: 1e-13 (exact build), 1e-12 (product build), relative L-inf per field
group.
"""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import events as EV
from echo_gpu import initial as I
from echo_gpu import params as P
from echo_gpu.batch import COOLED, CRASHED, DONE, SLOTS, Batch, event_grid
from helpers import eos_table, przero_of, rel_linf, smooth_pressure_of

pytestmark = pytest.mark.gpu


def _params(cfg):
    return cfg.to_c(przero=przero_of(cfg), smooth_pressure=smooth_pressure_of(cfg))


def _batch(es, v, exact=True, u=None):
    tab = eos_table() if es.cfg.eqstate == P.EOS_TABLE else None
    b = Batch(_params(es.cfg), tab, [event_grid(*es.grid(e)) for e in range(es.nev)], exact=exact)
    b.upload(v, u, es.cfg.tstart, es.tmax)
    return b


def _oracle_event(es, e, v, u=None):
    """Event e alone on the oracle, to t >= tmax; returns (v, u, steps, error)."""
    cfg = es.event_config(e)
    tab = eos_table() if cfg.eqstate == P.EOS_TABLE else None
    o = O.Oracle(_params(cfg), tab)
    o.set_state(v, u, cfg.tstart)
    o.set_tout(es.tmax, es.tmax - cfg.tstart, es.tmax)
    steps, err = 0, None
    while o.t < es.tmax:
        try:
            o.step()
        except RuntimeError as ex:
            err = ex
            break
        steps += 1
    vo, uo = o.state()
    return vo, uo, steps, err


@pytest.fixture(scope="module")
def small():
    es = EV.small_events()
    v = EV.event_primitives(es, eos_table())
    ref = [_oracle_event(es, e, v[e]) for e in range(es.nev)]
    return es, v, ref


@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
def test_batch_matches_oracle_per_event(small, exact, tol):
    es, v, ref = small
    b = _batch(es, v, exact=exact)
    b.run_to_end(chunk=4)
    st = b.status()
    vg, ug = b.download()
    steps = [r[2] for r in ref]
    assert len(set(steps)) > 1, steps  # the events need different numbers of steps
    for e, (vs, us) in enumerate(zip(b.split(vg), b.split(ug))):
        vo, uo, n, err = ref[e]
        assert err is None
        assert st[e]["state"] == DONE and st[e]["steps"] == n, (e, st[e], n)
        assert abs(st[e]["t"] - es.tmax) <= 1e-12
        assert rel_linf(vs, vo, b.nv) <= tol and rel_linf(us, uo, b.nv) <= tol, (e, rel_linf(vs, vo, b.nv))


def test_batch_launch_shapes_do_not_change_results(small):
    """Persistent grids, one CTA per tile, the autotuned shapes and a
    different event order give the same bits."""
    es, v, _ = small
    ref = _batch(es, v, exact=False)
    ref.run(5)
    v0, u0 = ref.download()
    for ctas, order in [([148] * 5, None), ([1, 2, 3, 1, 2], None), ([0] * 5, list(range(es.nev))[::-1])]:
        b = _batch(es, v, exact=False)
        b.set_schedule(ctas, order)
        b.run(5)
        v1, u1 = b.download()
        assert np.array_equal(v0, v1) and np.array_equal(u0, u1), (ctas, order)
    b = _batch(es, v, exact=False)
    b.run(1)
    ms = b.autotune(reps=2)
    assert set(ms) == set(SLOTS)
    b.run(4)
    v1, u1 = b.download()
    assert np.array_equal(v0, v1) and np.array_equal(u0, u1), b.get_schedule()


def test_tiles_and_one_launch_per_stage_do_not_change_results(small):
    """Tile lengths of 256 and 512 faces or cells, and the whole stage as one
    cooperative launch (all phases, grid-wide barriers between them) with the
    largest resident grid and with one CTA per SM, give the bits of the
    default one-launch-per-phase run."""
    es, v, _ = small
    ref = _batch(es, v, exact=True)
    ref.run(5)
    v0, u0 = ref.download()
    for tiles, mode, grid in [((256, 512), 0, 0), ((512, 256), 0, 0), ((128, 128), 1, 0), ((256, 256), 1, 148),
                              ((512, 128), 1, 0)]:
        b = _batch(es, v, exact=True)
        b.set_tiles(*tiles)
        b.set_mode(mode, grid)
        b.run(5)
        b.sync()
        v1, u1 = b.download()
        assert np.array_equal(v0, v1) and np.array_equal(u0, u1), (tiles, mode, grid, b.tuning())
        assert b.tuning()["mode"] == ("cooperative" if mode else "phased")


def test_cooperative_batch_matches_oracle_to_the_end(small):
    """Every event run to tmax with one launch per stage meets the oracle
    running it alone, step count and state."""
    es, v, ref = small
    b = _batch(es, v, exact=True)
    b.set_mode(1)
    b.run_to_end(chunk=4)
    b.sync()
    st = b.status()
    vg, ug = b.download()
    for e, (vs, us) in enumerate(zip(b.split(vg), b.split(ug))):
        vo, uo, n, err = ref[e]
        assert st[e]["state"] == DONE and st[e]["steps"] == n, (e, st[e], n)
        assert rel_linf(vs, vo, b.nv) <= 1e-13 and rel_linf(us, uo, b.nv) <= 1e-13


def test_autotune_search_space_and_choice(small):
    """The autotuner times every tile length with every launch shape per
    slot and both ways of running a stage, reports them, and its choice
    changes no bit."""
    es, v, _ = small
    ref = _batch(es, v, exact=False)
    ref.run(5)
    v0, u0 = ref.download()
    b = _batch(es, v, exact=False)
    b.run(1)
    b.autotune(reps=2)
    rows = b.autotune_report()
    upd = [r for r in rows if r["slot"] == "update"]
    assert {r["tile"] for r in upd} == {128, 256, 512}
    stages = [r for r in rows if r["slot"] == "stage"]
    assert {r["mode"] for r in stages} == {"phased", "cooperative"}
    print(b.tuning(), min(stages, key=lambda r: r["ms"]))
    b.run(4)
    v1, u1 = b.download()
    assert np.array_equal(v0, v1) and np.array_equal(u0, u1), b.tuning()


def test_crashed_event_is_abandoned_alone(small):
    """A 3x3 block of negative conserved energy in event 1: the inversion
    and its neighbour-average repair fail (reference code 1,
    evolve.f90:836-858), the event is dropped, and the other events carry
    on exactly as before."""
    es, v, ref = small
    tab = eos_table()
    u = []
    for e in range(es.nev):
        o = O.Oracle(_params(es.event_config(e)), tab)
        o.set_state(v[e], None, es.cfg.tstart)
        u.append(o.state()[1])
    bad = 1
    n = int(es.n[bad])
    uu = u[bad].reshape(12, n, n).copy()
    c = n // 2
    uu[4, c - 1:c + 2, c - 1:c + 2] = -1.0
    u[bad] = uu.reshape(-1)
    vo, uo, steps, err = _oracle_event(es, bad, v[bad], u[bad])
    assert err is not None and steps == 0
    b = _batch(es, v, exact=True, u=u)
    b.run_to_end(chunk=4)
    st = b.status()
    assert st[bad]["state"] == CRASHED and st[bad]["errcode"] == 1 and st[bad]["steps"] == 0
    vg, ug = b.download()
    for e, vs in enumerate(b.split(vg)):
        if e == bad:
            continue
        assert st[e]["state"] == DONE and st[e]["steps"] == ref[e][2]
        assert rel_linf(vs, ref[e][0], b.nv) <= 1e-13


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_of_hydro_and_mhd_events(mode):
    """The batch runs every equation set: ideal hydro (2+1D) and ideal RMHD
    with GLM cleaning (3+1D events: three face lists), one launch per phase
    or per stage."""
    for base, ns in [(P.config0(), (9, 12, 7)), (P.config1(), (7, 9, 8))]:
        es = EV.small_events(ns=ns, bs=(3.0, 7.0, 5.0), base=base, tmax=0.41 if base.mhd else 0.8,
                             maxdt=base.maxdt if base.mhd else 1.0)
        tab = eos_table() if base.eqstate == P.EOS_TABLE else None
        grids, vs = [], []
        for e in range(es.nev):
            n = int(es.n[e])
            cfg = P.small(base, n, nz=n if base.nz > 1 else None)
            grids.append((cfg.nx, cfg.ny, cfg.nz, cfg.x1, cfg.x2, cfg.y1, cfg.y2, cfg.z1, cfg.z2))
            vs.append(I.primitives(cfg, tab, b=float(es.b[e])))
        es.grid = lambda e, g=grids: g[e]
        b = _batch(es, vs, exact=True)
        b.set_mode(mode)
        b.run_to_end(chunk=4)
        st = b.status()
        vg, _ = b.download()
        for e, vv in enumerate(b.split(vg)):
            vo, uo, n, err = _oracle_event(es, e, vs[e])
            assert err is None and st[e]["state"] == DONE and st[e]["steps"] == n, (base.name, e, st[e], n)
            assert rel_linf(vv, vo, b.nv) <= 1e-13, (base.name, e)


def test_glauber_initial_state_matches_numpy(small):
    """The on-device Monte Carlo Glauber smearing and EoS step give the
    primitives of the numpy generator (same sources), and u their
    system_prim2cons."""
    es, v, _ = small
    srcs = EV.event_sources(es)
    b = Batch(_params(es.cfg), eos_table(), [event_grid(*es.grid(e)) for e in range(es.nev)])
    b.glauber(srcs, es.cfg.tstart, es.tmax)
    vg, ug = b.download()
    for e, (vs, us) in enumerate(zip(b.split(vg), b.split(ug))):
        o = O.Oracle(_params(es.event_config(e)), eos_table())
        o.set_state(v[e], None, es.cfg.tstart)
        vo, uo = o.state()
        assert rel_linf(vs, vo, b.nv) <= 1e-12 and rel_linf(us, uo, b.nv) <= 1e-12, e


def _oracle_event_stop(es, e, v, freeze_type, temp_end):
    """Event e alone on the oracle with the check_temp stop at the top of its
    time loop (echo.f90:187-190); returns (v, steps, cooled)."""
    cfg = es.event_config(e)
    o = O.Oracle(_params(cfg), eos_table())
    o.set_state(v, None, cfg.tstart)
    o.set_tout(es.tmax, es.tmax - cfg.tstart, es.tmax)
    steps = 0
    while o.t < es.tmax:
        if o.check_temp(freeze_type) < temp_end:
            return o.state()[0], steps, True
        o.step()
        steps += 1
    return o.state()[0], steps, False


def test_batch_check_temp_stop(small):
    """Per-event check_temp: events whose maximum energy density falls below
    TEMP_END stop there (ECHO_EVENT_COOLED), the others run to tmax; every
    event matches the oracle running it with the same stop criterion."""
    es, v, _ = small
    # scale each event's pressure so the events cool below the threshold at
    # different steps
    tab = eos_table()
    vs = []
    for e, fac in enumerate((0.35, 0.5, 0.7, 1.0, 0.25)):
        x = v[e].reshape(12, -1).copy()
        en = np.interp(x[4], tab[:, 2], tab[:, 1])
        x[4] = I.table_pressure(tab, fac * en)
        vs.append(x.reshape(-1))
    temp_end = 7.0
    ref = [_oracle_event_stop(es, e, vs[e], 1, temp_end) for e in range(es.nev)]
    cooled = [r[2] for r in ref]
    assert any(cooled) and not all(cooled), [r[1:] for r in ref]
    for exact, tol in ((True, 1e-13), (False, 1e-12)):
        b = _batch(es, vs, exact=exact)
        b.set_stop(1, temp_end)
        b.run_to_end(chunk=3)
        st = b.status()
        vg, _ = b.download()
        for e, vv in enumerate(b.split(vg)):
            vo, n, c = ref[e]
            assert st[e]["state"] == (COOLED if c else DONE) and st[e]["steps"] == n, (e, st[e], n, c)
            assert rel_linf(vv, vo, b.nv) <= tol, e
