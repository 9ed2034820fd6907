"""Host side of the batched event-by-event workload (no GPU): the event
set, the Monte Carlo Glauber sources and smearing, the extended EoS table."""
import numpy as np

from echo_gpu import events as EV
from echo_gpu import initial as I


def test_event_set_shapes():
    es = EV.batched_viscous()
    assert es.nev == 512
    assert es.n.min() >= 61 and es.n.max() <= 161
    assert np.all(np.diff(es.b) >= 0) and es.b.min() >= 0 and es.b.max() <= 12
    # n falls linearly with b: about 6.7 M cells in all
    assert 6.5e6 < es.cells.sum() < 7.0e6
    # same spacing on every grid, centred
    for e in (0, 100, 511):
        nx, ny, nz, x1, x2, y1, y2, z1, z2 = es.grid(e)
        assert nx == ny == es.n[e] and nz == 1
        assert abs((x2 - x1) / nx - es.dx) < 1e-12 and abs(x1 + x2) < 1e-12
    cfg = es.event_config(3)
    assert cfg.viscosity and cfg.nx == es.n[3] and cfg.enezero == 0.05 and cfg.maxdt == 1.0


def test_glauber_sources_are_seeded_and_physical():
    es = EV.batched_viscous(nev=8)
    a = EV.event_sources(es, seed=5)
    b = EV.event_sources(es, seed=5)
    for (pa, ca), (pb, cb) in zip(a, b):
        assert np.array_equal(pa, pb) and np.array_equal(ca, cb)
    # central Pb+Pb: most of the 416 nucleons participate, several collisions each
    parts, colls = a[0]
    assert 300 < len(parts) <= 416 and len(colls) > len(parts)


def test_smearing_integrates_to_the_weights():
    x = I.cell_centres(201, -10.05, 10.05)
    parts = np.array([[0.3, -0.7]])
    colls = np.array([[1.1, 0.4], [-2.0, 1.5]])
    e = I.smear_sources(x, x, parts, colls, smear=0.5, ah=0.15)
    dx = x[1] - x[0]
    assert abs(e.sum() * dx * dx - (0.85 + 2 * 0.15)) < 1e-10


def test_extended_table_agrees_with_the_workload_table():
    """The batched workload's table is the same crossover EoS extended down to
    1e-7 GeV/fm^3: on the common range p(e) agrees with the 2048-point table
    to interpolation accuracy, and below it the EoS is conformal."""
    t1 = I.eos_table_loaded()
    t2 = EV.batched_eos_table()
    assert t2[0, 1] < 1.1e-7 and abs(t2[-1, 1] - 1e3) < 1e-9
    assert np.all(np.diff(t2[:, 1]) > 0) and np.all(np.diff(t2[:, 2]) > 0)
    e = np.geomspace(1.1e-3, 900.0, 400)
    p1 = I.table_pressure(t1, e)
    p2 = I.table_pressure(t2, e)
    assert np.max(np.abs(p2 / p1 - 1)) < 1e-4
    low = t2[t2[:, 1] < 1e-4]
    assert np.allclose(low[:, 3], 1.0 / 3.0, atol=1e-6)
