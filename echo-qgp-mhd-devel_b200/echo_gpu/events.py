"""Event-by-event workloads: many Monte Carlo Glauber Pb+Pb events, each on
its own transverse grid sized to its fireball.

The batched viscous workload: 512 events, impact parameter b uniform in
[0, 12] fm (seeded), grid n x n with n falling linearly from 161 (b = 0) to
61 (b = 12) at dx = 0.15 fm, so the mean cell count is about 13,150 and the
batch holds about 6.7 M cells; 2+1D Israel-Stewart shear viscous hydro with
the physics of the single-event viscous workload (eta/s = 0.12, tau_pi =
5 eta/(e+p), tabulated crossover EoS, WENO5 + HLL, RK2, CFL 0.4), every
event run to tau = 10 fm/c with its own CFL-limited dt.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import initial as I
from . import params as P


@dataclasses.dataclass
class EventSet:
    cfg: P.Config             # shared physics; its grid fields describe event 0
    b: np.ndarray             # impact parameters (fm)
    n: np.ndarray             # grid size n x n of each event
    dx: float
    tmax: float

    @property
    def nev(self) -> int:
        return len(self.n)

    def grid(self, e: int):
        """(nx, ny, nz, x1, x2, y1, y2, z1, z2) of event e."""
        h = 0.5 * int(self.n[e]) * self.dx
        return (int(self.n[e]), int(self.n[e]), 1, -h, h, -h, h, -0.5, 0.5)

    def event_config(self, e: int) -> P.Config:
        nx, ny, nz, x1, x2, y1, y2, z1, z2 = self.grid(e)
        return self.cfg.replace(name=f"{self.cfg.name}-ev{e}", nx=nx, ny=ny, nz=nz,
                                x1=x1, x2=x2, y1=y1, y2=y2, z1=z1, z2=z2)

    @property
    def cells(self) -> np.ndarray:
        return self.n.astype(np.int64) ** 2


def batched_eos_table() -> np.ndarray:
    """The crossover EoS of the single-event workloads (initial.crossover_eos)
    extended from e >= 1e-3 down to 1e-7 GeV/fm^3 at the same number of
    points per decade: a run to tau = 10 fm/c dilutes the edge of a central
    fireball below 1e-3, where the shorter table stops the run with the
    reference's EoS range error 125 (p below the table)."""
    return I.eos_table_loaded(emin=1e-7, n=3414)


def batched_viscous(nev: int = 512, seed: int = 2024, dx: float = 0.15, nmin: int = 61, nmax: int = 161,
                    bmax: float = 12.0, tmax: float = 10.0, maxdt: float = 1.0, enezero: float = 0.05) -> EventSet:
    """The batched event-by-event viscous workload (see the module text).
    ``maxdt`` defaults to 1 fm/c so that dt is the CFL one (evolve_dt,
    evolve.f90:723-764) of each event.  The energy floor is the ENEZERO of
    the reference's param.dat (0.05 GeV/fm^3): with the 0.02 of the single
    event workloads, the rarefied edge of the most central events ends in a
    failed con2prim repair (reference code 1) before tau = 10 fm/c."""
    rng = np.random.default_rng(seed)
    b = np.sort(rng.uniform(0.0, bmax, nev))
    n = np.rint(nmax - (nmax - nmin) * b / bmax).astype(np.int64)
    base = P.config2()
    h = 0.5 * int(n[0]) * dx
    # IMEX RK2, the viscous workload's scheme (the Israel-Stewart relaxation
    # linearly implicit per stage)
    cfg = base.replace(name="batched-viscous-2d", nx=int(n[0]), ny=int(n[0]), x1=-h, x2=h, y1=-h, y2=h,
                       maxdt=maxdt, enezero=enezero, imex=1)
    return EventSet(cfg=cfg, b=b, n=n, dx=dx, tmax=tmax)


def small_events(ns=(9, 13, 11, 17, 15), bs=(2.0, 6.0, 9.0, 0.5, 4.0), dx: float = 0.15,
                 tmax: float = 0.9, base: P.Config | None = None, maxdt: float = 1.0) -> EventSet:
    """A handful of small events of different sizes for parity tests."""
    base = P.config2() if base is None else base
    n = np.array(ns, dtype=np.int64)
    h = 0.5 * int(n[0]) * dx
    cfg = base.replace(name="batched-small", nx=int(n[0]), ny=int(n[0]), x1=-h, x2=h, y1=-h, y2=h, maxdt=maxdt)
    return EventSet(cfg=cfg, b=np.array(bs, dtype=np.float64), n=n, dx=dx, tmax=tmax)


def event_sources(es: EventSet, seed: int = 11):
    """Participants and collision midpoints of every event (seeded)."""
    rng = np.random.default_rng(seed)
    return [I.glauber_sources(float(b), rng) for b in es.b]


def event_primitives(es: EventSet, tab, sources=None, seed: int = 11, peak: float = 30.0,
                     smear: float = 0.5, ah: float = 0.15) -> list[np.ndarray]:
    """Primitive grids of every event (numpy smearing), Fortran order: rho = 1,
    v = 0, p = p(e + ENEZERO) from the table, pi^{mu nu} = 0."""
    if sources is None:
        sources = event_sources(es, seed)
    out = []
    for e in range(es.nev):
        cfg = es.event_config(e)
        x = I.cell_centres(cfg.nx, cfg.x1, cfg.x2)
        y = I.cell_centres(cfg.ny, cfg.y1, cfg.y2)
        parts, colls = sources[e]
        e2 = I.smear_sources(x, y, parts, colls, smear, ah)
        if e2.max() > 0:
            e2 = e2 * (peak / e2.max())
        out.append(primitives_from_energy(cfg, tab, e2))
    return out


def primitives_from_energy(cfg: P.Config, tab, e2: np.ndarray) -> np.ndarray:
    e = e2[None, :, :] + cfg.enezero
    p = I.table_pressure(tab, e) if cfg.eqstate == P.EOS_TABLE else e / 3.0
    one = np.ones(e.shape)
    zero = np.zeros(e.shape)
    fields = [one, zero, zero, zero, p]
    if cfg.viscosity:
        fields += [zero] * 7
    return np.ascontiguousarray(np.stack(fields, 0)).reshape(-1)
