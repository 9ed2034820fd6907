"""Synthetic initial conditions and equation-of-state tables.

Initial-condition generation is outside the step path; this module only
produces the primitive grids that the step consumes, in the reference's
Fortran order v(ix,iy,iz,k) (flattened with x fastest).

* optical Glauber: init.f90:852-1242 (thickness, wound, bincoll, calc_enedens)
* Monte Carlo Glauber: the algorithm of glaubermc.f90:80-873 (Woods-Saxon
  sampling, collision criterion d^2 <= sigma/pi, Gaussian smearing) with a
  seeded numpy generator in place of gfortran's rand()
* tabulated EoS: the file format read by eos.f90:265-334
"""
from __future__ import annotations

import math

import numpy as np

from . import params as P

HC3 = 0.00768351  # (hbar c)^3 as written in eos.f90:275

NUCLEI = {  # nuclear_data.dat: A, R (fm), a (fm), rho0 (fm^-3)
    "Au": (197.0, 6.38, 0.535, 0.1693),
    "Pb": (208.0, 6.62, 0.546, 0.1604),
}


# ----------------------------------------------------------------------------
# equation of state
# ----------------------------------------------------------------------------
def crossover_eos(n: int = 2048, emin: float = 1e-3, emax: float = 1e3,
                  cs2_min: float = 0.15, e_dip: float = 0.5,
                  width: float = 1.0, g_dof: float = 37.0) -> np.ndarray:
    """Smooth-crossover EoS on ``n`` log-spaced energy densities.

    c_s^2(e) = 1/3 - (1/3 - cs2_min) exp(-ln(e/e_dip)^2 / (2 width^2));
    p(e) = integral of c_s^2 de (trapezoid on a 16x finer grid);
    d ln s = de/(e+p);  T = (e+p)/s normalised to the ideal-gas limit
    e = g pi^2/30 T^4/(hbar c)^3 at the top of the table.
    Returns rows (T, e, p, c_s^2) with e, p in GeV/fm^3, T in GeV.
    """
    fine = 16
    le = np.linspace(math.log(emin), math.log(emax), (n - 1) * fine + 1)
    e = np.exp(le)
    cs2 = 1.0 / 3.0 - (1.0 / 3.0 - cs2_min) * np.exp(-((le - math.log(e_dip)) ** 2) / (2 * width**2))
    p = np.empty_like(e)
    p[0] = cs2[0] * e[0]
    p[1:] = p[0] + np.cumsum(0.5 * (cs2[1:] + cs2[:-1]) * np.diff(e))
    dlns = np.diff(e) / (0.5 * ((e + p)[1:] + (e + p)[:-1]))
    lns = np.concatenate([[0.0], np.cumsum(dlns)])
    s = np.exp(lns)
    T = (e + p) / s
    a = g_dof * math.pi**2 / 30.0 / 0.197326**3
    T_ideal_top = (e[-1] / a) ** 0.25
    T *= T_ideal_top / T[-1]
    sel = slice(0, None, fine)
    return np.stack([T[sel], e[sel], p[sel], cs2[sel]], axis=1)


def write_eos_file(path: str, table: np.ndarray) -> None:
    """Write a table in the reference's eos_data format (eos.f90:288-327):
    first line the number of entries, then T, e/T^4*hc3, p/T^4*hc3, c_s^2."""
    with open(path, "w") as f:
        f.write(f"{len(table)}\n")
        for T, e, p, c in table:
            f.write(f"{T:.17g} {e / T**4 * HC3:.17g} {p / T**4 * HC3:.17g} {c:.17g}\n")


def read_eos_file(path: str) -> np.ndarray:
    """Read a table as read_data_from_tabulated_file does (eos.f90:322-327):
    e = col2/hc3*T**4.0, p = col3/hc3*T**4.0."""
    with open(path) as f:
        n = int(f.readline().split()[0])
        rows = [list(map(float, f.readline().split()[:4])) for _ in range(n)]
    out = np.empty((n, 4))
    for i, (T, ce, cp, c) in enumerate(rows):
        t4 = math.pow(T, 4.0)
        out[i] = (T, ce / HC3 * t4, cp / HC3 * t4, c)
    return out


def eos_table_loaded(**kw) -> np.ndarray:
    """The crossover table after a write/read round trip through the
    reference file format, i.e. exactly what the reference would load."""
    import os
    import tempfile

    tab = crossover_eos(**kw)
    fd, path = tempfile.mkstemp(suffix=".dat")
    os.close(fd)
    try:
        write_eos_file(path, tab)
        return read_eos_file(path)
    finally:
        os.remove(path)


def table_pressure(tab: np.ndarray, e: np.ndarray) -> np.ndarray:
    """p(e) by the bracket + linear interpolation of get_pressure."""
    te, tp = tab[:, 1], tab[:, 2]
    e = np.asarray(e, dtype=np.float64)
    h = np.searchsorted(te, e, side="left")
    h = np.clip(h, 1, len(te) - 1)
    e1, e2, p1, p2 = te[h - 1], te[h], tp[h - 1], tp[h]
    return p1 + (p2 - p1) * (e - e1) / (e2 - e1)


def table_temperature_to_pressure(tab: np.ndarray, temp: float) -> float:
    """p at temperature ``temp`` by interpolation in the table."""
    T, p = tab[:, 0], tab[:, 2]
    return float(np.interp(temp, T, p))


# ----------------------------------------------------------------------------
# Glauber models
# ----------------------------------------------------------------------------
def ws_thickness(r: np.ndarray, R: float, a: float, rho0: float,
                 zmax_factor: float = 2.0, nz: int = 4001) -> np.ndarray:
    """T(r) = int rho0/(exp((sqrt(r^2+z^2)-R)/a)+1) dz over |z| < 2R
    (init.f90:1164-1216 integrates the same range)."""
    r = np.asarray(r, dtype=np.float64)
    z = np.linspace(-zmax_factor * R, zmax_factor * R, nz)
    rr = np.sqrt(r[..., None] ** 2 + z**2)
    rho = rho0 / (np.exp((rr - R) / a) + 1.0)
    return np.trapezoid(rho, z, axis=-1)


def optical_glauber(x: np.ndarray, y: np.ndarray, b: float, nucleus: str = "Au",
                    sigma_in_mb: float = 42.0, ah: float = 0.15,
                    peak: float = 30.0) -> np.ndarray:
    """Energy density of calc_enedens for nz=1 (init.f90:902-912):
    e = ecenter (ah N_coll + (1-ah)(T_A^w + T_B^w)) / (same at b=0, r=0),
    rescaled so its maximum is ``peak``."""
    A, R, a, rho0 = NUCLEI[nucleus]
    sig = sigma_in_mb / 10.0  # fm^2 (common.f90:2259)
    X, Y = np.meshgrid(x, y, indexing="xy")
    rp = np.sqrt((X + 0.5 * b) ** 2 + Y**2)
    rm = np.sqrt((X - 0.5 * b) ** 2 + Y**2)
    rs = np.linspace(0.0, float(max(rp.max(), rm.max())) + 0.01, 2048)
    Ts = ws_thickness(rs, R, a, rho0)
    tp = np.interp(rp, rs, Ts)
    tm = np.interp(rm, rs, Ts)
    tA = (1.0 - (1.0 - sig * tm / A) ** A) * tp
    tB = (1.0 - (1.0 - sig * tp / A) ** A) * tm
    ncoll = sig * tp * tm
    e = ah * ncoll + (1.0 - ah) * (tA + tB)
    return e * (peak / e.max())


def glauber_sources(b: float, rng: np.random.Generator, nucleus: str = "Pb",
                    sigma_in_mb: float = 70.0) -> tuple[np.ndarray, np.ndarray]:
    """Participants and binary collisions of one Monte Carlo Glauber event:
    Woods-Saxon nucleons of both nuclei (centres at x = -+b/2), a nucleon
    pair collides when d^2 <= sigma/pi (glaubermc.f90:411).  Returns the
    transverse positions (n, 2) of the participants and of the collision
    midpoints."""
    A, R, a, rho0 = NUCLEI[nucleus]
    sig = sigma_in_mb / 10.0
    nA = int(A)

    def sample() -> np.ndarray:
        out = np.empty((0, 3))
        while len(out) < nA:
            m = 4 * nA
            r = rng.uniform(0, 3 * R, m)
            acc = rng.uniform(0, 1, m) < (r / (3 * R)) ** 2 / (np.exp((r - R) / a) + 1)
            r = r[acc]
            ct = rng.uniform(-1, 1, len(r))
            ph = rng.uniform(0, 2 * np.pi, len(r))
            st = np.sqrt(1 - ct**2)
            out = np.concatenate([out, np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], 1)])
        return out[:nA]

    pa = sample()[:, :2] + np.array([-0.5 * b, 0.0])
    pb = sample()[:, :2] + np.array([0.5 * b, 0.0])
    d2 = ((pa[:, None, :] - pb[None, :, :]) ** 2).sum(-1)
    hit = d2 <= sig / np.pi
    parts = np.concatenate([pa[hit.any(1)], pb[hit.any(0)]])
    ia, ib = np.nonzero(hit)
    colls = 0.5 * (pa[ia] + pb[ib])
    return parts, colls


def smear_sources(x: np.ndarray, y: np.ndarray, parts: np.ndarray, colls: np.ndarray,
                  smear: float = 0.5, ah: float = 0.15) -> np.ndarray:
    """Unnormalised energy density (ny, nx): every participant (weight 1-ah)
    and binary collision (weight ah) smeared by a normalised 2D Gaussian of
    width ``smear`` (generate_energy_density_profile, glaubermc.f90:686-873)."""
    X, Y = np.meshgrid(x, y, indexing="xy")
    e = np.zeros_like(X)
    norm = 1.0 / (2 * np.pi * smear**2)
    for (px, py) in parts:
        e += (1 - ah) * norm * np.exp(-((X - px) ** 2 + (Y - py) ** 2) / (2 * smear**2))
    for (px, py) in colls:
        e += ah * norm * np.exp(-((X - px) ** 2 + (Y - py) ** 2) / (2 * smear**2))
    return e


def mc_glauber(x: np.ndarray, y: np.ndarray, b: float, rng: np.random.Generator,
               nucleus: str = "Pb", sigma_in_mb: float = 70.0,
               smear: float = 0.5, ah: float = 0.15,
               peak: float = 30.0) -> np.ndarray:
    """One Monte Carlo Glauber event on the grid x, y, normalised to
    ``peak`` at its maximum."""
    parts, colls = glauber_sources(b, rng, nucleus, sigma_in_mb)
    e = smear_sources(x, y, parts, colls, smear, ah)
    if e.max() <= 0:
        return e
    return e * (peak / e.max())


def eta_profile(eta: np.ndarray, flat: float = 1.0, sig: float = 1.5) -> np.ndarray:
    """H_of_eta without tilting (init.f90:935-970): 1 on the plateau
    |eta| <= flat/2, Gaussian of width sig outside."""
    d = np.abs(eta) - 0.5 * flat
    return np.where(d > 0, np.exp(-(d**2) * 0.5 / sig**2), 1.0)


# ----------------------------------------------------------------------------
# primitive grids for the workloads
# ----------------------------------------------------------------------------
def cell_centres(n: int, lo: float, hi: float) -> np.ndarray:
    d = (hi - lo) / n
    return lo + (np.arange(1, n + 1) - 0.5) * d  # common_grid, common.f90:457


def _pack(fields: list[np.ndarray]) -> np.ndarray:
    """Stack (nz, ny, nx) fields into the Fortran layout v(ix,iy,iz,k)."""
    return np.ascontiguousarray(np.stack(fields, 0)).reshape(-1)


def primitives(cfg, tab: np.ndarray | None = None, seed: int = 7,
               b: float | None = None) -> np.ndarray:
    """Primitive variables of the named workload (flat, Fortran order)."""
    x = cell_centres(cfg.nx, cfg.x1, cfg.x2)
    y = cell_centres(cfg.ny, cfg.y1, cfg.y2)
    z = cell_centres(cfg.nz, cfg.z1, cfg.z2)
    if cfg.viscosity:
        rng = np.random.default_rng(seed)
        e2 = mc_glauber(x, y, 8.0 if b is None else b, rng)
    else:
        e2 = optical_glauber(x, y, 7.0 if b is None else b)
    if cfg.nz > 1:
        H = eta_profile(z)
        e = e2[None, :, :] * H[:, None, None]
    else:
        e = e2[None, :, :]
    e = e + cfg.enezero  # energy floor (the reference adds p(ENEZERO) to p)
    if cfg.eqstate == 3:
        p = table_pressure(tab, e)
    else:
        p = e / 3.0
    shape = e.shape
    rho = np.ones(shape)
    zero = np.zeros(shape)
    fields = [rho, zero, zero, zero, p]
    if cfg.viscosity:
        fields += [zero] * 7
    if cfg.mhd:
        e_c = float(e2.max())
        sigma_m = 0.3 if cfg.mhd == 2 else 0.1
        B0 = math.sqrt(2.0 * sigma_m * e_c)  # magnetisation B^2/(2e) at the centre
        X = np.broadcast_to(x[None, None, :], shape)
        Hz = np.broadcast_to((eta_profile(z) if cfg.nz > 1 else np.ones(1))[:, None, None], shape)
        by = B0 * np.exp(-(X**2) / (2 * 2.5**2)) * np.sqrt(Hz)
        fields += [zero, by, zero]
        if cfg.mhd == 2:
            fields += [zero, zero, zero]  # E = -v x B = 0 at rest
        if cfg.divclean:
            fields += [zero]
    return _pack(fields)


def with_ideal_e(cfg, v: np.ndarray, ideal: float) -> np.ndarray:
    """A resistive state (nv = 12) with its electric field set to `ideal`
    times the ideal-MHD field E = -v x B: covariant E_i = -sqrt(-g) [ijk]
    v^j B^k, raised with g_33 = tau^2 (tau = 1 in Minkowski coordinates)."""
    v = np.array(v, dtype=np.float64).reshape(cfg.nv, -1)
    tau = cfg.tstart if cfg.coordinates == P.BJORKEN else 1.0
    vx, vy, vz, bx, by, bz = v[1], v[2], v[3], v[5], v[6], v[7]
    e_cov = [-tau * (vy * bz - vz * by), -tau * (vz * bx - vx * bz), -tau * (vx * by - vy * bx)]
    v[8], v[9], v[10] = ideal * e_cov[0], ideal * e_cov[1], ideal * e_cov[2] / tau**2
    return v.reshape(-1)


def resistive_flow(cfg, tab, amp: float = 0.2, ideal: float = 0.7) -> np.ndarray:
    """The resistive workload's initial state (at rest, E = 0) given a
    smooth flow along x, y and eta of amplitude `amp` and an electric field
    that is `ideal` times the ideal -v x B: a state with Ohm currents and
    charges from the first step."""
    v = primitives(cfg, tab).reshape(cfg.nv, cfg.nz, cfg.ny, cfg.nx)
    x = cell_centres(cfg.nx, cfg.x1, cfg.x2)
    y = cell_centres(cfg.ny, cfg.y1, cfg.y2)
    z = cell_centres(cfg.nz, cfg.z1, cfg.z2)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    Lx, Lz = cfg.x2 - cfg.x1, max(cfg.z2 - cfg.z1, 1e-300)
    tau = cfg.tstart if cfg.coordinates == P.BJORKEN else 1.0
    v[1] = amp * np.sin(np.pi * Y / Lx) * np.cos(np.pi * Z / Lz)
    v[2] = amp * np.sin(np.pi * X / Lx)
    v[3] = 0.5 * amp / tau * np.sin(np.pi * (X + Y) / Lx)
    return with_ideal_e(cfg, v.reshape(-1), ideal)


def bjorken_uniform(cfg, e0: float = 10.0) -> np.ndarray:
    """Uniform Bjorken flow (zero transverse flow): the analytic solution
    e(tau) = e0 (tau0/tau)^(4/3) for p = e/3."""
    shape = (cfg.nz, cfg.ny, cfg.nx)
    p = np.full(shape, e0 / 3.0)
    z = np.zeros(shape)
    fields = [np.ones(shape), z, z, z, p]
    if cfg.viscosity:
        fields += [z] * 7
    if cfg.mhd:
        fields += [z] * (6 if cfg.mhd == 2 else 3) + ([z] if cfg.divclean else [])
    return _pack(fields)
