"""Shared set-up for the parity tests: workloads on small grids, the oracle
side and the CUDA side fed the same initial state."""
from __future__ import annotations

import functools

import numpy as np

from echo_gpu import initial as I
from echo_gpu import params as P


@functools.lru_cache(maxsize=None)
def eos_table():
    return I.eos_table_loaded()


def przero_of(cfg) -> float:
    if cfg.eqstate == P.EOS_TABLE:
        return float(I.table_pressure(eos_table(), np.array([cfg.enezero]))[0])
    return cfg.enezero / 3.0


def smooth_pressure_of(cfg) -> float:
    if cfg.viscosity and cfg.smooth_temp > 0 and cfg.eqstate == P.EOS_TABLE:
        return I.table_temperature_to_pressure(eos_table(), cfg.smooth_temp)
    return 0.0


def setup(cfg, seed: int = 7, v=None):
    tab = eos_table() if cfg.eqstate == P.EOS_TABLE else None
    pc = cfg.to_c(przero=przero_of(cfg), smooth_pressure=smooth_pressure_of(cfg))
    if v is None:
        v = I.primitives(cfg, tab, seed=seed)
    return pc, tab, v


def field_groups(nv: int) -> list[list[int]]:
    """Variables that share a physical scale: rho; the three velocity
    components; pressure and the viscous stresses (same units); the
    magnetic field together with the GLM scalar psi (psi has the units of B
    and, like B^x or B^eta here, is analytically zero -- normalising it by
    its own round-off-sized maximum would measure noise, not error)."""
    if nv == 5:
        return [[0], [1, 2, 3], [4]]
    if nv == 12:
        return [[0], [1, 2, 3], list(range(4, 12))]
    return [[0], [1, 2, 3], [4], list(range(5, nv))]


RES_GROUPS = [[0], [1, 2, 3], [4], list(range(5, 12))]  # resistive: B, E, psi share a scale


def rel_linf(a: np.ndarray, b: np.ndarray, nv: int, groups=None) -> float:
    """Relative L-inf error over primitives: max over variables of
    max|a-b| / S, where S is the largest |b| in the variable's field group
    (see field_groups; RES_GROUPS for resistive runs)."""
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    worst = 0.0
    for grp in (groups if groups is not None else field_groups(nv)):
        scale = max(float(np.max(np.abs(b[k]))) for k in grp)
        if scale == 0.0:
            scale = 1.0
        for k in grp:
            worst = max(worst, float(np.max(np.abs(a[k] - b[k]))) / scale)
    return worst


CASES = {
    "hd2d": lambda: P.small(P.config0(), 12),
    "rmhd3d": lambda: P.small(P.config1(), 10, nz=8),
    "visc2d": lambda: P.small(P.config2(), 14),
    "res3d": lambda: P.small(P.config4(), 10, nz=8),
}


def resistive_state(cfg, tab, amp: float = 0.2, ideal: float = 0.7) -> np.ndarray:
    """The resistive workload's state with a smooth flow and 0.7 of the
    ideal E (echo_gpu.initial.resistive_flow)."""
    return I.resistive_flow(cfg, tab, amp, ideal)


def gubser(tau, X, Y, q=1.0, T0=0.4):
    """Ideal Gubser flow (the reference's GUBSER_IDEAL initial state,
    init.f90:2901-2961, and the analytic solution it follows): temperature
    (GeV) and radial velocity at Milne time tau."""
    r2 = X * X + Y * Y
    T = T0 / tau * (4 * q * q * tau * tau) ** (1 / 3) / (
        1 + 2 * q * q * (tau * tau + r2) + q**4 * (tau * tau - r2) ** 2) ** (1 / 3)
    vr = 2 * q * q * tau * np.sqrt(r2) / (1 + q * q * tau * tau + q * q * r2)
    return T, vr


def gubser_case(n=81, dx=0.1, dt=0.01, tau0=1.0):
    """Conformal 2+1D Milne run of the Gubser state: config, primitives and
    the cell centres.  e from T by temperature.def (T = 0.148909 e^(1/4))."""
    h = 0.5 * n * dx
    cfg = P.Config("gubser-ideal", n, n, 1, -h, h, -h, h, tstart=tau0, maxdt=dt, cfl=0.4, enezero=1e-6,
                   recal="WENO5", nrk=P.RK2)
    x = I.cell_centres(n, -h, h)
    X, Y = np.meshgrid(x, x, indexing="xy")
    T, vr = gubser(tau0, X, Y)
    r = np.sqrt(X * X + Y * Y)
    rs = np.where(r > 0, r, 1.0)
    p = (T / 0.148909) ** 4 / 3.0
    z = np.zeros_like(X)
    v = np.stack([np.ones_like(X), vr * X / rs, vr * Y / rs, z, p]).reshape(-1)
    return cfg, v, X, Y


# the golden fixtures (tests/golden/<name>.npz): case, parameter changes,
# steps, and whether the state carries the resistive flow and field
GOLDEN_CASES = {
    "hd2d": ("hd2d", {}, 10, False),
    "rmhd3d": ("rmhd3d", {}, 3, False),
    "visc2d": ("visc2d", {}, 5, False),
    # the viscous inversion iterated to its fixed point, IMEX RK2
    "visc2d_fixed_point": ("visc2d", {"imex": 1, "algo_solver": P.C2P_NEWTON}, 5, False),
    # resistive RMHD, IMEX-SSP3(4,3,3) with the implicit Ohm's law
    "res3d": ("res3d", {"sigma_el": 500.0}, 3, True),
}


def golden_setup(name):
    """(cfg, params, eos table, initial primitives, steps) of a golden case."""
    case, changes, steps, resistive = GOLDEN_CASES[name]
    cfg = CASES[case]().replace(**changes)
    pc, tab, v0 = setup(cfg)
    if resistive:
        v0 = resistive_state(cfg, tab)
    return cfg, pc, tab, v0, steps

