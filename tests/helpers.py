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


def rel_linf(a: np.ndarray, b: np.ndarray, nv: int) -> float:
    """Relative L-inf error over primitives: max over variables of
    max|a-b| / S, where S is the largest |b| in the variable's field group
    (see field_groups)."""
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    worst = 0.0
    for grp in field_groups(nv):
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
}
