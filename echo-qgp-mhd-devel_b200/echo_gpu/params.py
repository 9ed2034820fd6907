"""Run-time parameters of the step path, mirroring ``EchoParams`` in
``include/echo_gpu.h`` field for field.

The field names follow the reference's param.dat keys (parsed in
common.f90:874-1212); defaults are the reference's own (common.f90:485-740).
"""
from __future__ import annotations

import ctypes
import dataclasses

ECHO_MAX_NV = 16

REC = {"TVD2": 0, "CENO3": 1, "WENO3": 2, "WENO5": 3, "PPM4": 4, "MPE3": 5, "MPE5": 6}
RK2, RK3, SSP = 2, 3, 4
MINKOWSKI, BJORKEN = 1, 2
EOS_CONFORMAL, EOS_IDEALGAS, EOS_TABLE = 1, 2, 3
C2P_BRENT, C2P_NEWTON, C2P_MLP = 1, 100, 101


class EchoParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("x1", ctypes.c_double), ("x2", ctypes.c_double),
        ("y1", ctypes.c_double), ("y2", ctypes.c_double),
        ("z1", ctypes.c_double), ("z2", ctypes.c_double),
        ("coordinates", ctypes.c_int),
        ("mhd", ctypes.c_int),
        ("divclean", ctypes.c_int),
        ("viscosity", ctypes.c_int),
        ("bulkvis", ctypes.c_int),
        ("recal", ctypes.c_int),
        ("nrk", ctypes.c_int),
        ("eqstate", ctypes.c_int),
        ("algo_solver", ctypes.c_int),
        ("obtained_zz", ctypes.c_int),
        ("init_type", ctypes.c_int),
        ("enable_smooth_viscosity", ctypes.c_int),
        ("ibc", ctypes.c_int * 3 * 2 * ECHO_MAX_NV),
        ("cfl", ctypes.c_double),
        ("maxdt", ctypes.c_double),
        ("maxspeed", ctypes.c_double),
        ("glm_alpha", ctypes.c_double),
        ("eta_over_s", ctypes.c_double),
        ("tau_pi_coeff", ctypes.c_double),
        ("smooth_pressure", ctypes.c_double),
        ("enezero", ctypes.c_double),
        ("przero", ctypes.c_double),
        ("c2p_tol", ctypes.c_double),
        ("imex", ctypes.c_int),
        ("sigma_el", ctypes.c_double),
        ("sigma_chiral", ctypes.c_double),
    ]


@dataclasses.dataclass
class Config:
    """One workload: grid, physics switches and numerics.

    ``nv`` follows system_setup (system.f90:67-128): 5 hydro variables,
    +7 viscous, +3 magnetic, +1 GLM.
    """

    name: str
    nx: int
    ny: int
    nz: int
    x1: float
    x2: float
    y1: float
    y2: float
    z1: float = -0.5
    z2: float = 0.5
    coordinates: int = BJORKEN
    mhd: int = 0
    divclean: int = 0
    viscosity: int = 0
    bulkvis: int = 0
    recal: str = "WENO5"
    nrk: int = RK2
    eqstate: int = EOS_CONFORMAL
    algo_solver: int = C2P_BRENT
    obtained_zz: int = 1
    init_type: int = 0
    smooth_temp: float = 0.0
    boundary: int = 2          # bound_con: 2 outflow (default), 0 periodic
    cfl: float = 0.4
    maxdt: float = 0.002
    maxspeed: float = 0.995
    glm_alpha: float = 5.0
    eta_over_s: float = 0.08
    tau_pi_coeff: float = 5.0
    enezero: float = 0.001
    tstart: float = 0.4
    steps: int = 10
    c2p_tol: float = 1e-10
    imex: int = 0              # viscous: Israel-Stewart relaxation linearly implicit per stage
    sigma_el: float = 0.0      # EL_COND (resistive runs, mhd = 2)
    sigma_chiral: float = 0.0  # CHIR_COND

    @property
    def nv(self) -> int:
        nv = 12 if self.viscosity else 5
        if self.mhd:
            nv += (6 if self.mhd == 2 else 3) + (1 if self.divclean else 0)
        return nv

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def replace(self, **kw) -> "Config":
        return dataclasses.replace(self, **kw)

    def to_c(self, przero: float, smooth_pressure: float = 0.0) -> EchoParams:
        p = EchoParams()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.x1, p.x2, p.y1, p.y2, p.z1, p.z2 = self.x1, self.x2, self.y1, self.y2, self.z1, self.z2
        p.coordinates = self.coordinates
        p.mhd = self.mhd
        p.divclean = self.divclean
        p.viscosity = self.viscosity
        p.bulkvis = self.bulkvis
        p.recal = REC[self.recal]
        p.nrk = self.nrk
        p.eqstate = self.eqstate
        p.algo_solver = self.algo_solver
        p.obtained_zz = self.obtained_zz
        p.init_type = self.init_type
        p.enable_smooth_viscosity = 1 if (self.viscosity and self.smooth_temp > 0) else 0
        for k in range(ECHO_MAX_NV):
            for s in range(2):
                for d in range(3):
                    p.ibc[k][s][d] = self.boundary
        p.cfl = self.cfl
        p.maxdt = self.maxdt
        p.maxspeed = self.maxspeed
        p.glm_alpha = self.glm_alpha
        p.eta_over_s = self.eta_over_s
        p.tau_pi_coeff = self.tau_pi_coeff
        p.smooth_pressure = smooth_pressure
        p.enezero = self.enezero
        p.przero = przero
        p.c2p_tol = self.c2p_tol
        p.imex = self.imex
        p.sigma_el = self.sigma_el
        p.sigma_chiral = self.sigma_chiral
        return p


def _grid(n: int, d: float) -> tuple[float, float]:
    h = 0.5 * n * d
    return -h, h


def config0() -> Config:
    """2+1D boost-invariant ideal hydro, p=e/3, 101x101, dx=0.2, WENO5+HLL,
    RK2 at CFL 0.4, 100 steps, optical-Glauber Au+Au b=7 fm."""
    x1, x2 = _grid(101, 0.2)
    return Config("ideal-hd-2d-101", 101, 101, 1, x1, x2, x1, x2, -0.5, 0.5,
                  recal="WENO5", nrk=RK2, eqstate=EOS_CONFORMAL, cfl=0.4,
                  maxdt=0.1, enezero=0.001, steps=100)


def config1() -> Config:
    """3+1D ideal RMHD in Milne coordinates, 97x97x81, dx=deta=0.15,
    tabulated crossover EoS, WENO5+HLL+GLM, RK3, 200 steps."""
    x1, x2 = _grid(97, 0.15)
    z1, z2 = _grid(81, 0.15)
    return Config("ideal-rmhd-3d-97x97x81", 97, 97, 81, x1, x2, x1, x2, z1, z2,
                  mhd=1, divclean=1, glm_alpha=10.0, recal="WENO5", nrk=RK3,
                  eqstate=EOS_TABLE, cfl=0.4, maxdt=0.002, enezero=0.02,
                  steps=200)


def config2() -> Config:
    """2+1D Israel-Stewart shear viscous hydro, 201x201, dx=0.1,
    eta/s=0.12, tau_pi=5 eta/(e+p) T, tabulated EoS, MC-Glauber Pb+Pb."""
    x1, x2 = _grid(201, 0.1)
    return Config("viscous-hd-2d-201", 201, 201, 1, x1, x2, x1, x2, -0.5, 0.5,
                  viscosity=1, recal="WENO5", nrk=RK2, eqstate=EOS_TABLE,
                  eta_over_s=0.12, tau_pi_coeff=5.0, smooth_temp=0.08,
                  cfl=0.4, maxdt=0.01, enezero=0.02, steps=100)


def config4() -> Config:
    """3+1D resistive RMHD in Milne coordinates, 193x193x129, dx=deta=0.1,
    config-1 EoS and profile, B_y as config 1 at magnetisation 0.3, E =
    -v x B initially, sigma_el = 5.8 MeV, IMEX-SSP3(4,3,3), 300 steps.
    ENEZERO = 0.05 GeV/fm^3 (param.dat:115): B_y(x, eta) fills the whole y
    range, and at the y edges, where e = ENEZERO, the magnetic work of the
    Bjorken source over one frozen-metric step (dt B^2 / (2 tau) ~ 0.02)
    would take the fluid energy below the table with 0.02."""
    x1, x2 = _grid(193, 0.1)
    z1, z2 = _grid(129, 0.1)
    return Config("resistive-rmhd-3d-193x193x129", 193, 193, 129, x1, x2, x1, x2, z1, z2,
                  mhd=2, divclean=1, glm_alpha=10.0, recal="WENO5", nrk=SSP,
                  eqstate=EOS_TABLE, cfl=0.4, maxdt=0.002, enezero=0.05,
                  sigma_el=0.0058, sigma_chiral=0.0015, steps=300)


def small(cfg: Config, n: int = 12, nz: int | None = None) -> Config:
    """Same physics on a small grid (same spacing), for parity tests."""
    dx = (cfg.x2 - cfg.x1) / cfg.nx
    x1, x2 = _grid(n, dx)
    if cfg.nz > 1:
        nzz = nz if nz is not None else max(4, n - 2)
        dz = (cfg.z2 - cfg.z1) / cfg.nz
        z1, z2 = _grid(nzz, dz)
    else:
        nzz, z1, z2 = 1, cfg.z1, cfg.z2
    return cfg.replace(name=cfg.name + f"-small{n}", nx=n, ny=n, nz=nzz,
                       x1=x1, x2=x2, y1=x1, y2=x2, z1=z1, z2=z2)
