"""IMEX RK2 for the viscous equations, on the CPU oracle.

The reference integrates the Israel-Stewart relaxation -(pi + 2 eta sigma)/
tau_pi explicitly (its viscous runs are plain RK2, system.f90:1653-1743), so
a time step above ~2 gamma tau_pi blows up.  With ``imex = 1`` the
relaxation term of every stress component is taken at the new stage value,
linearly implicitly; everything else stays explicit.  There is no reference
output for this scheme, so it is checked against its limits:

* tau_pi >> dt: it approaches the reference's explicit scheme, the gap
  shrinking at least in proportion to dt / tau_pi;
* tau_pi ~ dt: both schemes converge to the same solution as dt shrinks;
* tau_pi -> 0 (explicit scheme unstable): it is stable and reproduces the
  Navier-Stokes limit pi = -2 eta sigma -- on Bjorken flow with constant
  eta, e(tau) = e0 (tau0/tau)^(4/3) + 4 eta (tau^(1/3) - tau0^(1/3)) /
  tau^(4/3) and tau^2 pi^{eta eta} = -4 eta / (3 tau), pi^{xx} = pi^{yy} =
  2 eta / (3 tau), first order in dt.
"""
import ctypes

import numpy as np
import pytest

import pyoracle as O
from echo_gpu import initial as I
from echo_gpu import params as P
from echo_gpu.lib import load
from helpers import CASES, rel_linf, setup

ETA = 0.2
E0 = 10.0
T0 = 0.4


def bjorken_visc(dt, coeff, imex):
    """Uniform viscous Bjorken flow on a 6x6 grid, p = e/3, eta = ETA
    (init_type 2 makes eta the eta_over_s value itself, viscous.f90:
    169-171), tau_pi = coeff eta / (T s)."""
    return P.small(P.config0(), 6).replace(viscosity=1, init_type=2, eta_over_s=ETA, tau_pi_coeff=coeff,
                                           maxdt=dt, cfl=10.0, imex=imex)


def run_bjorken(dt, coeff, imex, tend=0.8):
    cfg = bjorken_visc(dt, coeff, imex)
    o = O.Oracle(cfg.to_c(przero=cfg.enezero / 3))
    o.set_state(I.bjorken_uniform(cfg, E0), None, T0)
    for _ in range(int(round((tend - T0) / dt))):
        o.step()
    v, _ = o.state()
    v = v.reshape(12, -1)
    if np.all(np.isfinite(v)):
        assert np.all(np.ptp(v, axis=1) == 0.0)  # uniform stays uniform
    return o.t, v[:, 0]


def navier_stokes_energy(t):
    return E0 * (T0 / t) ** (4.0 / 3.0) + 4.0 * ETA * (t ** (1.0 / 3.0) - T0 ** (1.0 / 3.0)) / t ** (4.0 / 3.0)


def test_stiff_limit_is_navier_stokes():
    errs = []
    for dt in (0.02, 0.01, 0.005):
        t, v = run_bjorken(dt, 1e-6, imex=1)
        assert abs(t - 0.8) < 1e-12
        e = 3.0 * v[4]
        ns_pl = -4.0 * ETA / (3.0 * t)
        errs.append((abs(e / navier_stokes_energy(t) - 1.0), abs(t * t * v[11] / ns_pl - 1.0),
                     abs(v[9] / (2.0 * ETA / (3.0 * t)) - 1.0)))
        assert v[9] == v[10] and v[5] == 0.0 and v[6] == v[7] == v[8] == 0.0
    errs = np.array(errs)
    assert np.all(errs[-1] < 0.03), errs
    ratio = errs[:-1] / errs[1:]
    assert np.all((ratio > 1.8) & (ratio < 2.2)), ratio  # first order in dt


def test_stiff_limit_breaks_the_explicit_scheme():
    # the same run with the reference's explicit relaxation: dt / tau_pi ~ 1e6
    t, v = run_bjorken(0.01, 1e-6, imex=0, tend=0.45)
    assert not np.all(np.isfinite(v))


def test_refinement_converges_to_the_explicit_scheme():
    """tau_pi of a few dt: the energy gap between the two schemes is O(dt);
    the stress gap shrinks too (more slowly at the coarsest step, where the
    initial relaxation layer from pi = 0 spans only a few steps)."""
    ge, gp = [], []
    for dt in (0.01, 0.005, 0.0025):
        _, vi = run_bjorken(dt, 0.5, imex=1)
        _, ve = run_bjorken(dt, 0.5, imex=0)
        ge.append(abs(vi[4] / ve[4] - 1.0))
        gp.append(abs(vi[11] / ve[11] - 1.0))
    ge, gp = np.array(ge), np.array(gp)
    assert ge[0] < 1e-3 and gp[-1] < 2e-3, (ge, gp)
    ratio = ge[:-1] / ge[1:]
    assert np.all((ratio > 1.8) & (ratio < 2.2)), (ge, ratio)
    assert np.all(np.diff(gp) < 0), gp


def _visc2d(coeff, imex, steps=6):
    cfg = CASES["visc2d"]().replace(tau_pi_coeff=coeff, imex=imex)
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    for _ in range(steps):
        o.step()
    return o.state()[0], cfg.nv


def test_slow_relaxation_approaches_the_explicit_scheme():
    """The seeded 2+1D viscous state (tabulated EoS, gradients, shear):
    the relative gap to the explicit scheme falls with tau_pi at least like
    dt/tau_pi -- here like its square, because the stresses start at zero
    and their change over a step is itself O(dt/tau_pi)."""
    gaps = []
    for coeff in (50.0, 500.0):
        vi, nv = _visc2d(coeff, 1)
        ve, _ = _visc2d(coeff, 0)
        gaps.append(rel_linf(vi, ve, nv))
    assert gaps[1] < 1e-4, gaps
    assert gaps[0] / gaps[1] > 5.0, gaps


def test_imex_is_rejected_with_the_ssp_scheme():
    """The IMEX-SSP3(4,3,3) stage logic keeps its own stiff terms; imex = 1
    there is refused before any device call (host-side check)."""
    cfg = CASES["visc2d"]().replace(nrk=P.SSP, imex=1)
    pc, tab, _ = setup(cfg)
    with pytest.raises(ValueError):
        O.Oracle(pc, tab)
    lib = load(exact=False)
    ctx = ctypes.c_void_p()
    t = np.ascontiguousarray(tab, dtype=np.float64)
    rc = lib.echo_gpu_init(ctypes.byref(pc), t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(t),
                           ctypes.byref(ctx))
    assert rc == -3 and not ctx.value  # ECHO_ERR_UNSUPPORTED
