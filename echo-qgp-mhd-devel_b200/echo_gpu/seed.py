"""The learned con2prim seed: training pairs from the solver, GPU training,
loading into a run.

Pairs are (conserved, primitive) states the GPU solver itself produces:
ideal-RMHD runs of the 3+1D Milne workload (or resistive runs of the
resistive workload, or viscous runs of the 2+1D viscous workload) at
several energy scales and magnetisations (impact parameters), sampled every
few steps.  The invariants and targets are computed here from u and v
exactly as the device computes the invariants (csrc/kernels.cuh mlp_seed,
csrc/mlp.cuh mlp_invariants):
  U = u_E/tau, D = u_rho/tau, S_i = u_i/tau, B^i = u_B/tau, E^i = u_E^i/tau
  (1/sqrt(-g) = 1/tau)
  f = (log U, D/U, S^2/U^2, B^2/U, (S.B)^2/U^3, E^2/U), target = (v^2, p/U),
with E = 0 for ideal RMHD and B = E = 0 for viscous hydro (U, S then hold
the viscous stresses' share as well; the seed's v^2 and p/U are the
fluid's).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import initial as I
from . import params as P
from .lib import F, Evolve, load

NW = 13058  # ECHO_MLP_NWEIGHTS
NNORM = 16  # ECHO_MLP_NNORM
NIN = 6  # ECHO_MLP_NIN


def invariants_targets(u: np.ndarray, v: np.ndarray, t: float, cfg):
    """Invariants X (n x 6) and targets T (n x 2) of every cell of a state of
    a run of `cfg` (ideal RMHD: E^2/U = 0; resistive: E in u[8:11]; viscous
    hydro: B = E = 0)."""
    nv = cfg.nv
    uu = u.reshape(nv, -1) / t
    vv = v.reshape(nv, -1)
    g3 = t * t
    D, sx, sy, sz, E = uu[0], uu[1], uu[2], uu[3], uu[4]
    zero = np.zeros_like(E)
    if cfg.mhd:
        bx, by, bz = uu[5], uu[6], uu[7]
        B2 = bx * bx + by * by + bz * bz * g3
        SB = sx * bx + sy * by + sz * bz
    else:
        B2, SB = zero, zero
    SS2 = sx * sx + sy * sy + sz * sz / g3
    if cfg.mhd == 2:
        E2 = uu[8] ** 2 + uu[9] ** 2 + g3 * uu[10] ** 2
    else:
        E2 = zero
    X = np.stack([np.log(E), D / E, SS2 / E**2, B2 / E, SB * SB / E**3, E2 / E], 1)
    x2 = vv[1] ** 2 + vv[2] ** 2 + g3 * vv[3] ** 2
    T = np.stack([x2, vv[4] / E], 1)
    return X.astype(np.float32), T.astype(np.float32)


def _magnetised(cfg, tab, peak_scale: float, mag: float, seed: int, flow: float = 0.0):
    """Primitives of the workload with the energy density scaled and the
    field set to magnetisation B^2/(2e) = mag at the centre (the workload's
    own: 0.1 ideal, 0.3 resistive); resistive runs also get a smooth flow
    of amplitude `flow` and 0.7 times the ideal E = -v x B."""
    if cfg.mhd == 2:
        v = I.resistive_flow(cfg, tab, amp=flow, ideal=0.0).reshape(cfg.nv, -1).copy()
    else:
        v = I.primitives(cfg, tab, seed=seed).reshape(cfg.nv, -1).copy()
    e_floor = cfg.enezero
    p = v[4]
    # rescale pressure through e: e -> e_floor + s (e - e_floor)
    e = np.interp(p, tab[:, 2], tab[:, 1])
    e2 = e_floor + peak_scale * (e - e_floor)
    v[4] = I.table_pressure(tab, e2)
    v[5:8] *= math.sqrt(mag / (0.3 if cfg.mhd == 2 else 0.1) * peak_scale)
    if cfg.mhd == 2:
        v = I.with_ideal_e(cfg, v.reshape(-1), 0.7).reshape(cfg.nv, -1)
    return v.reshape(-1)


def _scaled(cfg, tab, peak_scale: float, b: float, seed: int):
    """Primitives of the viscous workload (MC Glauber at impact parameter b)
    with the energy density scaled as in _magnetised."""
    v = I.primitives(cfg, tab, seed=seed, b=b).reshape(cfg.nv, -1).copy()
    e = np.interp(v[4], tab[:, 2], tab[:, 1])
    v[4] = I.table_pressure(tab, cfg.enezero + peak_scale * (e - cfg.enezero))
    return v.reshape(-1)


def generate_pairs(n_target: int = 1_000_000, grid: int | None = None, steps: int = 12, every: int = 3,
                   rng_seed: int = 5, exact: bool = False, resistive: bool = False, viscous: bool = False):
    """Run the GPU solver on the RMHD workload (the full 97x97x81 grid, or a
    grid^3-sized version with the same spacing, EoS and scheme) at several
    energy scales and magnetisations and collect (invariants, targets)
    pairs.  The full grid covers the outer, dilute and strongly magnetised
    region a central sub-grid never reaches.  resistive: the resistive
    workload instead (193x193x129 over the same extent at half the
    resolution, or grid^3 at full resolution), at rest and with smooth flows
    of amplitude 0.1 and 0.3 carrying 0.7 of the ideal E.  viscous: the
    2+1D viscous workload (201x201, or grid^2), MC-Glauber events at 3
    energy scales x impact parameters 0, 5 and 10 fm."""
    rng = np.random.default_rng(rng_seed)
    tab = I.eos_table_loaded()
    if resistive:
        c4 = P.config4()
        if grid is None:
            base = c4.replace(nx=97, ny=97, nz=65, name=c4.name + "-half")
        else:
            base = P.small(c4, grid, nz=max(8, int(grid * 0.67)))
        variants = [(s, m, f) for s in (0.3, 1.0, 3.0) for m in (0.1, 0.3) for f in (0.0, 0.1, 0.3)]
    elif viscous:
        base = P.config2() if grid is None else P.small(P.config2(), grid)
        variants = [(s, b, 0.0) for s in (0.3, 1.0, 3.0) for b in (0.0, 5.0, 10.0)]
    else:
        base = P.config1() if grid is None else P.small(P.config1(), grid, nz=max(8, int(grid * 0.84)))
        base = base.replace(algo_solver=P.C2P_NEWTON)
        variants = [(s, m, 0.0) for s in (0.3, 1.0, 3.0) for m in (0.03, 0.1, 0.3)]
    przero = float(I.table_pressure(tab, np.array([base.enezero]))[0])
    Xs, Ts = [], []
    per = max(1, n_target // (len(variants) * (steps // every)))
    for k, (scale, mag, flow) in enumerate(variants):
        ev = Evolve(base.to_c(przero=przero), tab, exact=exact)
        if viscous:
            v0 = _scaled(base, tab, scale, mag, seed=k)
        else:
            v0 = _magnetised(base, tab, scale, mag, seed=k, flow=flow)
        ev.upload(v0, None, base.tstart)
        for s in range(1, steps + 1):
            ev.run(1)
            if s % every == 0:
                ev.sync()
                st = ev.stats()
                if st.errcode:
                    break
                v, u = ev.download()
                # the step's last inversion used the metric of the step's start
                X, T = invariants_targets(u, v, st.t - st.dt, base)
                ok = np.isfinite(X).all(1) & np.isfinite(T).all(1)
                idx = np.nonzero(ok)[0]
                take = rng.choice(idx, size=min(per, len(idx)), replace=False)
                Xs.append(X[take])
                Ts.append(T[take])
        ev.close()
    X = np.concatenate(Xs)
    T = np.concatenate(Ts)
    return X, T


def generate_event_pairs(es, tab, przero: float, smooth_pressure: float, n_target: int = 300_000,
                         every_event: int = 32, samples: int = 8, rng_seed: int = 6, sources=None):
    """Pairs from the batched event-by-event workload: every `every_event`-th
    event of the EventSet `es` run alone (single grid, its own EoS table,
    grid and end time) from its initial state to es.tmax, sampled at
    `samples` times spread over the run, so that the dilute late stages the
    batch reaches are in the training set."""
    from . import events as EV

    rng = np.random.default_rng(rng_seed)
    picks = list(range(0, es.nev, every_event))
    v0 = EV.event_primitives(EV.EventSet(cfg=es.cfg, b=es.b[picks], n=es.n[picks], dx=es.dx, tmax=es.tmax), tab,
                             sources=None if sources is None else [sources[e] for e in picks])
    per = max(1, n_target // (len(picks) * samples))
    Xs, Ts = [], []
    for k, e in enumerate(picks):
        cfg = es.event_config(e)
        ev = Evolve(cfg.to_c(przero=przero, smooth_pressure=smooth_pressure), tab)
        ev.upload(v0[k], None, cfg.tstart)
        ev.set_tout(es.tmax)
        span = es.tmax - cfg.tstart
        for j in range(1, samples + 1):
            target = cfg.tstart + span * j / samples
            for _ in range(20000):
                st = ev.stats()
                if st.errcode or st.t >= target - 1e-12:
                    break
                ev.run(4)
                ev.sync()
            if st.errcode:
                break
            v, u = ev.download()
            X, T = invariants_targets(u, v, st.t - st.dt, cfg)
            ok = np.nonzero(np.isfinite(X).all(1) & np.isfinite(T).all(1))[0]
            take = rng.choice(ok, size=min(per, len(ok)), replace=False)
            Xs.append(X[take])
            Ts.append(T[take])
        ev.close()
    return np.concatenate(Xs), np.concatenate(Ts)


def train(X: np.ndarray, T: np.ndarray, steps: int = 3000, batch: int = 4096, lr: float = 3e-3,
          seed: int = 1, report_every: int = 100):
    """Train the seed network on the GPU; returns (weights, norm, losses)."""
    L = load(False)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    w = np.zeros(NW, dtype=np.float32)
    norm = np.zeros(NNORM, dtype=np.float32)
    losses = np.zeros(max(1, steps // report_every), dtype=np.float32)
    rc = L.echo_gpu_mlp_train(X.ctypes.data_as(F), T.ctypes.data_as(F), len(X), steps, batch, lr, seed,
                              w.ctypes.data_as(F), norm.ctypes.data_as(F), losses.ctypes.data_as(F),
                              report_every)
    if rc:
        raise RuntimeError(f"echo_gpu_mlp_train status {rc}")
    return w, norm, losses


def infer(weights, norm, X):
    """Tensor-core inference of the seed (BF16 operands, FP32 accumulation)."""
    L = load(False)
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.zeros((len(X), 2), dtype=np.float32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    nm = np.ascontiguousarray(norm, dtype=np.float32)
    rc = L.echo_gpu_mlp_infer(w.ctypes.data_as(F), nm.ctypes.data_as(F), X.ctypes.data_as(F), len(X),
                              out.ctypes.data_as(F))
    if rc:
        raise RuntimeError(f"echo_gpu_mlp_infer status {rc}")
    return out


def gradient(weights, Xs, Ts):
    """Loss and gradient from the GPU training kernels on standardised rows."""
    L = load(False)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    Xs = np.ascontiguousarray(Xs, dtype=np.float32)
    Ts = np.ascontiguousarray(Ts, dtype=np.float32)
    g = np.zeros(NW, dtype=np.float32)
    loss = ctypes.c_float(0)
    rc = L.echo_gpu_mlp_grad(w.ctypes.data_as(F), Xs.ctypes.data_as(F), Ts.ctypes.data_as(F), len(Xs),
                             ctypes.pointer(loss), g.ctypes.data_as(F))
    if rc:
        raise RuntimeError(f"echo_gpu_mlp_grad status {rc}")
    return float(loss.value), g
