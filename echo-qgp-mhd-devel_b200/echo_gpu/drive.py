"""Run a named workload for a number of steps through the C-ABI.

    python -m echo_gpu.drive --config rmhd --steps 3 [--c2p newton|mlp] [--exact] [--imex] [--n N]
    python -m echo_gpu.drive --config batch --events 64 --steps 3

Used for profiling runs: it does exactly the product path (upload, the
per-step CUDA graph, stats) and nothing else.  ``--c2p mlp`` first trains
the seed network briefly on pairs from the solver; ``--config batch`` runs
evenly spaced events of the batched viscous workload, initial state
generated on the device.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import initial as I
from . import params as P
from .lib import Evolve

CONFIGS = {"hd": P.config0, "rmhd": P.config1, "visc": P.config2, "res": P.config4}


def run_batch(a) -> None:
    from . import events as EV
    from .batch import Batch, event_grid

    es0 = EV.batched_viscous()
    sel = np.arange(0, es0.nev, max(1, es0.nev // max(1, a.events)))[: a.events]
    es = EV.EventSet(cfg=es0.cfg, b=es0.b[sel], n=es0.n[sel], dx=es0.dx, tmax=es0.tmax)
    tab = EV.batched_eos_table()
    pc = es.cfg.to_c(przero=float(I.table_pressure(tab, np.array([es.cfg.enezero]))[0]),
                     smooth_pressure=I.table_temperature_to_pressure(tab, es.cfg.smooth_temp))
    b = Batch(pc, tab, [event_grid(*es.grid(e)) for e in range(es.nev)], exact=a.exact)
    b.glauber(EV.event_sources(es), es.cfg.tstart, es.tmax)
    t0 = time.perf_counter()
    b.run(a.steps)
    b.sync()
    el = time.perf_counter() - t0
    st = b.status()
    bad = [s["errcode"] for s in st if s["errcode"]]
    print(f"batch of {es.nev} events ({int(es.cells.sum())} cells): {a.steps} steps in {el*1e3:.1f} ms wall, "
          f"{b.cell_updates()} cell-updates, crashed events {len(bad)}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="rmhd", choices=list(CONFIGS) + ["batch"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--c2p", default="brent", choices=["brent", "newton", "mlp"])
    ap.add_argument("--exact", action="store_true")
    ap.add_argument("--imex", action="store_true", help="viscous: Israel-Stewart relaxation implicit per stage")
    ap.add_argument("--n", type=int, default=0, help="cells per side of a smaller grid (0 = full size)")
    ap.add_argument("--events", type=int, default=64, help="events of the batched workload")
    ap.add_argument("--pairs", type=int, default=100_000, help="training pairs for --c2p mlp")
    ap.add_argument("--train-steps", type=int, default=500)
    ap.add_argument("--stage", default="auto", choices=["auto", "fused", "sweeps"],
                    help="fused stage kernel or the sweep kernels (auto: the library's default)")
    ap.add_argument("--tile", default="", help="fused stage tile tx,ty,zseg (0 = chosen for the grid)")
    ap.add_argument("--faces", type=int, default=-1, choices=[-1, 0, 8, 16],
                    help="product build face sweeps: 0 one thread per face, 8/16 cell-centred segments "
                         "(-1: the library's default)")
    a = ap.parse_args()
    if a.config == "batch":
        run_batch(a)
        return
    cfg = CONFIGS[a.config]()
    if a.n:
        cfg = P.small(cfg, a.n, nz=a.n if cfg.nz > 1 else None)
    if a.c2p == "newton":
        cfg = cfg.replace(algo_solver=P.C2P_NEWTON)
    if a.c2p == "mlp":
        cfg = cfg.replace(algo_solver=P.C2P_MLP)
    if a.imex:
        cfg = cfg.replace(imex=1)
    tab = I.eos_table_loaded() if cfg.eqstate == P.EOS_TABLE else None
    przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0]) if tab is not None else cfg.enezero / 3
    sp = I.table_temperature_to_pressure(tab, cfg.smooth_temp) if (tab is not None and cfg.viscosity) else 0.0
    ev = Evolve(cfg.to_c(przero=przero, smooth_pressure=sp), tab, exact=a.exact)
    if a.c2p == "mlp":
        from . import seed as S

        # pairs of the run's own equation set
        X, T = S.generate_pairs(n_target=a.pairs, resistive=cfg.mhd == 2, viscous=bool(cfg.viscosity))
        w, norm, _ = S.train(X, T, steps=a.train_steps)
        ev.set_seed_network(w, norm)
    if a.stage != "auto" or a.tile:
        tx, ty, zs = (int(x) for x in a.tile.split(",")) if a.tile else (0, 0, 0)
        info = ev.set_stage(a.stage != "sweeps", tx, ty, zs)
        print(f"stage: {info}")
    if a.faces >= 0:
        ev.set_faces(a.faces)
    ev.upload(I.primitives(cfg, tab), None, cfg.tstart)
    t0 = time.perf_counter()
    ev.run(a.steps)
    ev.sync()
    el = time.perf_counter() - t0
    st = ev.stats()
    print(f"{cfg.name}: {a.steps} steps in {el*1e3:.1f} ms wall, t={st.t:.6f}, errcode={st.errcode}, "
          f"c2p iters/cell (last stage)={st.c2p_iters/cfg.ncell:.2f}")
    if st.errcode:
        raise SystemExit(1)


if __name__ == "__main__":
    main()
