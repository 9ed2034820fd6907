"""Run a named workload for a number of steps through the C-ABI.

    python -m echo_gpu.drive --config rmhd --steps 3 [--c2p newton] [--exact]

Used for profiling runs: it does exactly the product path (upload, the
per-step CUDA graph, stats) and nothing else.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import initial as I
from . import params as P
from .lib import Evolve

CONFIGS = {"hd": P.config0, "rmhd": P.config1, "visc": P.config2}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="rmhd", choices=list(CONFIGS))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--c2p", default="brent", choices=["brent", "newton"])
    ap.add_argument("--exact", action="store_true")
    ap.add_argument("--n", type=int, default=0, help="cells per side of a smaller grid (0 = full size)")
    a = ap.parse_args()
    cfg = CONFIGS[a.config]()
    if a.n:
        cfg = P.small(cfg, a.n, nz=a.n if cfg.nz > 1 else None)
    if a.c2p == "newton":
        cfg = cfg.replace(algo_solver=P.C2P_NEWTON)
    tab = I.eos_table_loaded() if cfg.eqstate == P.EOS_TABLE else None
    przero = float(I.table_pressure(tab, np.array([cfg.enezero]))[0]) if tab is not None else cfg.enezero / 3
    sp = I.table_temperature_to_pressure(tab, cfg.smooth_temp) if (tab is not None and cfg.viscosity) else 0.0
    ev = Evolve(cfg.to_c(przero=przero, smooth_pressure=sp), tab, exact=a.exact)
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
