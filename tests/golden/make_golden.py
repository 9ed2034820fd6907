"""Regenerate the golden fixtures: the CPU oracle run on the small parity
workloads (tests/helpers.CASES) for a fixed number of steps.

    python tests/golden/make_golden.py [name ...]

These vectors pin the oracle against regressions; they are produced by the
oracle itself because the reference (Fortran) cannot be built here.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "echo-qgp-mhd-devel_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import pyoracle as O  # noqa: E402
from helpers import GOLDEN_CASES, golden_setup  # noqa: E402

if __name__ == "__main__":
    only = sys.argv[1:] or list(GOLDEN_CASES)
    for name in only:
        cfg, pc, tab, v0, steps = golden_setup(name)
        o = O.Oracle(pc, tab)
        o.set_state(v0, None, cfg.tstart)
        for _ in range(steps):
            o.step()
        v, u = o.state()
        meta = json.dumps({"steps": steps, "t": o.t, "config": cfg.name})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), v0=v0, v=v, u=u, meta=meta)
        print(name, steps, o.t)
