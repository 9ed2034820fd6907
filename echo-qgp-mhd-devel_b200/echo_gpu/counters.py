"""Roofline counters of the step kernels: the FP64 operations and DRAM bytes
of one launch of each kernel class, as ncu measured them, tied to the
sources they were measured on.

    python -m echo_gpu.counters <report.ncu-rep | raw.csv> <out.json> --workload NAME

reads the raw page of an ncu report, or that page exported beforehand with
``ncu -i report --page raw --csv`` (metrics dfma/dadd/dmul thread
instructions, dram bytes, duration) and writes one record per kernel class
(faces_x/y/z, update_c2p, stage_fused) with the build hash of the CUDA
sources; ``load`` returns the records and whether they belong to the sources
in this tree.  bench.py reads the file to report FP64 FLOPs and measured
traffic beside its own event-timed durations.
"""
from __future__ import annotations

import argparse
import csv
import hashlib
import io
import json
import os
import subprocess

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ROOT = os.path.dirname(PKG)


def build_hash() -> str:
    """SHA-256 (16 hex digits) of the CUDA sources and the C-ABI header."""
    h = hashlib.sha256()
    csrc = os.path.join(PKG, "csrc")
    for f in sorted(os.listdir(csrc)):
        if f.endswith((".cu", ".cuh")):
            with open(os.path.join(csrc, f), "rb") as fh:
                h.update(f.encode() + b"\0" + fh.read())
    with open(os.path.join(ROOT, "include", "echo_gpu.h"), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()[:16]


def kernel_class(name: str) -> str | None:
    if name.startswith("void faces_kernel<"):
        d = name.split("<")[1].split(",")[1].strip()
        return "faces_" + "xyz"[int(d)]
    if name.startswith("void update_kernel<"):
        return "update_c2p"
    if name.startswith("void stage_kernel<"):
        return "stage_fused"
    return None


def parse(report: str) -> dict:
    if report.endswith(".csv"):
        with open(report) as fh:
            out = fh.read()
    else:
        out = subprocess.run(["ncu", "-i", report, "--page", "raw", "--csv"], check=True, capture_output=True,
                             text=True).stdout
    rows = list(csv.reader(io.StringIO(out)))
    hdr = rows[0]
    units = dict(zip(hdr, rows[1]))
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "nsecond": 1e-3, "usecond": 1.0,
             "msecond": 1e3, "second": 1e6}
    recs: dict[str, list[dict]] = {}
    for r in rows[2:]:
        d = dict(zip(hdr, r))
        cls = kernel_class(d.get("Kernel Name", ""))
        if cls is None:
            continue

        def f(k):
            v = d.get(k, "")
            if v in ("", "n/a"):
                return 0.0
            return float(v.replace(",", "")) * scale.get(units.get(k, ""), 1.0)

        dfma = f("sm__sass_thread_inst_executed_op_dfma_pred_on.sum")
        dadd = f("sm__sass_thread_inst_executed_op_dadd_pred_on.sum")
        dmul = f("sm__sass_thread_inst_executed_op_dmul_pred_on.sum")
        recs.setdefault(cls, []).append({
            "fp64_flop": 2 * dfma + dadd + dmul,
            "fp64_thread_inst": f("sm__thread_inst_executed_pipe_fp64_pred_on.sum"),
            "dram_bytes": f("dram__bytes_read.sum") + f("dram__bytes_write.sum"),
            "ncu_us": f("gpu__time_duration.sum"),
            "fp64_pipe_pct": f("sm__pipe_fp64_cycles_active.avg.pct_of_peak_sustained_active"),
        })
    return {k: {m: sum(x[m] for x in v) / len(v) for m in v[0]} | {"launches": len(v)} for k, v in recs.items()}


def load(path: str) -> tuple[dict, bool]:
    """(records, True when they were measured on the sources in this tree)"""
    with open(path) as f:
        d = json.load(f)
    return d, d.get("build_hash") == build_hash()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("report")
    ap.add_argument("out")
    ap.add_argument("--workload", required=True)
    ap.add_argument("--command", default="")
    a = ap.parse_args()
    rec = {"build_hash": build_hash(), "workload": a.workload, "command": a.command,
           "units": "per launch (ncu, cold cache, serialised)", "kernels": parse(a.report)}
    with open(a.out, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec, indent=1))


if __name__ == "__main__":
    main()
