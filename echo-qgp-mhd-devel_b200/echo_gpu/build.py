"""Build of the CUDA library (in-tree, sm_100a).

Two variants are built from the same sources:

* ``libechogpu.so``        -- the product build: FP64 with fused
  multiply-add contraction (``--fmad=true``), used by the benchmark;
* ``libechogpu_exact.so``  -- the parity build: ``--fmad=false``, so every
  multiply and add rounds separately exactly as the CPU restatement of the
  reference does; results agree with it bit for bit except where a
  transcendental (exp, pow) differs in the last place between libm and CUDA.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
LIBDIR = os.path.join(ROOT, "lib")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]

VARIANTS = {
    "libechogpu.so": ["--fmad=true"],
    "libechogpu_exact.so": ["--fmad=false", "-DECHO_EXACT"],
}

# one translation unit per equation set, compiled in parallel
SOURCES = ["echo_gpu.cu", "unit_tests.cu", "kind_hd.cu", "kind_visc.cu", "kind_mhd.cu", "kind_mhdglm.cu", "kind_res.cu",
           "noalloc.cu", "mlp_train.cu", "batch.cu", "hyper.cu", "output.cu", "glauber.cu"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(ROOT), "include", "echo_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, variants=None) -> list[str]:
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    out, jobs, links = [], [], []
    for name, flags in VARIANTS.items():
        if variants and name not in variants:
            continue
        target = os.path.join(LIBDIR, name)
        out.append(target)
        if not force and not _stale(target):
            continue
        objs = []
        for src in SOURCES:
            obj = os.path.join(objdir, name.replace(".so", "") + "_" + src.replace(".cu", ".o"))
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", "-o", obj, os.path.join(CSRC, src)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
            objs.append(obj)
        links.append([nvcc(), *ARCH, "-shared", "-o", target, *objs])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    for cmd in links:
        run(cmd)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
