"""Output files in the reference's layout (out_vars, out.f90:232-591).

The bytes of one outNNNN.dat come from Evolve.out_vars (assembled on the
device): t, then every selected field over the grid in Fortran order (x
fastest), in double or single precision.  This module names the fields and
their ECHO_OUT_* bits (include/echo_gpu.h), writes the files where the
reference writes them (outrNNNN/outNNNN.dat, with the "(I5,f16.9)" line of
time.dat, out.f90:257-283) and reads them back the way the reference's
tools read them (stream-binary, t first).
"""
from __future__ import annotations

import os

import numpy as np

# the out_sel flags (common.f90:122-151) in the order out_vars writes them
FIELDS = ["density", "vx", "vy", "vz", "pressure", "energy_density", "temperature", "entropy_density", "bulk",
          "pitt", "pitx", "pity", "pitz", "pixy", "pixz", "piyz", "pixx", "piyy", "pizz", "v0",
          "bx", "by", "bz", "ex", "ey", "ez", "glm"]
BIT = {name: 1 << k for k, name in enumerate(FIELDS)}
# their defaults (common.f90:724-805)
DEFAULT = sum(BIT[n] for n in ("density", "vx", "vy", "vz", "pressure", "energy_density",
                               "bx", "by", "bz", "ex", "ey", "ez"))


def mask(*names: str) -> int:
    return sum(BIT[n] for n in names)


def written(cfg, sel: int) -> list[str]:
    """The fields a run of `cfg` writes for `sel`, in file order: viscous
    fields only for viscous runs, B and E only for MHD runs, psi only with
    divclean as well."""
    out = []
    for k, name in enumerate(FIELDS):
        if not sel >> k & 1:
            continue
        if 8 <= k <= 18 and not cfg.viscosity:
            continue
        if 20 <= k <= 25 and not cfg.mhd:
            continue
        if k == 26 and not (cfg.mhd and cfg.divclean):
            continue
        out.append(name)
    return out


def file_name(iout: int) -> str:
    return f"out{iout:04d}.dat"


def run_dir(id_of_the_run: int) -> str:
    return f"outr{id_of_the_run:04d}"


def write(root: str, id_of_the_run: int, iout: int, blob: bytes, t: float, append_time: bool) -> str:
    """Write one output as the reference does: the blob to
    outrNNNN/outNNNN.dat and "iout t" to outrNNNN/time.dat (replaced on the
    first output of a run, appended after)."""
    d = os.path.join(root, run_dir(id_of_the_run))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, file_name(iout))
    with open(path, "wb") as f:
        f.write(blob)
    with open(os.path.join(d, "time.dat"), "a" if append_time else "w") as f:
        f.write(f"{iout:5d}{t:16.9f}\n")
    return path


def read(data: bytes, cfg, sel: int, precision: int = 8):
    """(t, {field: array (nz, ny, nx)}) of one outNNNN.dat."""
    dt = np.float64 if precision == 8 else np.float32
    arr = np.frombuffer(data, dtype=dt)
    names = written(cfg, sel)
    n = cfg.nx * cfg.ny * cfg.nz
    if arr.size != 1 + n * len(names):
        raise ValueError(f"{arr.size} values for {len(names)} fields of {n} cells")
    shape = (cfg.nz, cfg.ny, cfg.nx)
    return float(arr[0]), {name: arr[1 + i * n:1 + (i + 1) * n].reshape(shape) for i, name in enumerate(names)}


def write_dump(root: str, id_of_the_run: int, blob: bytes) -> str:
    """Write the bytes of echo_gpu_dump to outrNNNN/dump.dat (out_dump,
    out.f90:1349-1381); returns the path."""
    d = os.path.join(root, run_dir(id_of_the_run))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, "dump.dat")
    with open(path, "wb") as f:
        f.write(blob)
    return path


def read_dump(data: bytes, cfg) -> dict:
    """Parse dump.dat as out_restart reads it (out.f90:1422-1432):
    iout, t, timeold, timeinterval, vall, uall, vallold, uallold (the fields
    krh..kvold_end: 8 with MHD, else 5), g_cov_3_old."""
    nc = cfg.nx * cfg.ny * cfg.nz
    kold = 8 if cfg.mhd else 5
    iout = int(np.frombuffer(data, dtype="<i4", count=1)[0])
    rest = np.frombuffer(data, dtype="<f8", offset=4)
    want = 3 + nc * (2 * cfg.nv + 2 * kold) + 1
    if rest.size != want:
        raise ValueError(f"dump.dat holds {rest.size} doubles after iout, a run of this shape writes {want}")
    o = 3
    out = {"iout": iout, "t": float(rest[0]), "timeold": float(rest[1]), "timeinterval": float(rest[2])}
    for name, n in (("vall", cfg.nv), ("uall", cfg.nv), ("vallold", kold), ("uallold", kold)):
        out[name] = rest[o:o + n * nc].copy()
        o += n * nc
    out["g_cov_3_old"] = float(rest[o])
    return out
