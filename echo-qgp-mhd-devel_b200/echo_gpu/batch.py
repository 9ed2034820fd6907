"""Batched event-by-event runs behind the C-ABI (echo_batch_* in
include/echo_gpu.h).

The reference's Monte Carlo mode runs events one after another through
the whole time loop (events loop, echo.f90:113-308).  ``Batch`` advances
many events, each on its own grid, together on one GPU; every event keeps
its own t, dt, stop test (t >= tmax, echo.f90:187) and crash state (a
crashed event is abandoned, echo.f90:206-209).  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .lib import LL, EchoEventGrid, EchoEventStatus, F, I, P, _dp, load
from .params import EchoParams

LIVE, DONE, CRASHED, COOLED = 0, 1, 2, 3
SLOTS = ("faces_x", "faces_y", "faces_z", "update", "smooth")
KERNEL_CLASSES = ("faces_x", "faces_y", "faces_z", "scalars", "update_c2p", "repair_smooth", "end_step",
                  "stage_fused")


def event_grid(nx: int, ny: int, nz: int, x1: float, x2: float, y1: float, y2: float,
               z1: float = -0.5, z2: float = 0.5) -> EchoEventGrid:
    return EchoEventGrid(nx, ny, nz, x1, x2, y1, y2, z1, z2)


class Batch:
    """Device-resident state of many events and their batched step."""

    def __init__(self, params: EchoParams, eos_table, grids, exact: bool = False):
        self.lib = load(exact)
        self.params = params
        self._tab = None if eos_table is None else np.ascontiguousarray(eos_table, dtype=np.float64)
        n = 0 if self._tab is None else len(self._tab)
        self.nev = len(grids)
        self._grids = (EchoEventGrid * self.nev)(*grids)
        h = P()
        rc = self.lib.echo_batch_init(ctypes.byref(params), _dp(self._tab), n, self.nev, self._grids,
                                      ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"echo_batch_init failed with status {rc}")
        self.h = h
        self.nv = self.lib.echo_batch_nv(h)
        off = np.zeros(self.nev + 1, dtype=np.int64)
        self._check(self.lib.echo_batch_offsets(h, off.ctypes.data_as(LL)), "offsets")
        self.offsets = off
        self.ncell = int(off[-1])

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"echo_batch_{what} failed with status {rc}")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.echo_batch_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- arena <-> per-event arrays ------------------------------------------
    def pack(self, per_event) -> np.ndarray:
        """Concatenate per-event flat arrays (nv * ncell_e, Fortran order)."""
        out = np.concatenate([np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in per_event])
        if out.size != self.nv * self.ncell:
            raise ValueError("per-event arrays do not match the event grids")
        return out

    def split(self, arena: np.ndarray) -> list[np.ndarray]:
        o = self.offsets * self.nv
        return [arena[o[e]:o[e + 1]] for e in range(self.nev)]

    # -- state -----------------------------------------------------------------
    def upload(self, v, u=None, t: float = 0.4, tmax: float = 10.0) -> None:
        v = self.pack(v) if isinstance(v, (list, tuple)) else np.ascontiguousarray(v, dtype=np.float64)
        if u is not None:
            u = self.pack(u) if isinstance(u, (list, tuple)) else np.ascontiguousarray(u, dtype=np.float64)
        self._v_keep = v
        self._check(self.lib.echo_batch_upload(self.h, _dp(v), _dp(u), t, tmax), "upload")

    def upload_device(self, v_ptr: int, u_ptr: int | None, t: float, tmax: float) -> None:
        self._check(self.lib.echo_batch_upload_device(self.h, v_ptr, u_ptr, t, tmax), "upload_device")

    def glauber(self, sources, t: float = 0.4, tmax: float = 10.0, sigma: float = 0.5, peak: float = 30.0,
                ah: float = 0.15) -> None:
        """Initial state of every event from its Monte Carlo Glauber sources
        (``sources[e] = (participants (n, 2), collisions (m, 2))``), smeared
        and converted to primitives on the device."""
        rows, off = [], [0]
        for parts, colls in sources:
            w = np.concatenate([np.full(len(parts), 1.0 - ah), np.full(len(colls), ah)])
            xy = np.concatenate([np.reshape(parts, (-1, 2)), np.reshape(colls, (-1, 2))])
            rows.append(np.column_stack([xy, w]))
            off.append(off[-1] + len(w))
        src = np.ascontiguousarray(np.concatenate(rows) if rows else np.zeros((0, 3)), dtype=np.float64)
        o = np.ascontiguousarray(off, dtype=np.int64)
        self._check(self.lib.echo_batch_glauber(self.h, _dp(src), o.ctypes.data_as(LL), sigma, peak, t, tmax),
                    "glauber")

    def download(self):
        v = np.empty(self.nv * self.ncell)
        u = np.empty(self.nv * self.ncell)
        self._check(self.lib.echo_batch_download(self.h, _dp(v), _dp(u)), "download")
        return v, u

    def set_seed_network(self, weights, norm) -> None:
        """Load a trained con2prim seed (echo_gpu.seed.train); needed before
        running with algo_solver = C2P_MLP."""
        w = np.ascontiguousarray(weights, dtype=np.float32)
        n = np.ascontiguousarray(norm, dtype=np.float32)
        self._check(self.lib.echo_batch_mlp_set(self.h, w.ctypes.data_as(F), n.ctypes.data_as(F)), "mlp_set")

    # -- stepping --------------------------------------------------------------
    def run(self, nsteps: int) -> None:
        self._check(self.lib.echo_batch_run(self.h, nsteps), "run")

    def live(self) -> int:
        n = ctypes.c_int(0)
        self._check(self.lib.echo_batch_live(self.h, ctypes.byref(n)), "live")
        return n.value

    def run_to_end(self, chunk: int = 8, max_steps: int = 100000) -> int:
        """Step until every event has finished or crashed; returns the number
        of batched steps launched."""
        done = 0
        while done < max_steps:
            self.run(chunk)
            done += chunk
            if self.live() == 0:
                break
        return done

    def sync(self) -> None:
        self._check(self.lib.echo_batch_sync(self.h), "sync")

    def status(self) -> list[dict]:
        st = (EchoEventStatus * self.nev)()
        self._check(self.lib.echo_batch_status(self.h, st), "status")
        return [dict(t=s.t, dt=s.dt, steps=s.steps, state=s.state, errcode=s.errcode, err_cell=s.err_cell,
                     c2p_iters=s.c2p_iters, repairs=s.repairs, seed_fallbacks=s.seed_fallbacks) for s in st]

    def cell_updates(self) -> int:
        """Cells times completed steps, summed over the events."""
        ncell = np.diff(self.offsets)
        steps = np.array([s["steps"] for s in self.status()], dtype=np.int64)
        return int((ncell * steps).sum())

    def stream_handle(self) -> int:
        s = P()
        self._check(self.lib.echo_batch_stream(self.h, ctypes.byref(s)), "stream")
        return s.value or 0

    def set_stop(self, freeze_type: int = 1, temp_end: float = 0.0) -> None:
        """Per-event check_temp stop criterion (TEMP_END; 0 turns it off)."""
        self._check(self.lib.echo_batch_set_stop(self.h, freeze_type, temp_end), "set_stop")

    # -- launch shapes ---------------------------------------------------------
    def set_schedule(self, ctas=None, order=None) -> None:
        c = None if ctas is None else np.ascontiguousarray(ctas, dtype=np.int32)
        o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
        self._check(self.lib.echo_batch_set_schedule(self.h, None if c is None else c.ctypes.data_as(I),
                                                     None if o is None else o.ctypes.data_as(I)), "set_schedule")

    def get_schedule(self) -> dict:
        c = np.zeros(len(SLOTS), dtype=np.int32)
        self._check(self.lib.echo_batch_get_schedule(self.h, c.ctypes.data_as(I)), "get_schedule")
        return dict(zip(SLOTS, c.tolist()))

    def autotune(self, reps: int = 3) -> dict:
        ms = np.zeros(len(SLOTS))
        self._check(self.lib.echo_batch_autotune(self.h, reps, _dp(ms)), "autotune")
        return dict(zip(SLOTS, ms.tolist()))

    def autotune_report(self) -> list[dict]:
        """Every candidate the last autotune timed."""
        n = ctypes.c_int(0)
        self._check(self.lib.echo_batch_autotune_report(self.h, None, 0, ctypes.byref(n)), "autotune_report")
        rows = np.zeros(4 * max(n.value, 1))
        self._check(self.lib.echo_batch_autotune_report(self.h, _dp(rows), n.value, ctypes.byref(n)),
                    "autotune_report")
        out = []
        for i in range(n.value):
            what, shape, ctas, ms = rows[4 * i:4 * i + 4]
            if int(what) < len(SLOTS):
                out.append({"slot": SLOTS[int(what)], "tile": int(shape), "ctas": int(ctas), "ms": float(ms)})
            else:
                out.append({"slot": "stage", "mode": "cooperative" if int(shape) else "phased",
                            "ctas": int(ctas), "ms": float(ms)})
        return out

    def set_tiles(self, faces: int = 128, cells: int = 128):
        t = np.array([faces, faces, faces, cells], dtype=np.int32)
        self._check(self.lib.echo_batch_set_tiles(self.h, t.ctypes.data_as(I)), "set_tiles")

    def set_mode(self, mode: int, grid: int = 0):
        """0: one launch per phase; 1: one cooperative launch per stage."""
        self._check(self.lib.echo_batch_set_mode(self.h, mode, grid), "set_mode")

    def tuning(self) -> dict:
        out = np.zeros(7, dtype=np.int32)
        self._check(self.lib.echo_batch_get_tuning(self.h, out.ctypes.data_as(I)), "get_tuning")
        return {"tiles": out[:4].tolist(), "mode": "cooperative" if out[4] else "phased",
                "coop_grid": int(out[5]), "graphs": bool(out[6])}

    def profile_step(self):
        ms = np.zeros(len(KERNEL_CLASSES))
        n = np.zeros(len(KERNEL_CLASSES), dtype=np.int32)
        self._check(self.lib.echo_batch_profile_step(self.h, _dp(ms), n.ctypes.data_as(I)), "profile_step")
        return dict(zip(KERNEL_CLASSES, ms.tolist())), dict(zip(KERNEL_CLASSES, n.tolist()))
