"""ctypes binding of libechogpu.so and the host-side mirror of the
reference's step interface.

``Evolve`` mirrors the Fortran module `evolve` (evolve.f90): evolve_main(irk)
returns dt and raises on a crashed stage exactly where the reference sets
run_crashed; step() is one iteration of the time loop of echo.f90:185-262.
There is no CPU fallback: constructing an ``Evolve`` without the CUDA
library or without a GPU raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import EchoParams

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(_ROOT, "lib")
_libs: dict[str, ctypes.CDLL] = {}

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)
F = ctypes.POINTER(ctypes.c_float)
P = ctypes.c_void_p


class EchoStats(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double), ("t", ctypes.c_double), ("glm_ch", ctypes.c_double),
        ("c2p_iters", ctypes.c_longlong), ("c2p_cells", ctypes.c_longlong),
        ("repairs", ctypes.c_longlong), ("seed_fallbacks", ctypes.c_longlong),
        ("errcode", ctypes.c_int), ("err_cell", ctypes.c_int),
        ("bracket_fallbacks", ctypes.c_longlong),
    ]


class EchoEventGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("x1", ctypes.c_double), ("x2", ctypes.c_double), ("y1", ctypes.c_double),
                ("y2", ctypes.c_double), ("z1", ctypes.c_double), ("z2", ctypes.c_double)]


class EchoEventStatus(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("state", ctypes.c_int), ("errcode", ctypes.c_int), ("err_cell", ctypes.c_int),
                ("pad", ctypes.c_int), ("c2p_iters", ctypes.c_longlong), ("repairs", ctypes.c_longlong),
                ("seed_fallbacks", ctypes.c_longlong)]


LL = ctypes.POINTER(ctypes.c_longlong)


class EchoOpticalGlauber(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "mass_number", "radius", "delta", "roze", "sigma_in", "ah", "bimpact", "ecenter", "rhocenter",
        "dr", "dz1", "acc", "deta", "sigeta", "sqrt_s", "nucleon_mass")]


def optical_glauber_params(nucleus: str = "Au", b: float = 7.0, sigma_in_mb: float = 42.0, ah: float = 0.15,
                           ecenter: float = 1.0, rhocenter: float = 0.1, dr: float = 0.001, dz1: float = 0.001,
                           acc: float = 1e-7, deta: float = 2.0, sigeta: float = 1.5, sqrt_s: float = 200.0,
                           nucleon_mass: float = 0.938) -> EchoOpticalGlauber:
    """The GLAUBER_GEOMETRIC parameters: nucleus from nuclear_data.dat
    (projmass, radius, delta, roze), SIGMA_IN in mb (stored in fm^2,
    common.f90:2259), AH, impact parameter, ECENTER, the thickness table's
    r and z steps and accuracy (the reference's printed defaults 0.001,
    0.001, 1e-7), the eta plateau and Gaussian width and the collision's
    sqrt(s) for 3+1D."""
    A, R, a, rho0 = {"Au": (197.0, 6.38, 0.535, 0.1693), "Pb": (208.0, 6.62, 0.546, 0.1604)}[nucleus]
    return EchoOpticalGlauber(mass_number=A, radius=R, delta=a, roze=rho0, sigma_in=sigma_in_mb / 10.0, ah=ah,
                              bimpact=b, ecenter=ecenter, rhocenter=rhocenter, dr=dr, dz1=dz1, acc=acc, deta=deta,
                              sigeta=sigeta, sqrt_s=sqrt_s, nucleon_mass=nucleon_mass)

FUNCTIONS = {
    "echo_gpu_init": (ctypes.c_int, [P, D, ctypes.c_int, ctypes.POINTER(P)]),
    "echo_gpu_free": (ctypes.c_int, [P]),
    "echo_gpu_nv": (ctypes.c_int, [P]),
    "echo_gpu_upload": (ctypes.c_int, [P, D, D, ctypes.c_double]),
    "echo_gpu_download": (ctypes.c_int, [P, D, D]),
    "echo_gpu_upload_device": (ctypes.c_int, [P, P, P, ctypes.c_double]),
    "echo_gpu_download_device": (ctypes.c_int, [P, P, P]),
    "echo_gpu_set_tout": (ctypes.c_int, [P, ctypes.c_double]),
    "echo_gpu_evolve_main": (ctypes.c_int, [P, ctypes.c_int, D, I]),
    "echo_gpu_end_step": (ctypes.c_int, [P]),
    "echo_gpu_step": (ctypes.c_int, [P, D, I]),
    "echo_gpu_run": (ctypes.c_int, [P, ctypes.c_int]),
    "echo_gpu_stats": (ctypes.c_int, [P, ctypes.POINTER(EchoStats)]),
    "echo_gpu_sync": (ctypes.c_int, [P]),
    "echo_gpu_rhs": (ctypes.c_int, [P, D, D]),
    "echo_gpu_stream": (ctypes.c_int, [P, ctypes.POINTER(P)]),
    "echo_gpu_put_state": (ctypes.c_int, [P, P, P]),
    "echo_gpu_rhs_noalloc": (ctypes.c_int, [P, P, ctypes.c_int, ctypes.c_double, P, P, P, I]),
    "echo_gpu_fp64_peak": (ctypes.c_int, [D, D]),
    "echo_gpu_mlp_train": (ctypes.c_int, [F, F, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_uint, F, F, F, ctypes.c_int]),
    "echo_gpu_mlp_grad": (ctypes.c_int, [F, F, F, ctypes.c_int, F, F]),
    "echo_gpu_mlp_set": (ctypes.c_int, [P, F, F]),
    "echo_gpu_mlp_infer": (ctypes.c_int, [F, F, F, ctypes.c_int, F]),
    "echo_gpu_test_c2p_seeded": (ctypes.c_int, [P, D, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                F, F, D, D, I, I, I]),
    "echo_gpu_get_state": (ctypes.c_int, [P, P, P]),
    "echo_gpu_profile_step": (ctypes.c_int, [P, D, I]),
    "echo_gpu_set_stage": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, I]),
    "echo_gpu_set_faces": (ctypes.c_int, [P, ctypes.c_int]),
    "echo_gpu_set_sweeps": (ctypes.c_int, [P, ctypes.c_int]),
    "echo_gpu_advance_host": (ctypes.c_int, [P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int]),
    "echo_gpu_test_recon": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D]),
    "echo_gpu_test_fastdiv": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_void_p]),
    "echo_gpu_test_c2p": (ctypes.c_int, [P, D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, D, D, I, I]),
    "echo_gpu_hyp_init": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double]),
    "echo_gpu_hyp_step": (ctypes.c_int, [P, I, I]),
    "echo_gpu_hyp_get": (ctypes.c_int, [P, D]),
    "echo_gpu_checkpoint_size": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
    "echo_gpu_checkpoint": (ctypes.c_int, [P, P]),
    "echo_gpu_restart": (ctypes.c_int, [P, P]),
    "echo_gpu_keep_old": (ctypes.c_int, [P, ctypes.c_int]),
    "echo_gpu_optical_glauber": (ctypes.c_int, [P, ctypes.POINTER(EchoOpticalGlauber), ctypes.c_double, D, D]),
    "echo_gpu_dump_size": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_size_t)]),
    "echo_gpu_dump": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.c_size_t]),
    "echo_gpu_restart_dump": (ctypes.c_int, [P, P, ctypes.c_size_t, I]),
    "echo_gpu_check_temp": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, D, I]),
    "echo_gpu_out_vars_size": (ctypes.c_int, [P, ctypes.c_uint, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "echo_gpu_out_vars": (ctypes.c_int, [P, ctypes.c_uint, ctypes.c_int, P, ctypes.c_size_t, I]),
    "echo_batch_set_stop": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double]),
    "echo_batch_init": (ctypes.c_int, [P, D, ctypes.c_int, ctypes.c_int, ctypes.POINTER(EchoEventGrid),
                                       ctypes.POINTER(P)]),
    "echo_batch_free": (ctypes.c_int, [P]),
    "echo_batch_nv": (ctypes.c_int, [P]),
    "echo_batch_offsets": (ctypes.c_int, [P, LL]),
    "echo_batch_upload": (ctypes.c_int, [P, D, D, ctypes.c_double, ctypes.c_double]),
    "echo_batch_upload_device": (ctypes.c_int, [P, P, P, ctypes.c_double, ctypes.c_double]),
    "echo_batch_download": (ctypes.c_int, [P, D, D]),
    "echo_batch_glauber": (ctypes.c_int, [P, D, LL, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double]),
    "echo_batch_run": (ctypes.c_int, [P, ctypes.c_int]),
    "echo_batch_mlp_set": (ctypes.c_int, [P, F, F]),
    "echo_batch_live": (ctypes.c_int, [P, I]),
    "echo_batch_status": (ctypes.c_int, [P, ctypes.POINTER(EchoEventStatus)]),
    "echo_batch_sync": (ctypes.c_int, [P]),
    "echo_batch_stream": (ctypes.c_int, [P, ctypes.POINTER(P)]),
    "echo_batch_set_schedule": (ctypes.c_int, [P, I, I]),
    "echo_batch_get_schedule": (ctypes.c_int, [P, I]),
    "echo_batch_autotune": (ctypes.c_int, [P, ctypes.c_int, D]),
    "echo_batch_autotune_report": (ctypes.c_int, [P, D, ctypes.c_int, I]),
    "echo_batch_set_tiles": (ctypes.c_int, [P, I]),
    "echo_batch_set_mode": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int]),
    "echo_batch_get_tuning": (ctypes.c_int, [P, I]),
    "echo_batch_profile_step": (ctypes.c_int, [P, D, I]),
}


def library_path(exact: bool = False) -> str:
    return os.path.join(LIBDIR, "libechogpu_exact.so" if exact else "libechogpu.so")


def load(exact: bool = False) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    path = library_path(exact)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing: run __graft_entry__.build()")
    L = ctypes.CDLL(path)
    for name, (res, args) in FUNCTIONS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[path] = L
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(I)


class CrashError(RuntimeError):
    """A stage failed: the reference would set run_crashed (echo.f90:206)."""

    def __init__(self, code: int, cell: int = -1):
        super().__init__(f"run crashed, reference error code {code} at cell {cell}")
        self.code = code
        self.cell = cell


class Evolve:
    """Device-resident state and the step of evolve.f90 behind the C-ABI."""

    def __init__(self, params: EchoParams, eos_table=None, exact: bool = False):
        self.lib = load(exact)
        self.params = params
        self._tab = None if eos_table is None else np.ascontiguousarray(eos_table, dtype=np.float64)
        n = 0 if self._tab is None else len(self._tab)
        h = P()
        rc = self.lib.echo_gpu_init(ctypes.byref(params), _dp(self._tab), n, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"echo_gpu_init failed with status {rc}")
        self.h = h
        self.nv = self.lib.echo_gpu_nv(h)
        self.ncell = params.nx * params.ny * params.nz

    def close(self):
        if getattr(self, "h", None):
            self.lib.echo_gpu_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise RuntimeError(f"{what} failed with status {rc}")

    def upload(self, v, u=None, t: float = 0.4):
        v = np.ascontiguousarray(v, dtype=np.float64)
        u = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        self._check(self.lib.echo_gpu_upload(self.h, _dp(v), _dp(u), t), "upload")

    def upload_device(self, v_ptr: int, u_ptr: int | None, t: float):
        self._check(self.lib.echo_gpu_upload_device(self.h, v_ptr, u_ptr, t), "upload_device")

    def download(self):
        v = np.empty(self.ncell * self.nv)
        u = np.empty(self.ncell * self.nv)
        self._check(self.lib.echo_gpu_download(self.h, _dp(v), _dp(u)), "download")
        return v, u

    def download_device(self, v_ptr: int, u_ptr: int | None):
        self._check(self.lib.echo_gpu_download_device(self.h, v_ptr, u_ptr), "download_device")

    def put_state(self, v_host_ptr: int, u_host_ptr: int):
        self._check(self.lib.echo_gpu_put_state(self.h, v_host_ptr, u_host_ptr), "put_state")

    def get_state(self, v_host_ptr: int, u_host_ptr: int | None):
        self._check(self.lib.echo_gpu_get_state(self.h, v_host_ptr, u_host_ptr), "get_state")

    def set_tout(self, tout: float):
        self._check(self.lib.echo_gpu_set_tout(self.h, tout), "set_tout")

    def evolve_main(self, irk: int) -> float:
        dt = ctypes.c_double(0)
        code = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_evolve_main(self.h, irk, ctypes.byref(dt), ctypes.byref(code)),
                    "evolve_main")
        if code.value:
            raise CrashError(code.value)
        return dt.value

    def end_step(self):
        self._check(self.lib.echo_gpu_end_step(self.h), "end_step")

    def step(self) -> float:
        dt = ctypes.c_double(0)
        code = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_step(self.h, ctypes.byref(dt), ctypes.byref(code)), "step")
        if code.value:
            raise CrashError(code.value)
        return dt.value

    def advance_host(self, v_in_ptr: int, u_in_ptr: int, v_out_ptr: int | None, u_out_ptr: int | None,
                     nsteps: int = 1):
        """put_state, run(nsteps) and get_state in one call (host pointers,
        asynchronous); the copy of u overlaps the first flux sweeps."""
        self._check(self.lib.echo_gpu_advance_host(self.h, v_in_ptr, u_in_ptr, v_out_ptr, u_out_ptr, nsteps),
                    "advance_host")

    def run(self, nsteps: int):
        self._check(self.lib.echo_gpu_run(self.h, nsteps), "run")

    def sync(self):
        self._check(self.lib.echo_gpu_sync(self.h), "sync")

    def stats(self) -> EchoStats:
        st = EchoStats()
        self._check(self.lib.echo_gpu_stats(self.h, ctypes.byref(st)), "stats")
        return st

    def set_seed_network(self, weights, norm):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        n = np.ascontiguousarray(norm, dtype=np.float32)
        self._check(self.lib.echo_gpu_mlp_set(self.h, w.ctypes.data_as(F), n.ctypes.data_as(F)), "mlp_set")

    def stream_handle(self) -> int:
        s = P()
        self._check(self.lib.echo_gpu_stream(self.h, ctypes.byref(s)), "stream")
        return s.value or 0

    KERNEL_CLASSES = ("faces_x", "faces_y", "faces_z", "stage_scalars", "update_c2p", "repair", "end_step",
                      "stage_fused")

    def profile_step(self):
        ms = np.zeros(len(self.KERNEL_CLASSES))
        n = np.zeros(len(self.KERNEL_CLASSES), dtype=np.int32)
        self._check(self.lib.echo_gpu_profile_step(self.h, _dp(ms), _ip(n)), "profile_step")
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_CLASSES)}

    def set_faces(self, mode: int):
        """Product build: how the WENO5 face sweeps run -- 0 one thread per
        face (the default), 8 or 16 cell-centred segments of that many
        cells."""
        self._check(self.lib.echo_gpu_set_faces(self.h, mode), "set_faces")

    def set_sweeps(self, concurrent: bool = True):
        """The x, y and eta sweeps of a stage side by side on three streams
        (the default) or one after another."""
        self._check(self.lib.echo_gpu_set_sweeps(self.h, int(concurrent)), "set_sweeps")

    def set_stage(self, fused: bool = True, tx: int = 0, ty: int = 0, zseg: int = 0) -> dict:
        """Fused stage kernel on or off (and its tile); returns the choice."""
        info = np.zeros(7, dtype=np.int32)
        rc = self.lib.echo_gpu_set_stage(self.h, int(fused), tx, ty, zseg, _ip(info))
        if rc not in (0, -3) or (rc == -3 and fused):
            raise RuntimeError(f"set_stage failed with status {rc}")
        return dict(zip(("fused", "tx", "ty", "zseg", "threads", "ctas", "smem_bytes"), info.tolist()))

    def hyp_init(self, freeze_type: int, freeze_value: float) -> None:
        """Freeze-out hypersurface on T (0) or e (1) = freeze_value."""
        self._check(self.lib.echo_gpu_hyp_init(self.h, freeze_type, freeze_value), "hyp_init")

    def hyp_step(self) -> np.ndarray:
        """One out_hyp call: the elements found now, shape (n, 8 + nv)."""
        n = ctypes.c_int(0)
        err = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_hyp_step(self.h, ctypes.byref(n), ctypes.byref(err)), "hyp_step")
        if err.value:
            raise CrashError(err.value)
        out = np.empty((n.value, 8 + self.nv))
        if n.value:
            self._check(self.lib.echo_gpu_hyp_get(self.h, _dp(out)), "hyp_get")
        return out

    def optical_glauber(self, g: EchoOpticalGlauber, t: float, peak: float | None = None) -> tuple[float, float]:
        """The optical Glauber initial state on the device, uploaded at time
        t; with `peak`, ecenter is rescaled so that the grid's largest e is
        `peak` (a second device pass).  Returns (check mass, max e)."""
        chk = ctypes.c_double(0)
        mx = ctypes.c_double(0)
        self._check(self.lib.echo_gpu_optical_glauber(self.h, ctypes.byref(g), t, ctypes.byref(chk),
                                                      ctypes.byref(mx)), "optical_glauber")
        if peak is not None:
            g2 = EchoOpticalGlauber.from_buffer_copy(g)
            g2.ecenter = g.ecenter * peak / mx.value
            self._check(self.lib.echo_gpu_optical_glauber(self.h, ctypes.byref(g2), t, ctypes.byref(chk),
                                                          ctypes.byref(mx)), "optical_glauber")
        return chk.value, mx.value

    def keep_old(self, on: bool = True):
        """Keep the reference's vold/uold (for a complete dump.dat)."""
        self._check(self.lib.echo_gpu_keep_old(self.h, int(on)), "keep_old")

    def dump(self, iout: int) -> bytes:
        """The bytes of dump.dat (out_dump, out.f90:1313-1392)."""
        n = ctypes.c_size_t(0)
        self._check(self.lib.echo_gpu_dump_size(self.h, ctypes.byref(n)), "dump_size")
        buf = ctypes.create_string_buffer(n.value)
        self._check(self.lib.echo_gpu_dump(self.h, iout, ctypes.cast(buf, P), n.value), "dump")
        return buf.raw

    def restart_dump(self, data: bytes) -> int:
        """Restart from the bytes of a dump.dat (out_restart); returns iout."""
        buf = ctypes.create_string_buffer(data, len(data))
        io = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_restart_dump(self.h, ctypes.cast(buf, P), len(data), ctypes.byref(io)),
                    "restart_dump")
        return io.value

    def checkpoint(self) -> bytes:
        """The run state at this step boundary (out_dump's role)."""
        n = ctypes.c_size_t(0)
        self._check(self.lib.echo_gpu_checkpoint_size(self.h, ctypes.byref(n)), "checkpoint_size")
        buf = ctypes.create_string_buffer(n.value)
        self._check(self.lib.echo_gpu_checkpoint(self.h, buf), "checkpoint")
        return buf.raw

    def restart(self, blob: bytes) -> None:
        """Continue from a checkpoint of a run of the same shape (out_restart)."""
        buf = ctypes.create_string_buffer(blob, len(blob))
        self._check(self.lib.echo_gpu_restart(self.h, buf), "restart")

    def check_temp(self, freeze_type: int = 1, temp_end: float = 0.0):
        """check_temp (out.f90:1487-1557) on the device: (maximum, stop)."""
        m = ctypes.c_double(0)
        stop = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_check_temp(self.h, freeze_type, temp_end, ctypes.byref(m),
                                                 ctypes.byref(stop)), "check_temp")
        return m.value, bool(stop.value)

    def out_vars(self, sel: int, precision: int = 8):
        """out_vars (out.f90:232-591) staged on the device: (bytes of one
        outNNNN.dat, errcode of the first cell whose derived data fail)."""
        n = ctypes.c_size_t(0)
        self._check(self.lib.echo_gpu_out_vars_size(self.h, sel, precision, ctypes.byref(n)), "out_vars_size")
        buf = ctypes.create_string_buffer(n.value)
        err = ctypes.c_int(0)
        self._check(self.lib.echo_gpu_out_vars(self.h, sel, precision, ctypes.cast(buf, ctypes.c_void_p), n.value,
                                               ctypes.byref(err)), "out_vars")
        return bytes(buf.raw), err.value

    def rhs(self):
        du = np.empty(self.ncell * self.nv)
        am = np.empty(3)
        rc = self.lib.echo_gpu_rhs(self.h, _dp(du), _dp(am))
        if rc < 0:
            raise RuntimeError(f"rhs failed with status {rc}")
        return du, am


def unit_recon(recal: int, f: np.ndarray, n: int, exact: bool = True):
    L = load(exact)
    f = np.ascontiguousarray(f, dtype=np.float64)
    m = f.shape[0]
    gl = np.empty((m, n + 1))
    gr = np.empty((m, n + 1))
    rc = L.echo_gpu_test_recon(recal, m, n, _dp(f), _dp(gl), _dp(gr))
    if rc:
        raise RuntimeError(f"test_recon status {rc}")
    return gl, gr


def unit_fastdiv(d, n, exact: bool = False):
    """n[j] // d[i] on the device by the kernels' multiply-high division."""
    L = load(exact)
    d = np.ascontiguousarray(d, dtype=np.uint32)
    n = np.ascontiguousarray(n, dtype=np.uint32)
    q = np.empty((len(d), len(n)), dtype=np.uint32)
    rc = L.echo_gpu_test_fastdiv(d.ctypes.data, len(d), n.ctypes.data, len(n), q.ctypes.data)
    if rc:
        raise RuntimeError(f"test_fastdiv status {rc}")
    return q


def unit_c2p(params, eos_table, g3, gp, u, vguess, exact: bool = True):
    L = load(exact)
    tab = None if eos_table is None else np.ascontiguousarray(eos_table, dtype=np.float64)
    n = 0 if tab is None else len(tab)
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(vguess, dtype=np.float64).copy()
    nc = u.shape[0]
    err = np.zeros(nc, dtype=np.int32)
    it = np.zeros(nc, dtype=np.int32)
    rc = L.echo_gpu_test_c2p(ctypes.byref(params), _dp(tab), n, nc, g3, gp, _dp(u), _dp(v), _ip(err), _ip(it))
    if rc:
        raise RuntimeError(f"test_c2p status {rc}")
    return v, err, it


def unit_c2p_seeded(params, eos_table, g3, gp, u, vguess, weights=None, norm=None):
    """con2prim of independent RMHD cells from the learned seed (weights
    given) or by Newton from vguess; returns v, err, iters, seed_failed."""
    L = load(False)
    tab = np.ascontiguousarray(eos_table, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(vguess, dtype=np.float64).copy()
    nc = u.shape[0]
    err = np.zeros(nc, dtype=np.int32)
    it = np.zeros(nc, dtype=np.int32)
    sf = np.zeros(nc, dtype=np.int32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    nm = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
    rc = L.echo_gpu_test_c2p_seeded(ctypes.byref(params), _dp(tab), len(tab), nc, g3, gp,
                                    None if w is None else w.ctypes.data_as(F),
                                    None if nm is None else nm.ctypes.data_as(F),
                                    _dp(u), _dp(v), _ip(err), _ip(it), _ip(sf))
    if rc:
        raise RuntimeError(f"test_c2p_seeded status {rc}")
    return v, err, it, sf


def fp64_peak() -> tuple[float, float]:
    """Measured FP64 GFLOP/s of the current GPU and the timed launch's ms."""
    L = load(False)
    g = ctypes.c_double(0)
    ms = ctypes.c_double(0)
    rc = L.echo_gpu_fp64_peak(ctypes.byref(g), ctypes.byref(ms))
    if rc:
        raise RuntimeError(f"fp64_peak status {rc}")
    return g.value, ms.value
