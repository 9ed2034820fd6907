"""ctypes binding of the CPU oracle (liboracle_echo.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py for the CPU baseline.  The product path never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_echo.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = P
        L.orc_create.argtypes = [P, D, ctypes.c_int]
        L.orc_free.argtypes = [P]
        L.orc_nv.argtypes = [P]
        L.orc_set_threads.argtypes = [P, ctypes.c_int]
        L.orc_set_state.argtypes = [P, D, D, ctypes.c_double]
        L.orc_get_state.argtypes = [P, D, D]
        L.orc_set_tout.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_evolve_main.argtypes = [P, ctypes.c_int, D]
        L.orc_step.argtypes = [P, D]
        L.orc_rhs.argtypes = [P, D, D]
        for f in ("orc_time", "orc_dt", "orc_glm_ch"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [P]
        for f in ("orc_repairs", "orc_c2p_iters"):
            getattr(L, f).restype = ctypes.c_longlong
            getattr(L, f).argtypes = [P]
        L.orc_hyp_init.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.orc_hyp_step.argtypes = [P, I]
        L.orc_hyp_get.argtypes = [P, D]
        L.orc_check_temp.restype = ctypes.c_double
        L.orc_check_temp.argtypes = [P, ctypes.c_int]
        L.orc_out_vars.restype = ctypes.c_size_t
        L.orc_out_vars.argtypes = [P, ctypes.c_uint, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.orc_recon.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D]
        L.orc_c2p.argtypes = [P, D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                              ctypes.c_double, D, D, I, I]
        L.orc_prim2cons.argtypes = [P, D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, D, D]
        L.orc_flux.argtypes = [P, D, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                               ctypes.c_int, D, D, D, D]
        Fp = ctypes.POINTER(ctypes.c_float)
        L.orc_mlp_grad.argtypes = [Fp, Fp, Fp, ctypes.c_int, D, D]
        L.orc_mlp_forward.argtypes = [Fp, Fp, Fp, ctypes.c_int, D]
        L.orc_eos_energy.argtypes = [P, D, ctypes.c_int, ctypes.c_double, D]
        L.orc_thickness.restype = ctypes.c_double
        L.orc_thickness.argtypes = [ctypes.c_double] * 6 + [ctypes.c_int, D]
        L.orc_optical_glauber.restype = ctypes.c_double
        L.orc_optical_glauber.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 + [D]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _tab(tab):
    if tab is None:
        return None, 0
    t = np.ascontiguousarray(tab, dtype=np.float64)
    return t, len(t)


class Oracle:
    """The reference step on the CPU (evolve.f90 restated)."""

    def __init__(self, params, eos_table=None, threads: int = 1):
        self.params = params
        self._tab, n = _tab(eos_table)
        self.h = lib().orc_create(ctypes.byref(params), _dp(self._tab), n)
        if not self.h:
            raise ValueError("oracle: unsupported parameter combination")
        self.nv = lib().orc_nv(self.h)
        self.ncell = params.nx * params.ny * params.nz
        lib().orc_set_threads(self.h, threads)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def set_state(self, v, u=None, t: float = 0.4):
        v = np.ascontiguousarray(v, dtype=np.float64)
        uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        err = lib().orc_set_state(self.h, _dp(v), _dp(uu), t)
        if err:
            raise RuntimeError(f"oracle prim2cons error {err}")

    def set_tout(self, tout: float, dtout: float = 1e300, tmax: float = 1e300):
        lib().orc_set_tout(self.h, tout, dtout, tmax)

    def state(self):
        v = np.empty(self.ncell * self.nv)
        u = np.empty(self.ncell * self.nv)
        lib().orc_get_state(self.h, _dp(v), _dp(u))
        return v, u

    def step(self) -> float:
        dt = ctypes.c_double(0)
        err = lib().orc_step(self.h, ctypes.byref(dt))
        if err:
            raise RuntimeError(f"oracle step error {err}")
        return dt.value

    def evolve_main(self, irk: int) -> float:
        dt = ctypes.c_double(0)
        err = lib().orc_evolve_main(self.h, irk, ctypes.byref(dt))
        if err:
            raise RuntimeError(f"oracle evolve_main error {err}")
        return dt.value

    def rhs(self):
        du = np.empty(self.ncell * self.nv)
        am = np.empty(3)
        err = lib().orc_rhs(self.h, _dp(du), _dp(am))
        if err:
            raise RuntimeError(f"oracle rhs error {err}")
        return du, am

    @property
    def t(self) -> float:
        return lib().orc_time(self.h)

    @property
    def dt(self) -> float:
        return lib().orc_dt(self.h)

    @property
    def glm_ch(self) -> float:
        return lib().orc_glm_ch(self.h)

    def out_vars(self, sel: int, precision: int = 8):
        """out_vars (out.f90:232-591): (bytes of one outNNNN.dat, errcode)."""
        n = lib().orc_out_vars(self.h, sel, precision, None, None)
        buf = ctypes.create_string_buffer(n)
        err = ctypes.c_int(0)
        lib().orc_out_vars(self.h, sel, precision, ctypes.cast(buf, ctypes.c_void_p), ctypes.byref(err))
        return bytes(buf.raw), err.value

    def check_temp(self, freeze_type: int = 1) -> float:
        """check_temp (out.f90:1487-1557): maximum T (0) or e (1) over the grid."""
        return lib().orc_check_temp(self.h, freeze_type)

    def hyp_init(self, freeze_type: int, freeze_value: float) -> None:
        if lib().orc_hyp_init(self.h, freeze_type, freeze_value):
            raise ValueError("freeze_type must be 0 or 1")

    def hyp_step(self) -> np.ndarray:
        """out_hyp: the surface elements found now, shape (n, 8 + nv)."""
        n = ctypes.c_int(0)
        err = lib().orc_hyp_step(self.h, ctypes.byref(n))
        if err:
            raise RuntimeError(f"oracle hypersurface error {err}")
        out = np.empty((n.value, 8 + self.nv))
        if n.value:
            lib().orc_hyp_get(self.h, _dp(out))
        return out

    @property
    def repairs(self) -> int:
        return lib().orc_repairs(self.h)

    @property
    def c2p_iters(self) -> int:
        return lib().orc_c2p_iters(self.h)


def recon(recal: int, f: np.ndarray, n: int):
    """f: (m, n+8) pencils with f[:, i+4] = f(i); returns gl, gr (m, n+1)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    m = f.shape[0]
    gl = np.empty((m, n + 1))
    gr = np.empty((m, n + 1))
    lib().orc_recon(recal, m, n, _dp(f), _dp(gl), _dp(gr))
    return gl, gr


def c2p(params, eos_table, g3, gp, u, vguess):
    t, n = _tab(eos_table)
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(vguess, dtype=np.float64).copy()
    nc = u.shape[0]
    err = np.zeros(nc, dtype=np.int32)
    it = np.zeros(nc, dtype=np.int32)
    lib().orc_c2p(ctypes.byref(params), _dp(t), n, nc, g3, gp, _dp(u), _dp(v), _ip(err), _ip(it))
    return v, err, it


def prim2cons(params, eos_table, g3, gp, v):
    t, n = _tab(eos_table)
    v = np.ascontiguousarray(v, dtype=np.float64).copy()
    u = np.zeros_like(v)
    bad = lib().orc_prim2cons(ctypes.byref(params), _dp(t), n, v.shape[0], g3, gp, _dp(v), _dp(u))
    return v, u, bad


def flux(params, eos_table, g3, gp, direction, v):
    t, n = _tab(eos_table)
    v = np.ascontiguousarray(v, dtype=np.float64).copy()
    u = np.zeros_like(v)
    f = np.zeros_like(v)
    vf = np.zeros(2)
    err = lib().orc_flux(ctypes.byref(params), _dp(t), n, g3, gp, direction, _dp(v), _dp(u), _dp(f), _dp(vf))
    return err, u, f, vf


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def mlp_grad(weights, Xs, Ts):
    """FP64 loss and gradient of the seed network on standardised rows."""
    W = np.ascontiguousarray(weights, dtype=np.float32)
    X = np.ascontiguousarray(Xs, dtype=np.float32)
    T = np.ascontiguousarray(Ts, dtype=np.float32)
    g = np.zeros(W.size)
    loss = ctypes.c_double(0)
    lib().orc_mlp_grad(_fp(W), _fp(X), _fp(T), len(X), ctypes.byref(loss), _dp(g))
    return loss.value, g


def mlp_forward(weights, norm, X):
    W = np.ascontiguousarray(weights, dtype=np.float32)
    N = np.ascontiguousarray(norm, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.zeros((len(X), 2))
    lib().orc_mlp_forward(_fp(W), _fp(N), _fp(X), len(X), _dp(out))
    return out


def eos_energy(params, eos_table, pr: float) -> tuple[int, float]:
    """get_energy (eos.f90:468-523) of the tabulated EoS at pressure pr."""
    tab, n = _tab(eos_table)
    en = ctypes.c_double(0)
    err = lib().orc_eos_energy(ctypes.byref(params), _dp(tab), n, pr, ctypes.byref(en))
    return err, en.value


def thickness(radius, delta, roze, dr, dz1, acc, nmax):
    """thickness (init.f90:1164-1219): (check mass, T(r) table)."""
    thick = np.empty(nmax)
    chk = lib().orc_thickness(radius, delta, roze, dr, dz1, acc, nmax, _dp(thick))
    return chk, thick


def optical_glauber(g, nx, ny, nz, x1, x2, y1, y2, z1, z2):
    """calc_enedens (init.f90:902-929) at the cell centres: (check mass, e)."""
    e = np.empty(nx * ny * nz)
    chk = lib().orc_optical_glauber(ctypes.byref(g), nx, ny, nz, x1, x2, y1, y2, z1, z2, _dp(e))
    return chk, e
