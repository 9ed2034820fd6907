"""echo_gpu_advance_host (the host-owned state advanced by n steps in one
call, the copy of u overlapping the first flux sweeps) against the same
steps through echo_gpu_put_state, echo_gpu_run and echo_gpu_get_state: the
same bits, for each way a step first touches u (explicit RK after the
sweeps; IMEX-SSP, the fused stage and the kept vold/uold at once), for one
and several steps per call, and with zero steps (the state copied in and
back out)."""
import numpy as np
import pytest

from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, resistive_state, setup

pytestmark = pytest.mark.gpu

RUNS = {
    "rmhd3d_rk3": (lambda: CASES["rmhd3d"](), {}),
    "visc2d_imex": (lambda: CASES["visc2d"]().replace(imex=1), {}),
    "res3d_ssp": (lambda: CASES["res3d"]().replace(sigma_el=500.0), {}),
    "hd2d_keep_old": (lambda: CASES["hd2d"](), {"keep_old": True}),
    "rmhd3d_fused": (lambda: CASES["rmhd3d"](), {"fused": True}),
}


def _make(pc, tab, exact, opt):
    g = Evolve(pc, tab, exact=exact)
    if opt.get("keep_old"):
        g.keep_old(True)
    if opt.get("fused"):
        assert g.set_stage(True)["fused"] == 1
    return g


@pytest.mark.parametrize("name", list(RUNS))
@pytest.mark.parametrize("exact", [False, True])
def test_advance_host_equals_put_run_get(name, exact):
    mk, opt = RUNS[name]
    cfg = mk()
    pc, tab, v = setup(cfg)
    if name.startswith("res"):
        v = resistive_state(cfg, tab)
    states = []
    for use_advance in (False, True):
        g = _make(pc, tab, exact, opt)
        g.upload(v, None, cfg.tstart)
        g.run(1)
        hv, hu = g.download()
        for n in (1, 3, 0, 2):
            if use_advance:
                g.advance_host(hv.ctypes.data, hu.ctypes.data, hv.ctypes.data, hu.ctypes.data, n)
            else:
                g.put_state(hv.ctypes.data, hu.ctypes.data)
                g.run(n)
                g.get_state(hv.ctypes.data, hu.ctypes.data)
            g.sync()
        st = g.stats()
        assert st.errcode == 0
        states.append((hv.copy(), hu.copy(), st.t, st.dt))
        g.close()
    (v0, u0, t0, d0), (v1, u1, t1, d1) = states
    assert t0 == t1 and d0 == d1
    assert np.array_equal(v0, v1) and np.array_equal(u0, u1)


def test_advance_host_and_set_sweeps_check_their_arguments():
    cfg = CASES["hd2d"]()
    pc, tab, v = setup(cfg)
    g = Evolve(pc, tab, exact=False)
    g.upload(v, None, cfg.tstart)
    hv, hu = g.download()
    with pytest.raises(RuntimeError):
        g.advance_host(hv.ctypes.data, hu.ctypes.data, None, None, -1)
    with pytest.raises(RuntimeError):
        g.advance_host(0, hu.ctypes.data, None, None, 1)
    with pytest.raises(RuntimeError):
        g.set_sweeps(2)
    # outputs may be omitted: the state advances on the device all the same
    g.advance_host(hv.ctypes.data, hu.ctypes.data, None, None, 2)
    g.sync()
    assert g.stats().errcode == 0
    g.close()
