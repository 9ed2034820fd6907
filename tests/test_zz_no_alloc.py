"""echo_gpu_rhs_noalloc against echo_gpu_rhs and against the oracle.

The allocation-free entry point serves callers that cannot allocate device
memory (a host code coupled inside a GPU application whose memory belongs
to another allocator, or a driver that must not allocate between graph
captures).  Its face-flux scratch is a fixed file-scope device array, so
this file is collected last: if it fails, a run that stops at the first
failure has already run every other test.  The checks, through the C-ABI
on device buffers the test owns, two calls in a row each:
  - the du of the existing entry point within the tolerance of the other
    parity tests, and the oracle's right-hand side (orc_rhs) directly;
  - the same in the middle of a run (after a few steps of the
    divergence-cleaning and viscous workloads): the call carries no run
    state, so its du is the one of a context that uploads the running
    primitives at the running time, which is what both sides compute.
"""
import ctypes
import sys
import os

import numpy as np
import pytest

from echo_gpu import lib as L
from helpers import CASES, rel_linf, setup

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import pyoracle as O  # noqa: E402  (the checker)

pytestmark = pytest.mark.gpu


def _noalloc_twice(pc, tab, t, v_dev, du_ref, du_oracle, nv):
    """Two calls in a row on the caller's buffers; each compared with the
    existing entry point and with the oracle."""
    import torch

    lib = L.load(exact=True)
    d_v = torch.from_numpy(np.ascontiguousarray(v_dev)).cuda()
    d_du = torch.empty_like(d_v)
    if tab is not None:
        d_tab = torch.from_numpy(np.ascontiguousarray(np.asarray(tab).T).reshape(-1)).cuda()
        tab_ptr, n_eos = d_tab.data_ptr(), len(tab)
    else:
        tab_ptr, n_eos = None, 0
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d_du.fill_(np.nan)
        code = ctypes.c_int(-1)
        rc = lib.echo_gpu_rhs_noalloc(ctypes.byref(pc), tab_ptr, n_eos, t, d_v.data_ptr(),
                                      d_du.data_ptr(), stream, ctypes.byref(code))
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        assert code.value == 0
        du = d_du.cpu().numpy()
        assert np.isfinite(du).all()
        assert rel_linf(du, du_ref, nv) <= 1e-13, (call, rel_linf(du, du_ref, nv))
        assert rel_linf(du, du_oracle, nv) <= 1e-13, (call, rel_linf(du, du_oracle, nv))


@pytest.mark.parametrize("case", ["rmhd3d", "hd2d", "visc2d"])
def test_rhs_noalloc_matches_rhs(case):
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    ref = L.Evolve(pc, tab, exact=True)
    ref.upload(v, None, cfg.tstart)
    du_ref, _ = ref.rhs()
    v_dev, _ = ref.download()  # the primitives the reference call saw
    ref.close()
    o = O.Oracle(pc, tab)
    o.set_state(v_dev, None, cfg.tstart)
    du_o, _ = o.rhs()
    _noalloc_twice(pc, tab, cfg.tstart, v_dev, du_ref, du_o, cfg.nv)


@pytest.mark.parametrize("case", ["rmhd3d", "visc2d"])
def test_rhs_noalloc_mid_run(case):
    """After four steps of a GLM or viscous run: the noalloc du equals the
    du of a context (and of the oracle) given the running primitives at the
    running time."""
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    run = L.Evolve(pc, tab, exact=True)
    run.upload(v, None, cfg.tstart)
    for _ in range(4):
        run.step()
    t = run.stats().t
    v_mid, _ = run.download()
    run.close()
    ref = L.Evolve(pc, tab, exact=True)
    ref.upload(v_mid, None, t)
    du_ref, _ = ref.rhs()
    v_dev, _ = ref.download()
    ref.close()
    o = O.Oracle(pc, tab)
    o.set_state(v_dev, None, t)
    du_o, _ = o.rhs()
    _noalloc_twice(pc, tab, t, v_dev, du_ref, du_o, cfg.nv)


def test_rhs_noalloc_rejects_grids_beyond_the_scratch():
    import torch

    from echo_gpu import params as P
    from helpers import eos_table

    cfg = P.config1()  # 97x97x81 x 9 variables: far beyond the fixed scratch
    pc, tab, _ = setup(cfg.replace(nx=8, ny=8, nz=8))
    pc.nx, pc.ny, pc.nz = cfg.nx, cfg.ny, cfg.nz
    lib = L.load(exact=True)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    d_tab = torch.from_numpy(np.ascontiguousarray(np.asarray(eos_table()).T).reshape(-1)).cuda()
    rc = lib.echo_gpu_rhs_noalloc(ctypes.byref(pc), d_tab.data_ptr(), len(eos_table()), 0.4, d.data_ptr(),
                                  d.data_ptr(), None, None)
    assert rc == -1  # ECHO_ERR_ARG, before any device work
    # an integrator echo_gpu_init refuses is refused here too, before any launch
    pc2, _, _ = setup(cfg.replace(nx=8, ny=8, nz=8))
    pc2.nrk = 0
    rc = lib.echo_gpu_rhs_noalloc(ctypes.byref(pc2), d_tab.data_ptr(), len(eos_table()), 0.4, d.data_ptr(),
                                  d.data_ptr(), None, None)
    assert rc != 0
