"""echo_gpu_rhs_noalloc against echo_gpu_rhs.

The allocation-free entry point serves callers that cannot allocate device
memory (a host code coupled inside a GPU application whose memory belongs
to another allocator, or a driver that must not allocate between graph
captures).  Its face-flux scratch is a fixed file-scope device array, so
this file is collected last: if it fails, a run that stops at the first
failure has already run every other test.  The check: through the C-ABI,
on device buffers the test owns, two calls in a row give the du of the
existing entry point within the tolerance of the other parity tests.
"""
import ctypes

import numpy as np
import pytest

from echo_gpu import lib as L
from helpers import CASES, eos_table, rel_linf, setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["rmhd3d", "hd2d", "visc2d"])
def test_rhs_noalloc_matches_rhs(case):
    import torch

    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    ref = L.Evolve(pc, tab, exact=True)
    ref.upload(v, None, cfg.tstart)
    du_ref, _ = ref.rhs()
    v_dev, _ = ref.download()  # the primitives the reference call saw

    lib = L.load(exact=True)
    d_v = torch.from_numpy(v_dev).cuda()
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
        rc = lib.echo_gpu_rhs_noalloc(ctypes.byref(pc), tab_ptr, n_eos, cfg.tstart, d_v.data_ptr(),
                                      d_du.data_ptr(), stream, ctypes.byref(code))
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        assert code.value == 0
        du = d_du.cpu().numpy()
        assert np.isfinite(du).all()
        assert rel_linf(du, du_ref, cfg.nv) <= 1e-13, (call, rel_linf(du, du_ref, cfg.nv))


def test_rhs_noalloc_rejects_grids_beyond_the_scratch():
    import torch

    from echo_gpu import params as P

    cfg = P.config1()  # 97x97x81 x 9 variables: far beyond the fixed scratch
    pc, tab, _ = setup(cfg.replace(nx=8, ny=8, nz=8))
    pc.nx, pc.ny, pc.nz = cfg.nx, cfg.ny, cfg.nz
    lib = L.load(exact=True)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    d_tab = torch.from_numpy(np.ascontiguousarray(np.asarray(eos_table()).T).reshape(-1)).cuda()
    rc = lib.echo_gpu_rhs_noalloc(ctypes.byref(pc), d_tab.data_ptr(), len(eos_table()), 0.4, d.data_ptr(),
                                  d.data_ptr(), None, None)
    assert rc == -1  # ECHO_ERR_ARG, before any device work
