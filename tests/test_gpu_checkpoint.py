"""Checkpoint and restart of a run (the role of out_dump / out_restart,
out.f90:1313-1483): a context restarted from a checkpoint continues bit for
bit as the original run does."""
import numpy as np
import pytest

from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,nrk", [("hd2d", None), ("rmhd3d", None), ("visc2d", None), ("hd2d", P.SSP), ("res3d", None)])
def test_restart_continues_bit_for_bit(case, nrk):
    cfg = CASES[case]()
    if nrk is not None:
        cfg = cfg.replace(nrk=nrk)
    if cfg.viscosity:
        cfg = cfg.replace(smooth_temp=0.35)  # smoothing and the lagged time derivatives both active
    pc, tab, v = setup(cfg)
    a = Evolve(pc, tab)
    a.upload(v, None, cfg.tstart)
    a.run(3)
    a.sync()
    blob = a.checkpoint()
    a.run(4)
    a.sync()
    va, ua = a.download()
    sa = a.stats()
    b = Evolve(pc.__class__.from_buffer_copy(pc), tab)
    b.upload(v, None, cfg.tstart)
    b.run(1)  # some other state first: the restart replaces all of it
    b.restart(blob)
    b.run(4)
    b.sync()
    vb, ub = b.download()
    sb = b.stats()
    assert sa.errcode == 0 and sb.errcode == 0
    assert np.array_equal(va, vb) and np.array_equal(ua, ub)
    assert sa.t == sb.t and sa.dt == sb.dt


def test_restart_rejects_another_shape():
    cfg = CASES["hd2d"]()
    pc, tab, v = setup(cfg)
    a = Evolve(pc, tab)
    a.upload(v, None, cfg.tstart)
    blob = a.checkpoint()
    other = P.small(P.config0(), 10)
    pc2, tab2, v2 = setup(other)
    b = Evolve(pc2, tab2)
    b.upload(v2, None, other.tstart)
    with pytest.raises(RuntimeError):
        b.restart(blob)
