"""dump.dat in the reference's layout (out_dump / out_restart,
out.f90:1313-1483): the device's dump parses as out_restart reads it, holds
the current state and the reference's vold/uold (the state at the start of
the previous step), and a context restarted from it continues as the
reference's restart does -- bit for bit with the uninterrupted run where the
reference's restart loses nothing (hydro and viscous runs: dt and the GLM
speed, which dump.dat does not hold, do not enter their next steps), and as
a fresh upload of the same state with divergence cleaning (the GLM speed
restarts from its initial value there, in the reference as here)."""
import numpy as np
import pytest

from echo_gpu import output as OUT
from echo_gpu.lib import Evolve
from helpers import CASES, setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["hd2d", "visc2d", "rmhd3d"])
def test_dump_layout_and_restart(case, tmp_path):
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    a = Evolve(pc, tab, exact=True)
    a.upload(v, None, cfg.tstart)
    a.keep_old(True)
    a.run(3)
    a.sync()
    v_prev, u_prev = a.download()  # the state at the start of the 4th step
    a.run(1)
    a.sync()
    st = a.stats()
    blob = a.dump(7)
    path = OUT.write_dump(str(tmp_path), 1, blob)
    with open(path, "rb") as f:
        d = OUT.read_dump(f.read(), cfg)
    vn, un = a.download()
    kold = 8 if cfg.mhd else 5
    nc = cfg.ncell
    assert d["iout"] == 7 and d["t"] == st.t and d["timeinterval"] == st.dt
    assert d["timeold"] == st.t - st.dt or abs(d["timeold"] - (st.t - st.dt)) <= 1e-15 * st.t
    assert d["g_cov_3_old"] == d["timeold"] ** 2  # Milne: g_33 of the previous step
    assert np.array_equal(d["vall"], vn) and np.array_equal(d["uall"], un)
    # vold / uold: the state at the start of the previous step, fields krh..kvold_end
    assert np.array_equal(d["vallold"], v_prev[:kold * nc]) and np.array_equal(d["uallold"], u_prev[:kold * nc])
    # continue the original, and restart a fresh context from the file
    a.run(3)
    a.sync()
    va, ua = a.download()
    b = Evolve(pc, tab, exact=True)
    b.keep_old(True)
    assert b.restart_dump(blob) == 7
    b.run(3)
    b.sync()
    vb, ub = b.download()
    if cfg.divclean:
        # the reference's restart starts the GLM speed afresh: the same as an upload of the dumped state
        c = Evolve(pc, tab, exact=True)
        c.upload(d["vall"], d["uall"], d["t"])
        c.run(3)
        c.sync()
        vc, uc = c.download()
        assert np.array_equal(vb, vc) and np.array_equal(ub, uc)
    else:
        assert np.array_equal(vb, va), np.max(np.abs(vb - va))
        assert np.array_equal(ub, ua), (np.max(np.abs(ub - ua)), np.argmax(np.abs(ub - ua)) // cfg.ncell)
    assert b.stats().t == a.stats().t
    # a dump of another run's shape is refused
    other = Evolve(*setup(CASES["hd2d"]().replace(nx=14))[:2], exact=True)
    with pytest.raises(RuntimeError):
        other.restart_dump(blob)
