"""The freeze-out hypersurface on the device against the oracle's
restatement of out_hyp / find_hypersurface_* (out.f90:1569-1650,
hypersurface.f90:172-460, 775-1117): the same elements, in the same order,
call after call.  Tolerances: the exact build bit-for-bit up to the last-place
differences of its input state (1e-13 relative), the product build 1e-12."""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, field_groups, setup

pytestmark = pytest.mark.gpu


def _freeze_value(cfg, tab, v, freeze_type):
    """The median of the freeze field over the initial grid, so the surface
    runs through it."""
    p = v.reshape(cfg.nv, -1)[4]
    if tab is None:  # p = e/3, T = 0.148909 e^(1/4) (temperature.def)
        e = 3.0 * p
        T = 0.148909 * e ** 0.25
    else:
        e = np.interp(p, tab[:, 2], tab[:, 1])
        T = np.interp(p, tab[:, 2], tab[:, 0])
    return float(np.median(T if freeze_type == 0 else e))


def _rel_err(a, b, nv):
    """Largest relative difference of two element lists: positions and dV by
    column, the interpolated primitives by field group (as the step parity
    tests: analytically zero fields hold only round-off)."""
    d = np.abs(a - b)
    worst = 0.0
    for cols in [[0], [1], [2], [3], [4 + nv], [5 + nv], [6 + nv], [7 + nv]] + \
            [[4 + k for k in grp] for grp in field_groups(nv)]:
        scale = np.abs(b[:, cols]).max()
        if scale > 0:
            worst = max(worst, float(d[:, cols].max() / scale))
    return worst


@pytest.mark.parametrize("case,freeze_type", [("hd2d", 0), ("visc2d", 1), ("rmhd3d", 0)])
@pytest.mark.parametrize("exact,tol", [(True, 1e-13), (False, 1e-12)])
def test_hypersurface_matches_oracle(case, freeze_type, exact, tol):
    cfg = CASES[case]()
    if case == "hd2d":
        cfg = P.small(P.config0(), 24)
    pc, tab, v = setup(cfg)
    fv = _freeze_value(cfg, tab, v, freeze_type)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc.__class__.from_buffer_copy(pc), tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    o.hyp_init(freeze_type, fv)
    g.hyp_init(freeze_type, fv)
    total, tau_elems = 0, 0
    for call in range(5):
        ho = o.hyp_step()
        hg = g.hyp_step()
        assert hg.shape == ho.shape, (call, hg.shape, ho.shape)
        if len(ho):
            assert _rel_err(hg, ho, g.nv) <= tol, call
            total += len(ho)
            tau_elems += int((ho[:, 4 + g.nv] != 0).sum())
        o.step()
        g.step()
    assert total > 0 and tau_elems > 0  # crossings in space and in tau were both exercised
