"""Output staging on the device (echo_gpu_out_vars) against the oracle's
out_vars: the same bytes from the same state (exact build), 1e-12 relative
per field after steps (product build); double and single precision."""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import output as OUT
from echo_gpu import params as P
from echo_gpu.lib import Evolve
from helpers import CASES, setup

pytestmark = pytest.mark.gpu

ALL = (1 << len(OUT.FIELDS)) - 1


def _pair(case, steps, exact, **kw):
    cfg = CASES[case]().replace(**kw)
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc, tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(steps):
        o.step()
        g.step()
    return cfg, o, g


@pytest.mark.parametrize("case", ["hd2d", "visc2d", "rmhd3d", "res3d"])
@pytest.mark.parametrize("precision", [8, 4])
def test_same_bytes_from_the_same_state(case, precision):
    """Bit for bit with a tabulated EoS; with the analytic one (hd2d) the
    temperature and entropy density call pow(), which may differ from libm's
    in the last place."""
    cfg, o, g = _pair(case, 0, True)
    bo, eo = o.out_vars(ALL, precision)
    bg, eg = g.out_vars(ALL, precision)
    assert eo == eg == 0
    assert len(bo) == len(bg)
    if cfg.eqstate == P.EOS_TABLE:
        assert bo == bg
    to, fo = OUT.read(bo, cfg, ALL, precision)
    tg, fg = OUT.read(bg, cfg, ALL, precision)
    assert to == tg
    eps = np.finfo(np.float64 if precision == 8 else np.float32).eps
    for name in fo:
        if name in ("temperature", "entropy_density"):
            assert np.allclose(fg[name], fo[name], rtol=2 * eps, atol=0), name
        else:
            assert np.array_equal(fg[name], fo[name]), name


@pytest.mark.parametrize("case", ["visc2d", "rmhd3d"])
def test_after_steps_product_build(case):
    cfg, o, g = _pair(case, 3, False)
    sel = ALL
    to, fo = OUT.read(o.out_vars(sel)[0], cfg, sel)
    tg, fg = OUT.read(g.out_vars(sel)[0], cfg, sel)
    assert abs(tg - to) <= 1e-14 * to
    # normalised per field group, as the step parity is (a component that is
    # analytically zero, like v^eta here, holds round-off only)
    group = {"vx": "v", "vy": "v", "vz": "v", "bx": "em", "by": "em", "bz": "em", "ex": "em", "ey": "em",
             "ez": "em", "glm": "em", "bulk": "p", "pressure": "p", "energy_density": "p"}
    group.update({n: "p" for n in OUT.FIELDS[9:19]})
    scale = {}
    for name in fo:
        key = group.get(name, name)
        scale[key] = max(scale.get(key, 0.0), float(np.abs(fo[name]).max()))
    for name in fo:
        sc = max(scale[group.get(name, name)], 1e-300)
        assert float(np.abs(fg[name] - fo[name]).max()) <= 1e-12 * sc, name


def test_derived_data_error_is_reported():
    """A pressure below the EoS table in one cell: the reference's code of
    get_derived_data (135), for the first such cell, on both sides."""
    cfg = CASES["visc2d"]()
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    vv = v0.reshape(cfg.nv, -1).copy()
    vv[4, 5] = 0.5 * tab[0, 2]
    vv[4, 9] = 0.5 * tab[0, 2]
    o.set_state(vv.reshape(-1), u0, cfg.tstart)
    g = Evolve(pc, tab, exact=True)
    g.upload(vv.reshape(-1), u0, cfg.tstart)
    sel = OUT.mask("temperature")
    bo, eo = o.out_vars(sel)
    bg, eg = g.out_vars(sel)
    assert eo == eg == 135
    assert bo == bg
