"""CUDA step vs the CPU oracle on the same seeded inputs.

Tolerances (relative L-inf per variable, see helpers.rel_linf):
  exact build (--fmad=false): 1e-13 -- the arithmetic is the oracle's
      operation for operation; the only admitted differences come from
      exp()/pow() of the CUDA math library vs libm in the last place.
  product build (--fmad=true): 1e-12 after the stated number of steps --
      the agreement the reference's own parity requirement states.
"""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu.lib import Evolve, unit_c2p, unit_recon
from helpers import CASES, gubser_case, rel_linf, resistive_state, setup

pytestmark = pytest.mark.gpu


def _corrupt_centre(cfg, u0):
    """|S^x| = 2 E in the centre cell: its inversion fails in the first stage
    and the neighbour-average repair (evolve.f90:795-842) takes over."""
    u = u0.reshape(cfg.nv, -1).copy()
    c = (cfg.nz // 2) * cfg.nx * cfg.ny + (cfg.ny // 2) * cfg.nx + cfg.nx // 2
    u[1, c] = 2.0 * u[4, c]
    return u.reshape(-1)


def _pair(cfg, steps, exact=True, use_run=False, prep=None):
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    if prep is not None:
        u0 = prep(cfg, u0)
        o.set_state(v0, u0, cfg.tstart)
    g = Evolve(pc, tab, exact=exact)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(steps):
        o.step()
    if use_run:
        g.run(steps)
        g.sync()
    else:
        for _ in range(steps):
            g.step()
    vo, uo = o.state()
    vg, ug = g.download()
    st = g.stats()
    assert st.errcode == 0
    assert abs(st.t - o.t) <= 1e-14 * o.t
    return rel_linf(vg, vo, o.nv), rel_linf(ug, uo, o.nv), o, g


@pytest.mark.parametrize("case,steps", [("hd2d", 20), ("rmhd3d", 6), ("visc2d", 8)])
def test_step_parity_exact(case, steps):
    ev, eu, o, g = _pair(CASES[case](), steps, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)


@pytest.mark.parametrize("case,steps", [("hd2d", 20), ("rmhd3d", 6), ("visc2d", 8)])
def test_step_parity_fast(case, steps):
    ev, eu, o, g = _pair(CASES[case](), steps, exact=False)
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)


@pytest.mark.parametrize("rec", list(P.REC))
def test_reconstructions_in_step(rec):
    cfg = CASES["hd2d"]().replace(recal=rec)
    ev, eu, _, _ = _pair(cfg, 5, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13, (rec, ev, eu)


@pytest.mark.parametrize("bc", [0, 1, 2, 3])
def test_boundaries(bc):
    cfg = CASES["hd2d"]().replace(boundary=bc, maxdt=0.02)
    ev, eu, _, _ = _pair(cfg, 3, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13, (bc, ev, eu)


def test_minkowski_rk3():
    cfg = CASES["hd2d"]().replace(coordinates=P.MINKOWSKI, nrk=P.RK3)
    ev, eu, _, _ = _pair(cfg, 5, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13


@pytest.mark.parametrize("case,steps", [("rmhd3d", 4), ("hd2d", 6), ("visc2d", 4)])
def test_imex_ssp_parity(case, steps):
    # IMEX-SSP3(4,3,3) (evolve.f90:204-267): the stiff terms are zero without
    # resistivity; the reference also runs it for hydro (common.f90:2076-2083)
    cfg = CASES[case]().replace(nrk=P.SSP)
    ev, eu, _, _ = _pair(cfg, steps, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)
    ev, eu, _, _ = _pair(cfg, steps, exact=False, use_run=True)
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)


@pytest.mark.parametrize("case,nrk", [("hd2d", P.RK2), ("visc2d", P.RK2), ("hd2d", P.RK3), ("hd2d", P.SSP)])
def test_repair_parity(case, nrk):
    cfg = CASES[case]().replace(nrk=nrk)
    ev, eu, o, g = _pair(cfg, 3, exact=True, prep=_corrupt_centre)
    assert o.repairs > 0 and g.stats().repairs == o.repairs, (o.repairs, g.stats().repairs)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)
    ev, eu, o, g = _pair(cfg, 3, exact=False, use_run=True, prep=_corrupt_centre)
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)


def _corrupt_cells(cells_of):
    """|S^x| = 2 E in each cell cells_of(cfg) returns."""
    def prep(cfg, u0):
        u = u0.reshape(cfg.nv, -1).copy()
        for c in cells_of(cfg):
            u[1, c] = 2.0 * u[4, c]
        return u.reshape(-1)
    return prep


def _scattered(cfg):
    # no two share a flat neighbour (c +- 1, c +- nx, c +- nx ny)
    return [iz * cfg.nx * cfg.ny + iy * cfg.nx + ix
            for iz in range(cfg.nz) for iy in range(1, cfg.ny - 1, 3) for ix in range(1, cfg.nx - 1, 3)
            if cfg.nz == 1 or iz % 2 == 1]


def _adjacent(cfg):
    c = (cfg.nz // 2) * cfg.nx * cfg.ny + (cfg.ny // 2) * cfg.nx + cfg.nx // 2
    return [c - 1, c, c + 1, c + cfg.nx]


REPAIR_CASES = {
    "hd2d": lambda: CASES["hd2d"](),
    "hd3d": lambda: P.small(P.config0(), 10).replace(nz=6, z1=-0.45, z2=0.45),
    "visc2d": lambda: CASES["visc2d"](),
}


@pytest.mark.parametrize("case", list(REPAIR_CASES))
@pytest.mark.parametrize("cells", [_scattered, _adjacent])
def test_repair_of_many_cells_parity(case, cells):
    """Many failed cells in one stage: scattered ones, which the repair
    kernel treats together, and neighbouring ones, which it treats one after
    another as the reference does; the same repaired state as the oracle
    either way.  (Ideal RMHD is left out as in test_repair_parity: there the
    repaired states leave the EoS table, and the reference stops with its
    range error.)"""
    cfg = REPAIR_CASES[case]()
    prep = _corrupt_cells(cells)
    ev, eu, o, g = _pair(cfg, 3, exact=True, prep=prep)
    assert o.repairs >= len(cells(cfg)) and g.stats().repairs == o.repairs, (o.repairs, g.stats().repairs)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)
    ev, eu, o, g = _pair(cfg, 3, exact=False, use_run=True, prep=prep)
    assert g.stats().repairs == o.repairs
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)


@pytest.mark.parametrize("nrk", [P.RK2, P.SSP])
def test_smoothing_parity(nrk):
    # T_cut = 0.35 GeV puts about three quarters of the cells under p_cut, so
    # evolve_smooth_viscosity (evolve.f90:1159-1207) acts after every stage
    cfg = CASES["visc2d"]().replace(smooth_temp=0.35, nrk=nrk)
    ev, eu, o, g = _pair(cfg, 6, exact=True)
    assert ev <= 1e-13 and eu <= 1e-13, (ev, eu)
    ev, eu, o, g = _pair(cfg, 6, exact=False, use_run=True)
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)


@pytest.mark.parametrize("case", ["hd2d", "rmhd3d", "visc2d"])
@pytest.mark.parametrize("exact,tol", [(True, 0.0), (False, 1e-13)])
def test_check_temp_matches_oracle(case, exact, tol):
    """check_temp (out.f90:1487-1557) on the device: the maximum temperature
    and energy density of the state after a few steps, and the stop flag."""
    ev, eu, o, g = _pair(CASES[case](), 3, exact=exact)
    for ft in (0, 1):
        mo = o.check_temp(ft)
        mg, stop = g.check_temp(ft, mo * 1.01)
        assert abs(mg - mo) <= tol * mo, (ft, mg, mo)
        assert stop
        assert not g.check_temp(ft, mo * 0.99)[1]


def test_gubser_flow_matches_oracle():
    """The reference's ideal Gubser test problem on the device: 50 steps of
    the 81x81 conformal run equal the oracle's (which converges to the
    analytic flow, tests/test_oracle.py)."""
    cfg, v, _, _ = gubser_case()
    pc = cfg.to_c(przero=cfg.enezero / 3)
    o = O.Oracle(pc, None)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    for exact, tol in ((True, 1e-13), (False, 1e-12)):
        g = Evolve(pc.__class__.from_buffer_copy(pc), None, exact=exact)
        g.upload(v0, u0, cfg.tstart)
        g.run(50)
        g.sync()
        vg, ug = g.download()
        if exact:
            for _ in range(50):
                o.step()
            vo, uo = o.state()
        assert rel_linf(vg, vo, 5) <= tol and rel_linf(ug, uo, 5) <= tol, exact


@pytest.mark.parametrize("case", ["visc2d", "rmhd3d"])
def test_eos_range_error_is_reported(case):
    """A pressure above the EoS table in one cell: the face states around it
    fall outside the table and the step fails with the reference's code
    (126, get_energy, eos.f90:468-523), on the device as on the oracle."""
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    vv = v0.reshape(cfg.nv, -1).copy()
    vv[4, cfg.ncell // 2 + cfg.nx // 2] = 1.5 * tab[-1, 2]
    o.set_state(vv.reshape(-1), u0, cfg.tstart)
    with pytest.raises(RuntimeError, match="126"):
        o.step()
    g = Evolve(pc, tab)
    g.upload(vv.reshape(-1), u0, cfg.tstart)
    g.run(1)
    g.sync()
    st = g.stats()
    assert st.errcode == 126 and st.err_cell >= 0


def test_graph_run_matches_steps():
    ev, eu, _, _ = _pair(CASES["rmhd3d"](), 4, exact=True, use_run=True)
    assert ev <= 1e-13 and eu <= 1e-13


@pytest.mark.parametrize("rec", list(P.REC))
def test_recon_kernel_bitexact(rec):
    rng = np.random.default_rng(3)
    n = 33
    f = rng.standard_normal((17, n + 8))
    f[:4] = np.cumsum(f[:4], axis=1)  # smooth rows exercise the other branches
    gl_o, gr_o = O.recon(P.REC[rec], f, n)
    gl_g, gr_g = unit_recon(P.REC[rec], f, n, exact=True)
    assert np.array_equal(gl_o, gl_g) and np.array_equal(gr_o, gr_g)


@pytest.mark.parametrize("case", ["hd2d", "rmhd3d", "visc2d"])
def test_c2p_kernel(case):
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    nv = cfg.nv
    cells = v.reshape(nv, -1).T.copy()
    t = 0.7
    g3, gp = t * t, t
    cells_p, u, bad = O.prim2cons(pc, tab, g3, gp, cells)
    assert bad == 0
    guess = cells_p * (1 + 1e-3)
    vo, eo, io = O.c2p(pc, tab, g3, gp, u, guess)
    vg, eg, ig = unit_c2p(pc, tab, g3, gp, u, guess, exact=True)
    assert np.array_equal(eo, eg)
    assert rel_linf(vg.T.copy(), vo.T.copy(), nv) <= 1e-14
    # the inversion recovers the primitives it started from
    assert rel_linf(vo.T.copy(), cells_p.T.copy(), nv) <= 1e-9


def test_rhs_parity():
    cfg = CASES["rmhd3d"]()
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(pc, tab, exact=True)
    g.upload(v0, u0, cfg.tstart)
    du_o, am_o = o.rhs()
    du_g, am_g = g.rhs()
    assert rel_linf(du_g, du_o, cfg.nv) <= 1e-13
    assert np.allclose(am_g, am_o, rtol=0, atol=0)


@pytest.mark.parametrize("case,nrk", [("rmhd3d", P.RK3), ("visc2d", P.RK2), ("res3d", P.SSP)])
def test_concurrent_sweeps_give_the_same_bits(case, nrk):
    """The three sweeps of a stage run side by side on three streams by
    default: they are independent (each writes its own face fluxes and its
    own signal-speed slots), so the run equals the one with the sweeps in
    order, bit for bit, in both builds; stepped eagerly and through the step
    graph."""
    cfg = CASES[case]().replace(nrk=nrk)
    if case == "res3d":
        cfg = cfg.replace(sigma_el=500.0)
    pc, tab, v = setup(cfg)
    if case == "res3d":
        v = resistive_state(cfg, tab)
    for exact in (True, False):
        out = []
        for concurrent in (False, True):
            g = Evolve(pc, tab, exact=exact)
            g.set_sweeps(concurrent)
            g.upload(v, None, cfg.tstart)
            g.step()
            g.run(3)
            g.sync()
            st = g.stats()
            assert st.errcode == 0
            out.append((g.download(), st.t))
            g.close()
        (v0, u0), t0 = out[0]
        (v1, u1), t1 = out[1]
        assert t0 == t1
        assert np.array_equal(v0, v1) and np.array_equal(u0, u1)
