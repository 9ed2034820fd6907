"""The CPU oracle against known answers of the reference's own test
problems (Bjorken flow; conservation on a periodic box; the con2prim
round trip) and against the committed golden vectors."""
import json
import os

import numpy as np
import pytest

import pyoracle as O
from echo_gpu import initial as I
from echo_gpu import params as P
from helpers import CASES, GOLDEN_CASES, eos_table, golden_setup, gubser, gubser_case, rel_linf, setup

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bjorken_error(dt, steps):
    cfg = P.small(P.config0(), 6).replace(maxdt=dt, cfl=10.0)
    pc = cfg.to_c(przero=cfg.enezero / 3)
    o = O.Oracle(pc)
    o.set_state(I.bjorken_uniform(cfg, 10.0), None, 0.4)
    for _ in range(steps):
        o.step()
    v, _ = o.state()
    p = v.reshape(5, -1)[4]
    exact = 10.0 / 3.0 * (0.4 / o.t) ** (4.0 / 3.0)
    assert np.ptp(p) == 0.0  # uniform stays uniform
    return abs(p[0] / exact - 1.0), o.t


def test_bjorken_flow_first_order_in_dt():
    # e(tau) = e0 (tau0/tau)^(4/3); the reference freezes the metric over a
    # step (echo.f90:211-214), so the scheme is first order in dt
    e1, t1 = _bjorken_error(0.02, 25)
    e2, t2 = _bjorken_error(0.01, 50)
    assert abs(t1 - t2) < 1e-12
    assert 1.8 < e1 / e2 < 2.2
    assert e2 < 2e-2


@pytest.mark.parametrize("rec", ["WENO5", "MPE5", "TVD2"])
def test_periodic_minkowski_conserves(rec):
    cfg = P.small(P.config0(), 16).replace(coordinates=P.MINKOWSKI, boundary=0, recal=rec, maxdt=0.05)
    pc = cfg.to_c(przero=cfg.enezero / 3)
    o = O.Oracle(pc)
    o.set_state(I.primitives(cfg), None, 0.4)
    _, u0 = o.state()
    for _ in range(10):
        o.step()
    _, u1 = o.state()
    tot0 = u0.reshape(5, -1).sum(1)
    tot1 = u1.reshape(5, -1).sum(1)
    assert np.allclose(tot0, tot1, rtol=1e-12, atol=1e-12 * np.abs(tot0).max())


@pytest.mark.parametrize("case", ["hd2d", "rmhd3d", "visc2d"])
def test_con2prim_round_trip(case):
    cfg = CASES[case]()
    pc, tab, v = setup(cfg)
    cells = v.reshape(cfg.nv, -1).T.copy()
    cells_p, u, bad = O.prim2cons(pc, tab, 0.64, 0.8, cells)
    assert bad == 0
    vr, err, it = O.c2p(pc, tab, 0.64, 0.8, u, cells_p * (1 + 1e-4))
    assert (err == 0).all()
    assert rel_linf(vr.T.copy(), cells_p.T.copy(), cfg.nv) < 1e-9


def test_eos_table_file_round_trip(tmp_path):
    tab = I.crossover_eos()
    path = tmp_path / "eos.dat"
    I.write_eos_file(str(path), tab)
    back = I.read_eos_file(str(path))
    assert np.allclose(back, tab, rtol=1e-14)
    assert (np.diff(back[:, 2]) > 0).all() and (np.diff(back[:, 0]) > 0).all()


@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_golden_vectors(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixture missing")
    g = np.load(path)
    meta = json.loads(str(g["meta"]))
    cfg, pc, tab, v, steps = golden_setup(name)
    assert steps == meta["steps"]
    assert np.array_equal(v, g["v0"])
    o = O.Oracle(pc, tab)
    o.set_state(g["v0"], None, cfg.tstart)
    for _ in range(meta["steps"]):
        o.step()
    vv, uu = o.state()
    assert np.array_equal(vv, g["v"]) and np.array_equal(uu, g["u"])
    assert o.t == meta["t"]


def test_mlp_oracle_gradient_by_finite_differences():
    # pins the FP64 network gradient the GPU training kernels are checked against
    rng = np.random.default_rng(2)
    w = (rng.standard_normal(13058) * 0.2).astype(np.float32)
    X = rng.standard_normal((16, 6)).astype(np.float32)
    T = rng.standard_normal((16, 2)).astype(np.float32)
    _, g = O.mlp_grad(w, X, T)
    for i in [0, 100, 330, 383, 400, 5000, 9000, 12929, 13057]:
        h = 2e-3 * max(1.0, abs(float(w[i])))
        wp = w.astype(np.float64).copy()
        wm = w.astype(np.float64).copy()
        wp[i] += h
        wm[i] -= h
        # weights are float32 in the interface: use steps exactly representable
        wp32, wm32 = wp.astype(np.float32), wm.astype(np.float32)
        lp, _ = O.mlp_grad(wp32, X, T)
        lm, _ = O.mlp_grad(wm32, X, T)
        fd = (lp - lm) / (float(wp32[i]) - float(wm32[i]))
        assert abs(fd - g[i]) <= 2e-3 * max(1e-3, abs(g[i])), (i, fd, g[i])


def test_check_temp_known_answers():
    """check_temp (out.f90:1487-1557): on a uniform state the maximum energy
    density is the state's e, and with p = e/3 the temperature is
    0.148909 e^(1/4) (temperature.def); on the table the maximum is that of
    the hottest cell."""
    cfg = P.small(P.config0(), 6)
    o = O.Oracle(cfg.to_c(przero=cfg.enezero / 3))
    o.set_state(I.bjorken_uniform(cfg, 12.0), None, 0.4)
    assert abs(o.check_temp(1) - 12.0) <= 1e-14 * 12.0
    assert abs(o.check_temp(0) - 0.148909 * 12.0 ** 0.25) <= 1e-14
    cfg = CASES["visc2d"]()
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    p = v.reshape(cfg.nv, -1)[4]
    e_of_p = np.interp(p, tab[:, 2], tab[:, 1])
    T_of_p = np.interp(p, tab[:, 2], tab[:, 0])
    assert abs(o.check_temp(1) / e_of_p.max() - 1) < 1e-12
    assert abs(o.check_temp(0) / T_of_p.max() - 1) < 1e-12


def _gubser_error(dt, tau1=1.5):
    cfg, v, X, Y = gubser_case(dt=dt)
    o = O.Oracle(cfg.to_c(przero=cfg.enezero / 3), None, threads=4)
    o.set_state(v, None, cfg.tstart)
    o.set_tout(tau1, 1e300, 1e300)
    while o.t < tau1 - 1e-12:
        o.step()
    p = o.state()[0].reshape(5, cfg.ny, cfg.nx)[4]
    T = 0.148909 * (3.0 * p) ** 0.25
    Ta, _ = gubser(o.t, X, Y)
    inner = np.sqrt(X * X + Y * Y) < 2.0  # away from the outflow boundaries
    return float(np.max(np.abs(T[inner] / Ta[inner] - 1)))


def test_gubser_flow_converges_first_order_in_dt():
    """Ideal Gubser flow, the reference's own analytic test (init.f90:
    2901-2961): the temperature at tau = 1.5 approaches the analytic one at
    first order in dt, the order of the reference's step (the metric is
    frozen over a step, echo.f90:211-214)."""
    e1 = _gubser_error(0.02)
    e2 = _gubser_error(0.01)
    e3 = _gubser_error(0.005)
    assert e3 < 1e-3
    assert 1.7 < e1 / e2 < 2.4 and 1.7 < e2 / e3 < 2.4, (e1, e2, e3)


def _bjorken_mhd_error(dt, steps):
    cfg = P.small(P.config1(), 6, nz=6).replace(maxdt=dt, cfl=10.0, eqstate=P.EOS_CONFORMAL,
                                                algo_solver=P.C2P_BRENT, enezero=1e-6)
    o = O.Oracle(cfg.to_c(przero=cfg.enezero / 3))
    v = np.zeros((cfg.nv, cfg.ncell))
    v[0], v[4], v[6] = 1.0, 10.0 / 3.0, 1.0  # rho, p = e/3 with e = 10, B^y = 1
    o.set_state(v.reshape(-1), None, 0.4)
    for _ in range(steps):
        o.step()
    vv = o.state()[0].reshape(cfg.nv, -1)
    assert np.ptp(vv[4]) == 0.0 and np.abs(vv[1:4]).max() == 0.0  # uniform and at rest
    e_err = vv[4, 0] * 3 / (10.0 * (0.4 / o.t) ** (4.0 / 3.0)) - 1
    b_err = vv[6, 0] * o.t / 0.4 - 1
    return abs(e_err), abs(b_err)


def test_bjorken_mhd_flow_first_order_in_dt():
    """1-D Bjorken MHD flow (the reference's Bjorken-MHD test, init.f90:
    2454-2499): with a transverse field, e ~ tau^(-4/3) and B ~ 1/tau, both
    reached at first order in dt by the frozen-metric step."""
    e1, b1 = _bjorken_mhd_error(0.02, 25)
    e2, b2 = _bjorken_mhd_error(0.01, 50)
    assert 1.8 < e1 / e2 < 2.2 and 1.8 < b1 / b2 < 2.2, (e1, e2, b1, b2)
    assert e2 < 1e-2 and b2 < 1.5e-2
