"""Output files in the reference's layout (out_vars, out.f90:232-591), on the
oracle: the bytes of one outNNNN.dat against the state they are made of."""
import os

import numpy as np

import pyoracle as O
from echo_gpu import output as OUT
from echo_gpu import params as P
from helpers import CASES, setup


def _oracle(case, steps=0, **kw):
    cfg = CASES[case]().replace(**kw)
    pc, tab, v = setup(cfg)
    o = O.Oracle(pc, tab)
    o.set_state(v, None, cfg.tstart)
    for _ in range(steps):
        o.step()
    return cfg, o


def test_header_order_and_fields_hd():
    cfg, o = _oracle("hd2d", steps=2)
    sel = OUT.DEFAULT | OUT.mask("v0", "temperature", "bulk", "bx")
    blob, err = o.out_vars(sel)
    assert err == 0
    t, f = OUT.read(blob, cfg, sel)
    assert t == o.t
    assert list(f) == ["density", "vx", "vy", "vz", "pressure", "energy_density", "temperature", "v0"]
    v = o.state()[0].reshape(cfg.nv, cfg.nz, cfg.ny, cfg.nx)
    for k, name in enumerate(["density", "vx", "vy", "vz", "pressure"]):
        assert np.array_equal(f[name], v[k])
    assert np.array_equal(f["energy_density"], 3.0 * v[4])  # p = e/3
    g3 = 1.0 if cfg.coordinates == P.MINKOWSKI else o.t**2
    gam = 1.0 / np.sqrt(1.0 - v[1] * v[1] - v[2] * v[2] - v[3] * v[3] * g3)
    assert np.allclose(f["v0"], gam, rtol=1e-15, atol=0)


def test_single_precision_is_the_rounded_double():
    cfg, o = _oracle("visc2d", steps=1)
    sel = OUT.DEFAULT | OUT.mask(*OUT.FIELDS[8:20])
    b8, _ = o.out_vars(sel, 8)
    b4, _ = o.out_vars(sel, 4)
    a8 = np.frombuffer(b8, np.float64)
    a4 = np.frombuffer(b4, np.float32)
    assert np.array_equal(a8.astype(np.float32), a4)
    t, f = OUT.read(b8, cfg, sel)
    assert len(f) == len(OUT.written(cfg, sel)) and "bx" not in f and "pitt" in f
    v = o.state()[0].reshape(cfg.nv, cfg.nz, cfg.ny, cfg.nx)
    assert np.array_equal(f["pixy"], v[6]) and np.array_equal(f["bulk"], v[5])


def test_ideal_mhd_electric_field():
    cfg, o = _oracle("rmhd3d", steps=1)
    sel = OUT.mask("ex", "ey", "ez", "glm", "bx", "by", "bz")
    blob, err = o.out_vars(sel)
    t, f = OUT.read(blob, cfg, sel)
    v = o.state()[0].reshape(cfg.nv, cfg.nz, cfg.ny, cfg.nx)
    vx, vy, vz, bx, by, bz = v[1], v[2], v[3], v[5], v[6], v[7]
    gp = t
    ex = -gp * (vy * bz - vz * by)
    ey = -gp * (vz * bx - vx * bz)
    ez = -gp * (vx * by - vy * bx) / (gp * gp)
    assert np.array_equal(f["ex"], ex) and np.array_equal(f["ey"], ey)
    assert np.allclose(f["ez"], ez, rtol=1e-15, atol=0)
    assert np.array_equal(f["glm"], v[8])


def test_files_named_as_the_reference(tmp_path):
    cfg, o = _oracle("hd2d")
    blob, _ = o.out_vars(OUT.DEFAULT)
    p0 = OUT.write(str(tmp_path), 1, 0, blob, o.t, append_time=False)
    OUT.write(str(tmp_path), 1, 1, blob, o.t + 0.1, append_time=True)
    assert p0.endswith(os.path.join("outr0001", "out0000.dat"))
    with open(tmp_path / "outr0001" / "time.dat") as f:
        assert f.read() == "    0     0.400000000\n    1     0.500000000\n"
    with open(p0, "rb") as f:
        assert f.read() == blob
