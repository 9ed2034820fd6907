"""The learned con2prim seed on the resistive equations (MHD = 2): six
invariants (E^2/U the sixth), pairs from resistive runs, and seeded
IMEX-SSP steps against the oracle's plain (warm-started) inversion.

Tolerances: the seed only moves where the fixed point starts, so the
seeded steps meet the plain path's product-build bar, 1e-12 relative L-inf
per field group (rho; v; p; B, E and psi together); seed accuracy as in the
ideal-RMHD tests (median |dv^2| < 0.02, median |d(p/U)|/(p/U) < 0.1).
"""
import numpy as np
import pytest

import pyoracle as O
from echo_gpu import params as P
from echo_gpu import seed as S
from echo_gpu.lib import Evolve
from helpers import CASES, RES_GROUPS, przero_of, rel_linf, resistive_state, setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    X, T = S.generate_pairs(n_target=150_000, grid=20, steps=6, every=3, resistive=True)
    w, norm, losses = S.train(X, T, steps=1500, batch=4096, lr=3e-3, report_every=100)
    return X, T, w, norm, losses


def test_pairs_carry_the_electric_field(trained):
    X, T, _, norm, losses = trained
    assert X.shape[1] == S.NIN and np.isfinite(X).all() and np.isfinite(T).all()
    assert (X[:, 5] > 0).mean() > 0.5  # E^2/U: nonzero wherever the fluid moves
    assert norm[S.NIN + 5] > 0
    assert losses[-1] < 0.1 * losses[0], losses


def test_seed_accuracy(trained):
    X, T, w, norm, _ = trained
    idx = np.random.default_rng(4).choice(len(X), 4000, replace=False)
    pred = S.infer(w, norm, X[idx])
    assert np.median(np.abs(pred[:, 0] - T[idx, 0])) < 0.02
    assert np.median(np.abs(pred[:, 1] / T[idx, 1] - 1)) < 0.1


@pytest.mark.parametrize("sigma", [0.0058, 500.0])
def test_seeded_steps_match_oracle(trained, sigma):
    _, _, w, norm, _ = trained
    cfg = CASES["res3d"]().replace(sigma_el=sigma)
    _, tab, _ = setup(cfg)
    pc = cfg.to_c(przero=przero_of(cfg))
    o = O.Oracle(pc, tab)
    o.set_state(resistive_state(cfg, tab), None, cfg.tstart)
    v0, u0 = o.state()
    g = Evolve(cfg.replace(algo_solver=P.C2P_MLP).to_c(przero=przero_of(cfg)), tab)
    g.set_seed_network(w, norm)
    g.upload(v0, u0, cfg.tstart)
    for _ in range(5):
        o.step()
        g.step()
    st = g.stats()
    assert st.errcode == 0
    vg, ug = g.download()
    vo, uo = o.state()
    ev, eu = rel_linf(vg, vo, 12, RES_GROUPS), rel_linf(ug, uo, 12, RES_GROUPS)
    assert ev <= 1e-12 and eu <= 1e-12, (ev, eu)
    # the seed was used: fallbacks are counted, and not every cell fell back
    assert 0 <= st.seed_fallbacks < 5 * 5 * cfg.ncell


def test_seeded_run_without_network_is_refused():
    cfg = CASES["res3d"]().replace(algo_solver=P.C2P_MLP)
    _, tab, _ = setup(cfg)
    g = Evolve(cfg.to_c(przero=przero_of(cfg)), tab)
    g.upload(resistive_state(cfg, tab), None, cfg.tstart)
    with pytest.raises(RuntimeError):
        g.run(1)
