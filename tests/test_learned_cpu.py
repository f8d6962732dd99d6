"""CPU tests of the learned indicator's checkers: the numpy network gradient against finite
differences, the C++ oracle's FP64 network against numpy, and the oracle's features."""
import numpy as np
import pytest

from nemo_b200 import abi, learned, mesh, setups
from oracle import mlp_oracle
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def test_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = learned.init_weights(3).astype(np.float64) + rng.normal(scale=0.05, size=mlp_oracle.NW)
    feat = rng.uniform(-27, 0, size=(64, 12))
    tgt = rng.uniform(0, 0.5, size=64)
    L, g = mlp_oracle.loss_and_grad(feat, tgt, w)
    for k in rng.choice(mlp_oracle.NW, size=40, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (mlp_oracle.loss_and_grad(feat, tgt, wp)[0] - mlp_oracle.loss_and_grad(feat, tgt, wm)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-9, (k, fd, g[k])


def test_oracle_network_matches_numpy_and_bounds():
    rng = np.random.default_rng(1)
    w = learned.init_weights(5).astype(np.float64)
    c = abi.default_cfg(indicator=abi.IND_LEARNED)
    lo, hi = np.full(12, -5.0), np.full(12, 5.0)
    orc.set_mlp(w, lo, hi)
    for _ in range(20):
        f = rng.uniform(-27, 0, size=12)
        ref = mlp_oracle.forward(f[None], w)[0]
        ref = 0.0 if ref < 0.001 else ref
        assert abs(orc.mlp_alpha(c, f) - ref) < 1e-14
    orc.set_mlp(w, np.full(12, 0.5), hi)            # inputs below the lower bound -> fallback
    assert orc.mlp_alpha(c, np.full(12, -20.0)) == -1.0


def test_oracle_features_of_simple_states():
    m = mesh.brick(2)
    const = np.broadcast_to(setups.prim2cons(1.3, 0.1, 0.2, 0.3, 0.9, 1.4)[:, None, None], (5, m.E, 64)).copy()
    f, a = orc.features(abi.default_cfg(), const)
    assert np.allclose(f, np.log(1e-12), atol=1e-6) and np.all(a == 0)
    # a density with content only in the highest x-mode: the (rho, x, N) feature is log(share) ~ max
    u = setups.smooth_random(m, seed=4)
    f, a = orc.features(abi.default_cfg(), u)
    assert np.all(f <= 0) and np.all(np.isfinite(f))


def test_weights_file_roundtrip(tmp_path):
    w = learned.init_weights(1)
    lo, hi = learned.input_bounds(np.random.default_rng(0).uniform(-27, 0, size=(100, 12)))
    p = tmp_path / "w.json"
    learned.save(w, lo, hi, {"x": 1}, str(p))
    w2, lo2, hi2, meta = learned.load(str(p))
    assert np.array_equal(w, w2) and np.array_equal(lo, lo2) and meta["x"] == 1
    assert len(w) == learned.MLP_NW == mlp_oracle.NW
