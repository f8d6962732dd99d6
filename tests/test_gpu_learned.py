"""GPU tests of the learned shock indicator: training kernels against the FP64 numpy oracle,
features against the C++ oracle, the learned indicator inside both stage forms, and what the
trained network gains over the untrained one."""
import ctypes
import os

import numpy as np
import pytest

from nemo_b200 import abi, learned, mesh, setups
from nemo_b200.solver import Solver
from oracle import mlp_oracle
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


def grad_gpu(feat, tgt, w):
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    tgt = np.ascontiguousarray(tgt, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    g = np.zeros(learned.MLP_NW, dtype=np.float32)
    abi.call("nemo_gpu_mlp_grad", abi.ptr(feat), abi.ptr(tgt), len(tgt), abi.ptr(w), ctypes.c_float(0.5),
             abi.ptr(loss), abi.ptr(g))
    return float(loss[0]), g


def test_training_gradient_matches_cpu_oracle():
    rng = np.random.default_rng(0)
    w = learned.init_weights(3) + rng.normal(scale=0.05, size=learned.MLP_NW).astype(np.float32)
    feat = rng.uniform(-27, 0, size=(3000, 12)).astype(np.float32)
    tgt = rng.uniform(0, 0.5, size=3000).astype(np.float32)
    L, g = grad_gpu(feat, tgt, w)
    Lr, gr = mlp_oracle.loss_and_grad(feat.astype(np.float64), tgt.astype(np.float64), w.astype(np.float64))
    assert abs(L - Lr) <= 1e-5 * Lr
    assert np.max(np.abs(g - gr)) <= 2e-4 * np.max(np.abs(gr))
    out = learned.forward(feat, w)
    assert np.max(np.abs(out - mlp_oracle.forward(feat, w))) < 2e-6


def test_features_match_oracle():
    m = mesh.brick(8)
    rng = np.random.default_rng(3)
    u = learned.random_problem(m, rng)
    c = abi.default_cfg(precision=abi.PREC_FP32, indicator=abi.IND_MODAL)
    s = Solver(c, m)
    s.upload(u)
    f = np.empty((m.E, 12), dtype=np.float32)
    a = np.empty(m.E)
    abi.call("nemo_gpu_features", abi.ptr(f), abi.ptr(a))
    fr, ar = orc.features(c, u)
    big = fr > -20                         # FP32 cannot resolve energy shares below ~1e-9
    assert np.max(np.abs(f[big] - fr[big])) < 2e-3
    assert np.mean(np.abs(a - ar)) < 1e-3


def _small_dataset():
    feat, alpha = learned.generate_dataset(nproblems=12, nx=8, steps=(0, 3), seed=5)
    return feat, alpha


def test_training_reduces_loss_and_beats_untrained():
    feat, alpha = _small_dataset()
    n = len(alpha)
    tr, te = slice(0, int(0.8 * n)), slice(int(0.8 * n), n)
    w0 = learned.init_weights(11)
    w, loss = learned.train(feat[tr], alpha[tr], epochs=25, batch=1024, lr=3e-3, seed=11, w0=w0)
    assert loss[-1] < 0.2 * loss[0]
    mae_tr = np.mean(np.abs(learned.forward(feat[te], w) - alpha[te]))
    mae_un = np.mean(np.abs(learned.forward(feat[te], w0) - alpha[te]))
    assert mae_tr < 0.5 * mae_un, (mae_tr, mae_un)


def _trained():
    if not os.path.exists(learned.WEIGHTS):
        pytest.skip("trained weights file not present")
    return learned.load()


def test_plain_path_learned_indicator_bit_exact_with_oracle():
    """Plain FP64 path with the learned indicator: alpha, rhs and a short blended run equal the oracle
    evaluating the same BF16-rounded network in FP64."""
    w, lo, hi, _ = _trained()
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    c = abi.default_cfg(indicator=abi.IND_LEARNED, positivity=1)
    s = Solver(c, m)
    learned.install()
    wb = (np.asarray(w, dtype=np.float32).view(np.uint32) + 0x7fff + ((np.asarray(w, np.float32).view(np.uint32) >> 16) & 1))
    wb = (wb & 0xffff0000).astype(np.uint32).view(np.float32).astype(np.float64)
    orc.set_mlp(wb, lo.astype(np.float64), hi.astype(np.float64))
    o = orc.Oracle(c, m.neighbors(), m.delta)
    s.upload(u)
    a_gpu, a_cpu = s.alpha(), o.alpha(u)
    assert np.array_equal(a_gpu, a_cpu)
    assert np.array_equal(s.rhs(), o.rhs(u, alpha=a_cpu))
    t, n = s.run(t_end=1e-3)
    uc, tc, nc, _ = o.run(u, t_end=1e-3)
    assert n == nc and np.array_equal(s.download(), uc)


def test_fp32_learned_close_to_fp64_learned_and_judged():
    _trained()
    m = mesh.brick(16, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP32):
        c = abi.default_cfg(precision=prec, indicator=abi.IND_LEARNED, positivity=1)
        s = Solver(c, m)
        learned.install()
        s.upload(u)
        s.run(t_end=0.01)
        fb, jn, mae = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        abi.call("nemo_gpu_indicator_stats", ctypes.byref(fb), ctypes.byref(jn), ctypes.byref(mae))
        out[prec] = (s.download(), fb.value, jn.value, mae.value)
        s.finalize()
    r64, r32 = out[abi.PREC_FP64][0][0], out[abi.PREC_FP32][0][0]
    assert np.sum(np.abs(r32 - r64)) / np.sum(np.abs(r64)) < 1e-6
    for prec in out:
        fb, jn, mae = out[prec][1:]
        assert jn > 0 and mae < 0.05      # the judge: mean |alpha_learned - alpha_modal|


def _element_means(u0, w):
    """Element means of a nodal field [E][64] (node = i + 4 j + 16 k) with the LGL weights w."""
    w3 = np.einsum("k,j,i->kji", w, w, w).reshape(64) / 8.0
    return u0 @ w3


def test_learned_vs_modal_indicator_against_a_fine_grid_solution():
    """What the learned indicator gains over the method without it (the modal indicator it was trained
    to imitate): both run the Sedov blast on 16^3 elements to t = 0.05 in the plain FP64 form, and their
    element-mean densities are compared with the mean densities of a 32^3 modal run over the same
    cells.  The numbers are printed (relative L1 error 1.4313e-2 modal, 1.4287e-2 learned on B200); the
    bound only says the learned run is not grossly worse.  It has no accuracy gain by construction -- its target is the modal alpha -- and
    it is not cheaper (its features need two modal transforms where the modal indicator needs one)."""
    _trained()
    lo, hi = (-0.5,) * 3, (0.5,) * 3
    _, w, _, _, _ = abi.operators()
    fine = mesh.brick(32, lo=lo, hi=hi)
    coarse = mesh.brick(16, lo=lo, hi=hi)
    res = {}
    for key, m, ind in (("fine_modal", fine, abi.IND_MODAL), ("modal", coarse, abi.IND_MODAL),
                        ("learned", coarse, abi.IND_LEARNED)):
        c = abi.default_cfg(indicator=ind, positivity=1, cfl=0.5)
        s = Solver(c, m)
        if ind == abi.IND_LEARNED:
            learned.install()
        s.upload(setups.sedov(m, sigma=0.05))
        t, n = s.run(t_end=0.05)
        assert abs(t - 0.05) < 1e-12 and s.status()[1] == 0
        res[key] = _element_means(s.download()[0], w)
        s.finalize()
    # the fine cells of each coarse element (both meshes are uniform bricks on the same box)
    cidx = np.floor((coarse.center - np.asarray(lo)) / (1.0 / 16)).astype(int)
    fidx = np.floor((fine.center - np.asarray(lo)) / (1.0 / 16)).astype(int)
    ckey = (cidx[:, 0] * 16 + cidx[:, 1]) * 16 + cidx[:, 2]
    fkey = (fidx[:, 0] * 16 + fidx[:, 1]) * 16 + fidx[:, 2]
    ref = np.zeros(16 ** 3)
    np.add.at(ref, fkey, res["fine_modal"] / 8.0)
    ref = ref[ckey]
    err = {k: float(np.sum(np.abs(res[k] - ref)) / np.sum(np.abs(ref))) for k in ("modal", "learned")}
    diff = float(np.sum(np.abs(res["learned"] - res["modal"])) / np.sum(np.abs(res["modal"])))
    print(f"rel. L1 error of element-mean density vs the 32^3 solution: modal {err['modal']:.4e}, "
          f"learned {err['learned']:.4e} (learned/modal {err['learned'] / err['modal']:.3f}); "
          f"learned vs modal {diff:.3e}")
    assert 0.0 < err["modal"] < 1.0 and 0.0 < err["learned"] < 1.0
    assert err["learned"] < 1.5 * err["modal"]
