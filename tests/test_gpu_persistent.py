"""The persistent FP32 stage kernel and the schedule autotuner: on a conforming mesh the persistent
kernel (any number of CTAs, tasks from the device queue) reproduces the one-CTA-per-tile kernel bit
for bit; on a 2:1 forest, where it also runs the mortar pairs as its first tasks, it agrees with the
mortar kernel + grid schedule to FP32 round-off; the autotuner leaves the state as it found it."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


def run_with(m, u, schedule, nsteps=5, groups=None, ind=abi.IND_MODAL):
    s = Solver(abi.default_cfg(precision=abi.PREC_FP32, indicator=ind, positivity=1), m, groups)
    if schedule is not None:
        s.set_schedule(*schedule)
    s.upload(u)
    t, n = s.run(nsteps=nsteps)
    out = s.download()
    s.finalize()
    return out, t


@pytest.mark.parametrize("ctas", [1, 5, 148, 296])
def test_persistent_equals_grid_conforming(ctas):
    m = mesh.brick(6)
    u = setups.smooth_random(m, seed=4)
    ref, tr = run_with(m, u, (0, 0))
    got, tg = run_with(m, u, (1, ctas))
    assert tg == tr
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("ctas", [1, 148, 296])
def test_persistent_forest_with_fused_mortars(ctas):
    f = mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)
    b = mesh.brick(4)
    m, g = mesh.concat([f, b, b])
    u = np.concatenate([setups.smooth_random(f, seed=1), setups.gaussian_blob(b, 0.3), setups.gaussian_blob(b, 0.9)],
                       axis=1)
    ref, _ = run_with(m, u, (0, 0), groups=g)
    got, _ = run_with(m, u, (1, ctas), groups=g)
    scale = np.max(np.abs(ref), axis=(1, 2), keepdims=True)
    assert np.max(np.abs(got - ref) / scale) < 1e-6
    # and both against the FP64 oracle of the forest group
    oref, _, _, _ = orc.Oracle.for_mesh(abi.default_cfg(indicator=abi.IND_MODAL, positivity=1), f).run(
        u[:, : f.E], nsteps=5)
    assert np.sum(np.abs(got[0, : f.E] - oref[0])) / np.sum(np.abs(oref[0])) < 1e-6


def test_autotune_keeps_state_and_picks_a_schedule():
    m = mesh.brick(8)
    u = setups.smooth_random(m, seed=8)
    s = Solver(abi.default_cfg(precision=abi.PREC_FP32, indicator=abi.IND_MODAL, positivity=1), m)
    s.upload(u)
    mode, ctas, ms = s.autotune(nsteps=2)
    assert mode in (0, 1, 2, 3) and (mode != 1 or ctas >= 148)
    assert np.all(ms[:2] > 0) and ms[5] > 0 and ms[6] > 0 and ms[7] == -1.0
    assert np.array_equal(s.download(), u)
    assert s.status()[0] == 0.0
    t, n = s.run(nsteps=3)
    got = s.download()
    s.finalize()
    # the same schedule set by hand from a fresh upload (FP32 results depend on the tile size, which
    # decides which neighbour traces come from the tile and which from global memory)
    ref, tr = run_with(m, u, (mode, ctas), nsteps=3)
    assert t == tr and np.array_equal(got, ref)


@pytest.mark.parametrize("mode", [2, 3])
def test_grid_tile_sizes_agree_with_the_default_tile(mode):
    """The grid schedule with 4 or 16 elements per CTA agrees with 8 elements per CTA to FP32 rounding:
    a neighbour inside the CTA's tile is read from the tile's FP32 primitives, one outside from the
    FP64 state in L2 (the same quantities, rounded differently), and each tile size is its own
    instantiation of the FP32 kernel; each schedule is reproducible run to run."""
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    ref, tr = run_with(m, u, (0, 0), nsteps=4)
    got, t = run_with(m, u, (mode, 0), nsteps=4)
    again, t2 = run_with(m, u, (mode, 0), nsteps=4)
    assert np.array_equal(got, again) and t == t2
    assert abs(t - tr) <= 1e-6 * tr
    scale = np.max(np.abs(ref), axis=(1, 2), keepdims=True)
    assert np.max(np.abs(got - ref) / scale) < 1e-5
    assert np.sum(np.abs(got[0] - ref[0])) / np.sum(np.abs(ref[0])) < 1e-7
