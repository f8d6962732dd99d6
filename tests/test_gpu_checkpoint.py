"""GPU checkpoints: the asynchronous snapshot holds the state, time and step count of the moment it
was taken while later steps run, and a restart from the file continues bit for bit as the
uninterrupted run does (plain FP64 path, a forest with mortars and a blast)."""
import numpy as np
import pytest

from nemo_b200 import abi, checkpoint, mesh, setups
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


def blast_forest():
    m = mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)
    x, y, z = m.node_coords(orc.lgl(3)[0])
    u = setups.smooth_random(m, seed=2)
    u[4] += 5.0 * np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) / 0.01)
    return m, u


def test_async_checkpoint_and_restart(tmp_path):
    m, u = blast_forest()
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    t3, _ = s.run(nsteps=3)
    u3 = s.download()
    ck = checkpoint.Checkpointer(s, directory=str(tmp_path))
    ck.begin()
    t5, _ = s.run(nsteps=2)             # runs while the snapshot is copied
    path, tc, nc = ck.finish()
    assert tc == t3 and nc == 3
    m2, u2, t, steps = checkpoint.read(path)
    assert np.array_equal(u2, u3) and t == t3 and steps == 3
    assert path.endswith(".f5")        # the reference's checkpoint name; an HDF5 file
    z = checkpoint.load_datasets(path)
    blnd = z["blnd"][z["node type"] == 1][:, 0, 0, 0]
    assert blnd.max() > 0.0 and blnd.max() <= c.alpha_max
    t8, _ = s.run(nsteps=3)
    u8 = s.download()
    s.finalize()
    r = checkpoint.restart(c, path)
    assert r.status()[0] == t3
    tr, _ = r.run(nsteps=5)
    assert tr == t8
    assert np.array_equal(r.download(), u8)


def test_checkpoint_after_adapt(tmp_path):
    m, u = blast_forest()
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    s.run(nsteps=2)
    f = np.where(m.center[:, 0] < 0.3, 1, np.where(m.center[:, 0] > 0.6, -1, 0))
    new, _ = s.adapt(f)
    ck = checkpoint.Checkpointer(s, directory=str(tmp_path))
    ck.begin()
    path, t, n = ck.finish()
    m2, u2, t2, n2 = checkpoint.read(path)
    assert m2.E == new.E and np.array_equal(m2.center, new.center)
    assert np.array_equal(u2, s.download()) and t2 == t and n2 == n == 2
