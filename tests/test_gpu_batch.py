"""The batched uneven workload on the GPU: a 2:1 forest and an ensemble of independent periodic
bricks in one element list, one group each (own time step and time), advanced by the CUDA-graph
run loop.  Every group must reproduce the oracle run of its own mesh alone, bit for bit on the
plain FP64 path; the FP32 form stays within FP32 tolerances."""
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


def parts(members=4):
    f = mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)
    b = mesh.brick(4)
    amps = np.linspace(0.1, 1.0, members)
    uf = setups.smooth_random(f, seed=9)
    ub = [setups.gaussian_blob(b, a) for a in amps]
    m, g = mesh.concat([f] + [b] * members)
    u = np.concatenate([uf] + ub, axis=1)
    return m, g, f, b, uf, ub


@pytest.mark.parametrize("ind", [abi.IND_NONE, abi.IND_MODAL])
def test_batch_groups_match_oracle_alone(ind):
    m, g, f, b, uf, ub = parts()
    c = abi.default_cfg(indicator=ind, positivity=1)
    s = Solver(c, m, g)
    s.upload(np.concatenate([uf] + ub, axis=1))
    s.run(nsteps=6)
    got = s.download()
    ref_f, _, _, _ = orc.Oracle.for_mesh(c, f).run(uf, nsteps=6)
    assert np.array_equal(got[:, : f.E], ref_f)
    for i, ui in enumerate(ub):
        ref, _, _, _ = orc.Oracle.for_mesh(c, b).run(ui, nsteps=6)
        lo = f.E + i * b.E
        assert np.array_equal(got[:, lo: lo + b.E], ref), i


def test_batch_to_t_end_per_group_clamp():
    """Groups reach t_end with their own number of steps; the run ends when all have."""
    m, g, f, b, uf, ub = parts(members=3)
    c = abi.default_cfg()
    s = Solver(c, m, g)
    s.upload(np.concatenate([uf] + ub, axis=1))
    t_end = 0.02
    t, n = s.run(t_end=t_end)
    got = s.download()
    for i, ui in enumerate(ub):
        ref, tr, nr, _ = orc.Oracle.for_mesh(c, b).run(ui, t_end=t_end)
        assert tr == t_end and nr <= n
        lo = f.E + i * b.E
        assert np.array_equal(got[:, lo: lo + b.E], ref), i
    ref_f, tf, nf, _ = orc.Oracle.for_mesh(c, f).run(uf, t_end=t_end)
    assert np.array_equal(got[:, : f.E], ref_f)


def test_batch_fp32_form_close():
    m, g, f, b, uf, ub = parts()
    u = np.concatenate([uf] + ub, axis=1)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP32):
        s = Solver(abi.default_cfg(precision=prec, indicator=abi.IND_MODAL, positivity=1), m, g)
        s.upload(u)
        s.run(nsteps=10)
        out[prec] = s.download()
        s.finalize()
    d = np.sum(np.abs(out[1][0] - out[0][0])) / np.sum(np.abs(out[0][0]))
    assert d < 1e-6, d
