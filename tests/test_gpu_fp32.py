"""GPU tests of the FP32-bulk form (FP32 fluxes, FP64 state/register/update/repair/reductions)
against the FP64 oracle and the bit-exact plain path.

Tolerances: the rhs agrees with the FP64 oracle to 2e-5 relative L-infinity (FP32 arithmetic and
approximate intrinsics, amplified by the 2/dx lift of nearly cancelling fluxes); the density after
a blended Sedov run to t_end agrees with the FP64 result to 1e-6 relative L1 (the accuracy target
of the chosen form).
"""
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


def rel_linf(a, b):
    return max(np.max(np.abs(a[v] - b[v])) / np.max(np.abs(b[v])) for v in range(a.shape[0]))


def rel_l1(a, b):
    return np.sum(np.abs(a - b)) / np.sum(np.abs(b))


@pytest.mark.parametrize("vf,sf", [(0, 0), (1, 1)])
def test_fp32_rhs_close_to_oracle(vf, sf):
    m = mesh.brick(4)
    u = setups.smooth_random(m, seed=11)
    c = abi.default_cfg(precision=abi.PREC_FP32, volume_flux=vf, surface_flux=sf)
    s = Solver(c, m)
    s.upload(u)
    r = s.rhs()
    ref = orc.Oracle(c, m.neighbors(), m.delta).rhs(u)
    assert rel_linf(r, ref) < 2e-5


def test_fp32_blended_sedov_rhs():
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    c = abi.default_cfg(precision=abi.PREC_FP32, indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    o = orc.Oracle(c, m.neighbors(), m.delta)
    a_cpu = o.alpha(u)
    assert np.max(np.abs(s.alpha() - a_cpu)) < 1e-5
    assert rel_linf(s.rhs(), o.rhs(u, alpha=a_cpu)) < 2e-5


def test_fp32_short_run_l1():
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    c = abi.default_cfg(precision=abi.PREC_FP32, indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    t, n = s.run(t_end=2e-3)
    ref, t_ref, n_ref, _ = orc.Oracle(c, m.neighbors(), m.delta).run(u, t_end=2e-3)
    assert abs(t - t_ref) < 1e-15
    assert rel_l1(s.download()[0], ref[0]) < 1e-6


def test_fp32_sedov32_to_t_end_within_1e6_l1():
    """Config-2 accuracy gate: Sedov 32^3 blended to t = 0.05, FP32-bulk form against the plain FP64
    path (which is bit-identical to the FP64 oracle; see test_gpu_parity.py)."""
    m = mesh.brick(32, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP32):
        c = abi.default_cfg(precision=prec, indicator=abi.IND_MODAL, positivity=1)
        s = Solver(c, m)
        s.upload(u)
        t, n = s.run(t_end=0.05)
        out[prec] = (s.download(), t, n, s.status()[1])
        s.finalize()
    (u64, t64, n64, b64), (u32, t32, n32, b32) = out[abi.PREC_FP64], out[abi.PREC_FP32]
    assert abs(t64 - 0.05) < 1e-15 and abs(t32 - 0.05) < 1e-15
    assert b64 == 0 and b32 == 0
    err = rel_l1(u32[0], u64[0])
    assert err < 1e-6, err


def test_fp32_repair_path():
    """A stage that leaves inadmissible nodes: the FP32 form's cooperative repair (16 threads per
    element) restores admissibility like the oracle's serial repair, and reports the elements it
    cannot repair."""
    kappa = 1.4
    m = mesh.brick(4)
    x = m.node_coords(setups.LGL4)[0]
    one = np.ones_like(x)
    u = np.ascontiguousarray(setups.prim2cons(one, np.where(x < 0.5, -3.0, 3.0), 0 * one, 0 * one, 0.05 * one, kappa))
    c = abi.default_cfg(precision=abi.PREC_FP32, positivity=1)
    s = Solver(c, m)
    o = orc.Oracle(abi.default_cfg(positivity=1), m.neighbors(), m.delta)
    s.upload(u)
    dt, _ = o.timestep(u)
    uc, reg = u.copy(), np.zeros_like(u)
    # without the repair the stage would leave negative pressures
    bare = u.copy()
    orc.Oracle(abi.default_cfg(positivity=0), m.neighbors(), m.delta).stage(bare, np.zeros_like(u), 0, 32 * dt)
    p_bare = 0.4 * (bare[4] - 0.5 * (bare[1] ** 2 + bare[2] ** 2 + bare[3] ** 2) / bare[0])
    assert (p_bare <= 0).any()
    assert o.stage(uc, reg, 0, 32 * dt) == 0
    assert s.stage(1, 32 * dt) == 0
    got = s.download()
    p = 0.4 * (got[4] - 0.5 * (got[1] ** 2 + got[2] ** 2 + got[3] ** 2) / got[0])
    assert (got[0] > 0).all() and (p > 0).all()
    assert rel_l1(got, uc) < 1e-3
    s.upload(u)
    uc, reg = u.copy(), np.zeros_like(u)
    nb_c = o.stage(uc, reg, 0, 64 * dt)
    with pytest.raises(abi.NemoError) as ei:
        s.stage(1, 64 * dt)
    assert ei.value.code == 4 and nb_c > 0 and s.status()[1] > 0
