"""GPU forest adapt: the device remap of the state equals the oracle's bit for bit, a run continued
on the adapted forest equals the oracle's run from the remapped state (plain FP64 path), the totals
survive the adapt, the FP32 form runs on after it, and malformed remap rows are refused before
anything on the device changes."""
import ctypes

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


def base_forest():
    return mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)


def blast(m):
    x, y, z = m.node_coords(orc.lgl(3)[0])
    u = setups.smooth_random(m, seed=2)
    u[4] += 5.0 * np.exp(-((x - 0.3) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) / 0.01)
    return u


def flags_for(m):
    f = np.zeros(m.E, dtype=np.int32)
    f[m.center[:, 0] < 0.3] = 1
    f[m.center[:, 0] > 0.6] = -1
    return f


def test_adapt_remap_and_continued_run_bit_exact():
    m = base_forest()
    u = blast(m)
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    t1, _ = s.run(nsteps=2)
    u1 = s.download()
    uc, tc, _, _ = orc.Oracle.for_mesh(c, m).run(u, nsteps=2)
    assert np.array_equal(u1, uc) and t1 == tc
    new, remap = s.adapt(flags_for(m))
    assert new.E != m.E and np.any(remap[:, 0] == 1) and np.any(remap[:, 0] == 2)
    u2 = s.download()
    want = orc.remap(u1, remap)
    assert np.array_equal(u2, want)
    t2, n2 = s.run(nsteps=3)
    uo, to, _, _ = orc.Oracle.for_mesh(c, new).run(want, nsteps=3)
    assert n2 == 3
    assert np.array_equal(s.download(), uo)
    assert abs(t2 - (t1 + to)) <= 1e-14 * t2


def test_adapt_conserves_totals_and_fp32_runs_on():
    m = base_forest()
    u = blast(m)
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1, precision=abi.PREC_FP32)
    s = Solver(c, m)
    s.upload(u)
    s.run(nsteps=2)
    tot0 = s.totals()
    new, remap = s.adapt(flags_for(m))
    tot1 = s.totals()
    assert np.all(np.abs(tot1[:5] - tot0[:5]) <= 1e-13 * np.maximum(np.abs(tot0[:5]), 1.0))
    u_ad = s.download()
    s.run(nsteps=3)
    u32 = s.download()
    assert np.all(np.isfinite(u32)) and u32[0].min() > 0
    c64 = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    u64, _, _, _ = orc.Oracle.for_mesh(c64, new).run(u_ad, nsteps=3)
    rel = np.abs(u32[0] - u64[0]).sum() / np.abs(u64[0]).sum()
    assert rel < 1e-5, rel
    assert np.all(np.abs(s.totals()[:5] - tot1[:5]) <= 1e-5 * np.maximum(np.abs(tot1[:5]), 1.0))


def test_adapt_rejects_bad_rows():
    m = base_forest()
    c = abi.default_cfg(indicator=abi.IND_MODAL)
    s = Solver(c, m)
    u = blast(m)
    s.upload(u)
    new, remap = mesh.adapt(m, flags_for(m))
    for bad in ([1, 0, 0, 0], [1, 0, 2, 4], [2, m.E - 4, 0, 0], [0, m.E, 0, 0], [3, 0, 0, 0]):
        r = remap.copy()
        r[len(r) // 2] = bad
        with pytest.raises(abi.NemoError) as ei:
            abi.call("nemo_gpu_adapt", new.E, abi.ptr(new.delta), abi.ptr(new.center), new.S,
                     abi.ptr(new.side_quads), abi.ptr(new.side_faceid), abi.ptr(new.side_nquads),
                     abi.ptr(new.boundary), abi.ptr(np.ascontiguousarray(r, dtype=np.int32)))
        assert ei.value.code == 1   # NEMO_ERR_ARG
    assert np.array_equal(s.download(), u)   # nothing changed


def test_device_amr_flags_match_the_probe():
    m = base_forest()
    u = setups.sedov(m, sigma=0.1, center=(0.5, 0.5, 0.5))
    u[0] *= 1.0 + 0.4 * np.exp(-((m.node_coords(orc.lgl(3)[0])[0] - 0.4) ** 2) / 0.1)
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    got = s.amr_flags(1.3, 1.2)
    want = orc.amr_flags(u, 1.3, 1.2)
    assert np.array_equal(got, want) and set(np.unique(got)) == {-1, 0, 1}


def test_inadmissible_refinement_falls_back_on_the_device():
    m = base_forest()
    x = orc.lgl(3)[0]
    i0 = int(np.nonzero(m.level == 0)[0][0])
    u = blast(m)
    prof = np.where(np.abs(np.abs(x) - 1.0) < 1e-12, 1.0, 1e-3)
    u[0, i0] = np.tile(prof, 16)
    u[1:4, i0] = 0.0
    u[4, i0] = 2.5
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    f = np.zeros(m.E, dtype=np.int32)
    f[i0] = 1
    f[m.center[:, 0] > 0.6] = -1
    new, remap = s.adapt(f)
    want = orc.remap(u, remap)
    kids = np.nonzero((remap[:, 0] == 1) & (remap[:, 1] == i0))[0]
    assert len(kids) == 8 and np.all(want[0, kids] == want[0, kids[0], 0])   # the mean
    assert np.array_equal(s.download(), want)


def test_sedov_run_with_adapt_every_8_steps_bit_exact():
    """The Sedov setup's adapt cycle (every 8 steps; density > 1.3 refines, <= 1.2 coarsens) on a 4^3
    base forest with two more levels: device flags, host rebuild and device remap against the
    oracle's loop, through the refinement of the shock (and the mortar trace guard it needs)."""
    m = mesh.forest(4, lambda lvl, c, s: np.zeros(len(c), dtype=bool), max_level=2)
    u = setups.sedov(m, sigma=0.1, center=(0.5, 0.5, 0.5))
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    s = Solver(c, m)
    s.upload(u)
    t, sizes = s.run_amr(88, 8, 1.3, 1.2)
    um, mo, to = u, m, 0.0
    osizes = []
    for _ in range(11):
        new, remap = mesh.adapt(mo, orc.amr_flags(um, 1.3, 1.2))
        if new.E != mo.E or np.any(remap[:, 0]):
            um, mo = orc.remap(um, remap), new
        osizes.append(mo.E)
        um, to, _, _ = orc.Oracle.for_mesh(c, mo).run(um, nsteps=8, t0=to)
    assert sizes == osizes and max(sizes) > 8 * m.E
    assert np.all(np.isfinite(um))
    assert np.array_equal(s.download(), um)
    assert t == to


def test_mhd_adapt_bit_exact():
    """GLM-MHD (HLLD faces): remap of the 9 variables (admissibility with the magnetic pressure) and
    the continued run against the oracle."""
    m = base_forest()
    u = setups.orszag_tang(m)
    c = abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_HLLD,
                        kappa=5 / 3, mu0=1.0, glm_ch=0.7, glm_alpha=0.3, indicator=abi.IND_MODAL)
    s = Solver(c, m)
    s.upload(u)
    s.run(nsteps=2)
    u1 = s.download()
    new, remap = s.adapt(flags_for(m))
    want = orc.remap(u1, remap, kappa=5 / 3, mu0=1.0)
    assert np.array_equal(s.download(), want)
    s.run(nsteps=2)
    uo, _, _, _ = orc.Oracle.for_mesh(c, new).run(want, nsteps=2)
    assert np.array_equal(s.download(), uo)
