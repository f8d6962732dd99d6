"""Barotropic cooling (CPU, oracle): after every stage the energy of each node is the barotropic
equation of state -- isothermal at or below dens_critical, adiabatic above -- and nothing else
changes (source/physics/cooling/barotropic_cooling_mod.f90:39-53)."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def cfg(source):
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.eqn = 4, 5, abi.EQN_EULER
    c.indicator, c.alpha_smoothing, c.positivity = abi.IND_MODAL, 1, 1
    c.kappa, c.mu0, c.cfl, c.alpha_max, c.alpha_min, c.repair_decr = 5.0 / 3.0, 1.0, 0.5, 0.5, 0.001, 0.01
    c.source = source
    c.dens_critical, c.k_isothermal = 1.0, 1.0
    c.k_adiabatic = 1.0 * 1.0 ** (1.0 - c.kappa)   # continuous pressure at dens_critical
    return c


def test_cooling_sets_the_barotropic_energy():
    m = mesh.brick(4)
    u = setups.smooth_random(m, seed=6, kappa=5.0 / 3.0)
    assert (u[0] < 1.0).any() and (u[0] > 1.0).any()
    c0, c1 = cfg(abi.SOURCE_NONE), cfg(abi.SOURCE_BAROTROPIC_COOLING)
    o0, o1 = orc.Oracle(c0, m.neighbors(), m.delta), orc.Oracle(c1, m.neighbors(), m.delta)
    dt, _ = o0.timestep(u)
    a, ra = u.copy(), np.zeros_like(u)
    b, rb = u.copy(), np.zeros_like(u)
    o0.stage(a, ra, 0, dt)
    o1.stage(b, rb, 0, dt)
    assert np.array_equal(a[:4], b[:4]) and np.array_equal(ra, rb)
    kin = 0.5 / b[0] * (b[1] ** 2 + b[2] ** 2 + b[3] ** 2)
    kap = c1.kappa
    expect = np.where(b[0] <= c1.dens_critical, kin + c1.k_isothermal / (kap - 1) * b[0],
                      kin + c1.k_adiabatic / (kap - 1) * b[0] ** kap)
    np.testing.assert_allclose(b[4], expect, rtol=1e-14, atol=0)
    p = (kap - 1) * (b[4] - kin)
    np.testing.assert_allclose(p, np.where(b[0] <= 1.0, b[0], b[0] ** kap), rtol=1e-12)


def test_cooled_run_conserves_mass_and_momentum():
    m = mesh.brick(4)
    u = setups.smooth_random(m, seed=7, kappa=5.0 / 3.0)
    o = orc.Oracle(cfg(abi.SOURCE_BAROTROPIC_COOLING), m.neighbors(), m.delta)
    uc, t, n, nbad = o.run(u, nsteps=5)
    assert n == 5 and nbad == 0 and np.all(np.isfinite(uc))
    t0, t1 = o.totals(u), o.totals(uc)
    np.testing.assert_allclose(t1[:4], t0[:4], rtol=0, atol=1e-13 * np.abs(t0).max())
