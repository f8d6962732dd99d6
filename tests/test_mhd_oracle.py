"""CPU tests of the GLM-MHD part of the oracle: consistency of the reference's flux functions,
the non-conservative term, free-stream preservation, mass conservation and a stable short run."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from oracle import oracle as orc

K, MU0 = 5.0 / 3.0, 1.0


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def mhd_cfg(**kw):
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.eqn = 4, 9, abi.EQN_MHD
    c.volume_flux, c.surface_flux = abi.VOLFLUX_EC_MHD, abi.SURFFLUX_RUSANOV
    c.alpha_smoothing, c.positivity = 1, 0
    c.kappa, c.mu0, c.cfl, c.alpha_max, c.alpha_min, c.repair_decr = K, MU0, 0.5, 0.5, 0.001, 0.01
    c.glm_ch, c.glm_alpha = 0.7, 0.3
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def rand_mhd(rng):
    return setups.mhd_prim2cons(rng.uniform(0.5, 2), *rng.uniform(-1, 1, 3), rng.uniform(0.5, 2),
                                *rng.uniform(-1, 1, 3), rng.uniform(-0.2, 0.2), K, MU0)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_mhd_flux_consistency(d):
    rng = np.random.default_rng(d)
    for _ in range(20):
        u = rand_mhd(rng)
        f = orc.mhd_flux(d, u, ch=0.7)
        np.testing.assert_allclose(orc.mhd_twopoint(abi.VOLFLUX_EC_MHD, d, u, u, ch=0.7), f, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(orc.mhd_twopoint(abi.VOLFLUX_CENTRAL, d, u, u, ch=0.7), f, rtol=1e-15, atol=1e-15)
        np.testing.assert_allclose(orc.mhd_riemann(d, u, u, ch=0.7), f, rtol=1e-14, atol=1e-14)


def test_mhd_physical_flux_values():
    """x-flux of a state against the textbook GLM-MHD flux (total pressure form)."""
    rng = np.random.default_rng(9)
    u = rand_mhd(rng)
    rho, m, E, B, psi = u[0], u[1:4], u[4], u[5:8], u[8]
    v = m / rho
    p = (K - 1) * (E - 0.5 * rho * v @ v - 0.5 * (B @ B + psi ** 2) / MU0)
    pt = p + 0.5 * B @ B / MU0
    ch = 0.7
    f = np.array([m[0], m[0] * v[0] + pt - B[0] ** 2, m[0] * v[1] - B[0] * B[1], m[0] * v[2] - B[0] * B[2],
                  (E - 0.5 * psi ** 2 + pt) * v[0] - B[0] * (v @ B) + ch * B[0] * psi, ch * psi,
                  v[0] * B[1] - B[0] * v[1], v[0] * B[2] - B[0] * v[2], ch * B[0]])
    np.testing.assert_allclose(orc.mhd_flux(0, u, ch=ch), f, rtol=1e-13, atol=1e-13)
    assert abs(orc.lib().or_mhd_pressure(orc._p(np.ascontiguousarray(u)), K, MU0) - p) < 1e-14


def test_mhd_nonconservative_term():
    rng = np.random.default_rng(3)
    ui, ul, ur = rand_mhd(rng), rand_mhd(rng), rand_mhd(rng)
    f = orc.mhd_nc(0, ui, ul, ur)
    bavg, gavg = 0.5 * (ul[5] + ur[5]), 0.5 * (ul[8] + ur[8])
    v = ui[1:4] / ui[0]
    ref = np.zeros(9)
    ref[1:4] = bavg * ui[5:8] / MU0
    ref[4] = bavg * (ui[5:8] @ v) / MU0 + gavg * v[0] * ui[8] / MU0
    ref[5:8] = bavg * v
    ref[8] = gavg * v[0]
    np.testing.assert_allclose(f, ref, rtol=1e-14, atol=1e-15)


def test_mhd_free_stream_and_mass_conservation():
    m = mesh.brick(3, 2, 2)
    o = orc.Oracle(mhd_cfg(), m.neighbors(), m.delta, nthreads=2)
    const = np.broadcast_to(setups.mhd_prim2cons(1.2, 0.3, -0.1, 0.2, 0.8, 0.4, 0.2, -0.3, 0.0, K)[:, None, None],
                            (9, m.E, 64)).copy()
    assert np.max(np.abs(o.rhs(const))) < 1e-12
    mo = mesh.brick(4)
    u = setups.orszag_tang(mo)
    oo = orc.Oracle(mhd_cfg(), mo.neighbors(), mo.delta, nthreads=4)
    r = oo.rhs(u)
    tot = oo.totals(r)
    assert abs(tot[0]) < 1e-13 * np.max(np.abs(r[0]))


def test_orszag_tang_short_run_stable_and_div_b_small():
    m = mesh.brick(4)
    u = setups.orszag_tang(m)
    o = orc.Oracle(mhd_cfg(), m.neighbors(), m.delta, nthreads=8)
    x, w, D, S, Vi = orc.operators()
    l2_0, _ = setups.divergence_b(m, u, D, w)
    u1, t, n, nbad = o.run(u, nsteps=10)
    assert np.all(np.isfinite(u1)) and nbad == 0 and t > 0
    l2_1, _ = setups.divergence_b(m, u1, D, w)
    assert l2_1 < 0.5, (l2_0, l2_1)   # the GLM cleaning keeps the discrete divergence bounded


HLLD = abi.SURFFLUX_HLLD


@pytest.mark.parametrize("d", [0, 1, 2])
def test_hlld_consistency(d):
    rng = np.random.default_rng(20 + d)
    for _ in range(50):
        u = rand_mhd(rng)
        np.testing.assert_allclose(orc.mhd_riemann(d, u, u, ch=0.7, kind=HLLD), orc.mhd_flux(d, u, ch=0.7),
                                   rtol=1e-12, atol=1e-12)


def test_hlld_mirror_symmetry():
    """x -> -x maps (m_x, B_x) -> -(m_x, B_x); a symmetric numerical flux obeys
    F(M uR, M uL) = S F(uL, uR) with S = diag(-1, 1, -1, -1, -1, 1, -1, -1, -1)."""
    rng = np.random.default_rng(31)
    M = np.array([1, -1, 1, 1, 1, -1, 1, 1, 1.0])
    S = np.array([-1, 1, -1, -1, -1, 1, -1, -1, -1.0])
    for _ in range(200):
        uL, uR = rand_mhd(rng), rand_mhd(rng)
        f = orc.mhd_riemann(0, uL, uR, ch=0.7, kind=HLLD)
        g = orc.mhd_riemann(0, M * uR, M * uL, ch=0.7, kind=HLLD)
        np.testing.assert_allclose(g, S * f, rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("bx", [0.0, 0.8])
def test_hlld_resolves_stationary_contact(bx):
    """An isolated stationary contact (equal p, B, zero velocity, density jump) has zero mass and
    energy flux under HLLD; Rusanov smears it."""
    uL = setups.mhd_prim2cons(1.0, 0, 0, 0, 1.0, bx, 0.3, -0.2, 0.0, K, MU0)
    uR = setups.mhd_prim2cons(0.2, 0, 0, 0, 1.0, bx, 0.3, -0.2, 0.0, K, MU0)
    f = orc.mhd_riemann(0, uL, uR, kind=HLLD)
    assert abs(f[0]) < 1e-14 and abs(f[4]) < 1e-14
    pt = 1.0 + 0.5 * (bx * bx + 0.09 + 0.04)
    assert abs(f[1] - (pt - bx * bx)) < 1e-13
    assert abs(orc.mhd_riemann(0, uL, uR, kind=abi.SURFFLUX_RUSANOV)[0]) > 0.1


def test_hlld_supersonic_upwinds():
    """Both states moving right faster than the fast speed: the flux is the left state's flux."""
    uL = setups.mhd_prim2cons(1.0, 5.0, 0.1, 0, 1.0, 0.3, 0.2, 0.1, 0.0, K, MU0)
    uR = setups.mhd_prim2cons(0.5, 6.0, 0.0, 0, 0.8, 0.3, 0.1, 0.0, 0.0, K, MU0)
    np.testing.assert_allclose(orc.mhd_riemann(0, uL, uR, ch=0.0, kind=HLLD), orc.mhd_flux(0, uL, ch=0.0),
                               rtol=1e-13, atol=1e-13)


def test_hlld_orszag_tang_run_stable():
    m = mesh.brick(4)
    u = setups.orszag_tang(m)
    c = mhd_cfg(surface_flux=HLLD)
    o = orc.Oracle(c, m.neighbors(), m.delta)
    uc, t, n, _ = o.run(u, nsteps=20)
    assert np.all(np.isfinite(uc)) and n == 20
    tot0, tot1 = o.totals(u), o.totals(uc)
    assert abs(tot1[0] - tot0[0]) < 1e-13 * abs(tot0[0])
