"""CPU tests of the FP64 oracle: known-answer values, identities of the reference's routines and of
the published methods, and an independent numpy restatement of the element operator.

The reference (Fortran) ships no tests or golden vectors and cannot be built here; these are the
pins of the oracle (see oracle/nemo_oracle.cpp)."""
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as orc
from nemo_b200 import abi, mesh, setups

HERE = os.path.dirname(os.path.abspath(__file__))
KAPPA = 1.4


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def cfg(**kw):
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.eqn = 4, 5, 0
    c.volume_flux, c.surface_flux, c.precision, c.indicator = 0, 0, 0, 0
    c.alpha_smoothing, c.positivity = 1, 0
    c.kappa, c.mu0, c.cfl, c.alpha_max, c.alpha_min, c.repair_decr = KAPPA, 1.0, 0.5, 0.5, 0.001, 0.01
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def rand_state(rng, n=1):
    rho = rng.uniform(0.5, 2.0, n)
    v = rng.uniform(-1, 1, (3, n))
    p = rng.uniform(0.3, 3.0, n)
    return setups.prim2cons(rho, v[0], v[1], v[2], p, KAPPA).T


# ---- known answers ------------------------------------------------------------------------------

def test_lgl_nodes_closed_form():
    x, w = orc.lgl(3)
    a = 1.0 / math.sqrt(5.0)
    np.testing.assert_allclose(x, [-1, -a, a, 1], rtol=0, atol=2e-16)
    np.testing.assert_allclose(w, [1 / 6, 5 / 6, 5 / 6, 1 / 6], rtol=0, atol=4e-16)
    for N in (2, 4, 5, 7):  # exact integration of x^(2N-1)... by the Lobatto rule
        x, w = orc.lgl(N)
        for p in range(0, 2 * N):
            exact = (1 - (-1) ** (p + 1)) / (p + 1)
            assert abs(np.sum(w * x ** p) - exact) < 1e-13


def test_golden_known_answers():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        gold = json.load(f)
    for case in gold["flux"]:
        np.testing.assert_allclose(orc.flux(case["dir"], case["u"]), case["f"], rtol=1e-15, atol=1e-15)
    for case in gold["logmean"]:
        assert abs(orc.logmean(case["a"], case["b"]) - case["r"]) <= 1e-15 * abs(case["r"])
    for case in gold["rusanov"]:
        np.testing.assert_allclose(orc.riemann(1, case["dir"], case["uL"], case["uR"]), case["f"], rtol=1e-14,
                                   atol=1e-14)
    for case in gold["hllc"]:
        np.testing.assert_allclose(orc.riemann(0, case["dir"], case["uL"], case["uR"]), case["f"], rtol=1e-13,
                                   atol=1e-13)
    for case in gold["chandrashekar"]:
        np.testing.assert_allclose(orc.twopoint(0, case["dir"], case["u"], case["v"]), case["f"], rtol=1e-13,
                                   atol=1e-13)


def test_rk_coefficients_exact_and_fourth_order():
    a, b, c = orc.rk_coeffs()
    A = [Fraction(0), Fraction(-567301805773, 1357537059087), Fraction(-2404267990393, 2016746695238),
         Fraction(-3550918686646, 2091501179385), Fraction(-1275806237668, 842570457699)]
    C = [Fraction(1432997174477, 9575080441755), Fraction(5161836677717, 13612068292357),
         Fraction(1720146321549, 2090206949498), Fraction(3134564353537, 4481467310338),
         Fraction(2277821191437, 14882151754819)]
    assert all(float(x) == y for x, y in zip(A, a))
    assert all(float(x) == y for x, y in zip(C, c))
    # 2N scheme on y' = -y: global error order 4
    errs = []
    for n in (20, 40, 80):
        dt, y, reg = 1.0 / n, 1.0, 0.0
        for _ in range(n):
            for s in range(5):
                r = -y
                reg = r if s == 0 else a[s] * reg + r
                y = y + c[s] * dt * reg
        errs.append(abs(y - math.exp(-1.0)))
    orders = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(3.8 < o < 4.3 for o in orders), orders


# ---- identities of the flux functions -----------------------------------------------------------

@pytest.mark.parametrize("d", [0, 1, 2])
def test_flux_consistency(d):
    rng = np.random.default_rng(3 + d)
    for u in rand_state(rng, 20):
        f = orc.flux(d, u)
        np.testing.assert_allclose(orc.twopoint(0, d, u, u), f, rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(orc.twopoint(1, d, u, u), f, rtol=1e-15, atol=1e-15)
        np.testing.assert_allclose(orc.riemann(0, d, u, u), f, rtol=1e-14, atol=1e-14)
        np.testing.assert_allclose(orc.riemann(1, d, u, u), f, rtol=1e-14, atol=1e-14)


def _entropy_vars(u):
    rho, m, E = u[0], u[1:4], u[4]
    p = (KAPPA - 1) * (E - 0.5 * np.dot(m, m) / rho)
    s = math.log(p) - KAPPA * math.log(rho)
    beta = rho / p
    v = m / rho
    return np.concatenate([[(KAPPA - s) / (KAPPA - 1) - 0.5 * beta * np.dot(v, v)], beta * v, [-beta]])


@pytest.mark.parametrize("d", [0, 1, 2])
def test_chandrashekar_entropy_conservation(d):
    """(w_v - w_u) . f#(u,v) = psi_v - psi_u with psi = rho v_n (Chandrashekar 2013, Tadmor 1987)."""
    rng = np.random.default_rng(11 + d)
    us, vs = rand_state(rng, 30), rand_state(rng, 30)
    for u, v in zip(us, vs):
        f = orc.twopoint(0, d, u, v)
        lhs = np.dot(_entropy_vars(v) - _entropy_vars(u), f)
        rhs = v[1 + d] - u[1 + d]
        assert abs(lhs - rhs) < 1e-11 * (1 + abs(rhs)), (lhs, rhs)


def test_twopoint_symmetry():
    rng = np.random.default_rng(5)
    for u, v in zip(rand_state(rng, 20), rand_state(rng, 20)):
        np.testing.assert_allclose(orc.twopoint(0, 0, u, v), orc.twopoint(0, 0, v, u), rtol=1e-13, atol=1e-14)


def test_own_log_exp_accuracy():
    """The oracle's (and the plain CUDA path's) log/exp stay within 3 ulp (log) and 2 ulp (exp) of the correctly rounded
    values: about as close to the reference's intrinsic log/exp as two libms are to each other."""
    rng = np.random.default_rng(0)
    L = orc.lib()
    xs = np.concatenate([rng.uniform(0.5, 2.0, 3000), np.exp(rng.uniform(-700, 700, 3000)),
                         1.0 + rng.uniform(-1e-4, 1e-4, 2000), [1.0, 2.0, 0.5, 1e-310]])
    worst = 0.0
    for x in xs:
        ref = np.log(np.longdouble(x))
        got = L.or_log(float(x))
        if ref != 0:
            worst = max(worst, float(abs(np.longdouble(got) - ref) / np.spacing(np.float64(abs(ref)))))
    assert worst <= 3.0, worst
    assert L.or_log(1.0) == 0.0
    ys = np.concatenate([rng.uniform(-700, 700, 4000), rng.uniform(-1, 1, 2000), [0.0, -745.0, 709.7]])
    worst = 0.0
    for y in ys:
        ref = np.exp(np.longdouble(y))
        got = L.or_exp(float(y))
        if np.isfinite(ref) and ref > 2.3e-308:
            worst = max(worst, float(abs(np.longdouble(got) - ref) / np.spacing(np.float64(ref))))
    assert worst <= 2.0, worst
    assert L.or_exp(0.0) == 1.0 and L.or_exp(-800.0) == 0.0 and np.isinf(L.or_exp(800.0))


def test_logmean_series_branch():
    # near the switch the series and the direct formula agree to the conditioning of the latter
    for a in (0.5, 1.0, 3.0):
        for db in (2e-5, 5e-5, 9e-5):
            b = a + db
            exact = float((np.longdouble(a) - np.longdouble(b)) / np.log(np.longdouble(a) / np.longdouble(b)))
            assert abs(orc.logmean(a, b) - exact) < 1e-14 * exact
    assert orc.logmean(2.0, 2.0) == 2.0


# ---- the element operator ------------------------------------------------------------------------

def _numpy_rhs_central(u, m, w, D):
    """Independent strong-form DG restatement (the split form with the central flux equals it):
    du/dt = -(2/dx) [D f + (1/w)(e_N (f*_N - f_N) - e_0 (f*_0 - f_0))], summed over directions."""
    V, E, _ = u.shape
    nbr = m.neighbors()
    U = u.reshape(V, E, 4, 4, 4)  # [v][e][k][j][i]
    out = np.zeros_like(U)

    def node(d, a, b, i):  # (k, j, i) of line position i on line (a, b) of direction d
        return (b, a, i) if d == 0 else ((b, i, a) if d == 1 else (i, b, a))

    for e in range(E):
        for d in range(3):
            c = 2.0 / m.delta[e, d]
            for a in range(4):
                for b in range(4):
                    ul = [U[(slice(None), e) + node(d, a, b, i)] for i in range(4)]
                    f = [orc.flux(d, x) for x in ul]
                    nm, npl = nbr[e, 2 * d], nbr[e, 2 * d + 1]
                    um = U[(slice(None), nm) + node(d, a, b, 3)] if nm >= 0 else ul[0]
                    up = U[(slice(None), npl) + node(d, a, b, 0)] if npl >= 0 else ul[3]
                    fsm, fsp = orc.riemann(0, d, um, ul[0]), orc.riemann(0, d, ul[3], up)
                    for i in range(4):
                        s = sum(D[i, j] * f[j] for j in range(4))
                        if i == 0:
                            s = s - (fsm - f[0]) / w[0]
                        if i == 3:
                            s = s + (fsp - f[3]) / w[3]
                        out[(slice(None), e) + node(d, a, b, i)] += -c * s
    return out.reshape(V, E, 64)


def test_rhs_matches_numpy_strong_form():
    m = mesh.brick(2)
    u = setups.density_wave(m, seed=1)
    x, w, D, S, Vi = orc.operators()
    o = orc.Oracle(cfg(volume_flux=1), m.neighbors(), m.delta, nthreads=1)
    r = o.rhs(u)
    ref = _numpy_rhs_central(u, m, w, D)
    assert np.max(np.abs(r - ref)) < 1e-11 * np.max(np.abs(ref))


@pytest.mark.parametrize("vf", [0, 1])
def test_free_stream_and_conservation(vf):
    m = mesh.brick(3, 2, 2)
    o = orc.Oracle(cfg(volume_flux=vf), m.neighbors(), m.delta, nthreads=2)
    const = np.broadcast_to(setups.prim2cons(1.3, 0.4, -0.2, 0.1, 0.9, KAPPA)[:, None, None], (5, m.E, 64)).copy()
    assert np.max(np.abs(o.rhs(const))) < 1e-13
    u = setups.density_wave(m, seed=2)
    r = o.rhs(u)
    tot = o.totals(r)
    assert np.max(np.abs(tot)) < 1e-13 * np.max(np.abs(r))


def test_entropy_conservative_volume_term():
    """With the EC volume flux and an entropy-conservative surface flux (here: the same two-point
    flux), sum_nodes w J (w_entropy . rhs) = 0 on a periodic mesh (Gassner-Winters-Kopriva 2016)."""
    m = mesh.brick(2)
    u = setups.density_wave(m, seed=3, noise=0.05)
    o = orc.Oracle(cfg(volume_flux=0), m.neighbors(), m.delta, nthreads=1)
    r = o.rhs(u)
    x, w, *_ = orc.operators()
    W = np.einsum("i,j,k->kji", w, w, w).ravel()
    ent = sum(W[p] * np.dot(_entropy_vars(u[:, e, p]), r[:, e, p]) for e in range(m.E) for p in range(64))
    # HLLC is entropy stable, not conservative: the production is non-positive
    assert ent <= 1e-10


def test_convergence_order_advected_wave():
    """Smooth advected density wave (constant u and p make it an exact Euler solution): error order
    N+1 = 4 in x (cf. the manufactured wave of source/setups/euler/3d/convergence-test)."""
    errs = []
    t_end = 0.1
    for nx in (8, 16):
        m = mesh.brick(nx, 2, 2)
        xx, yy, zz = m.node_coords(setups.LGL4)
        one = np.ones_like(xx)
        u0 = np.ascontiguousarray(setups.prim2cons(1 + 0.5 * np.sin(2 * np.pi * xx), one, 0 * one, 0 * one, one, KAPPA))
        o = orc.Oracle(cfg(), m.neighbors(), m.delta)
        u, t, steps, nbad = o.run(u0, t_end=t_end)
        exact = 1.0 + 0.5 * np.sin(2 * np.pi * (xx - t))
        errs.append(np.max(np.abs(u[0] - exact)))
        assert abs(t - t_end) < 1e-14 and nbad == 0
    order = math.log2(errs[0] / errs[1])
    assert order > 3.7, (errs, order)


def test_indicator_and_blend_properties():
    m = mesh.brick(4, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    o = orc.Oracle(cfg(indicator=1), m.neighbors(), m.delta)
    al = o.alpha(u)
    assert al.max() <= 0.5 and al.min() >= 0.0
    assert al.max() > 0.0                      # the blast is detected
    ms = mesh.brick(16, 2, 2)
    xx = ms.node_coords(setups.LGL4)[0]
    one = np.ones_like(xx)
    us = np.ascontiguousarray(setups.prim2cons(1 + 0.5 * np.sin(2 * np.pi * xx), one, 0 * one, 0 * one, one, KAPPA))
    smooth = orc.Oracle(cfg(indicator=1), ms.neighbors(), ms.delta).alpha(us)
    assert smooth.max() == 0.0                 # a resolved smooth wave is left to the DG operator
    # blended operator is conservative and reduces to DG for alpha = 0
    r = o.rhs(u, alpha=al)
    assert np.max(np.abs(o.totals(r))) < 1e-12 * np.max(np.abs(r))
    r0 = o.rhs(u, alpha=np.zeros(m.E))
    rdg = orc.Oracle(cfg(indicator=0), m.neighbors(), m.delta).rhs(u)
    assert np.array_equal(r0, rdg)


def separating_streams(m, speed=3.0, p0=0.05):
    """rho = 1, u = -/+ speed across x = 1/2, low pressure: a strong rarefaction."""
    x = m.node_coords(setups.LGL4)[0]
    one = np.ones_like(x)
    return np.ascontiguousarray(setups.prim2cons(one, np.where(x < 0.5, -speed, speed), 0 * one, 0 * one,
                                                 p0 * one, KAPPA))


def _pres(u):
    return (KAPPA - 1) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0])


def test_repair_restores_admissibility():
    m = mesh.brick(4)
    u = separating_streams(m)
    o0 = orc.Oracle(cfg(positivity=0), m.neighbors(), m.delta, nthreads=4)
    o1 = orc.Oracle(cfg(positivity=1), m.neighbors(), m.delta, nthreads=4)
    dt, _ = o0.timestep(u)
    a, b = u.copy(), u.copy()
    o0.stage(a, np.zeros_like(u), 0, 32 * dt)
    nb = o1.stage(b, np.zeros_like(u), 0, 32 * dt)
    assert (_pres(a) <= 0).sum() > 0          # the update alone leaves inadmissible nodes
    assert nb == 0 and _pres(b).min() > 0     # the repair fixes all of them
    # repaired elements keep their means (the squeeze is mean-preserving)
    x, w, *_ = orc.operators()
    changed = np.nonzero(np.abs(a - b).max(axis=(0, 2)) > 0)[0]
    assert len(changed) > 0
    np.testing.assert_allclose(a[:, changed].mean(axis=2), b[:, changed].mean(axis=2), rtol=1e-12, atol=1e-12)
    # single-element entry: an inadmissible node inside an admissible element is repaired
    st = u[:, 0].copy()
    st[4, 21] = 0.0
    fixed, ok = orc.repair(cfg(positivity=1), st)
    assert ok and _pres(fixed).min() > 0


def test_timestep_formula():
    m = mesh.brick(2)
    u = setups.density_wave(m, noise=0)
    o = orc.Oracle(cfg(cfl=0.5), m.neighbors(), m.delta)
    dt, lmax = o.timestep(u)
    rho = u[0]
    p = (KAPPA - 1) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / rho)
    lam = np.abs(u[1] / rho) + np.sqrt(KAPPA * p / rho)
    assert abs(lmax - lam.max()) < 1e-15
    assert abs(dt - 0.25 * 0.5 / 7 * (0.5 / lam.max())) < 1e-15
