"""CPU tests of the 2:1 forest generator and of the oracle's mortar operator on it: mesh invariants,
the mortar matrices, free-stream preservation, conservation of the totals and the convergence order
of a smooth wave across refinement interfaces."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def band_forest(nb, max_level=2, width=0.2):
    """nb^3 base elements on [0,1]^3 refined around the plane y = 0.5 (level 1 within width, level 2
    within width/2)."""
    return mesh.forest(nb, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < width / (1 + lvl), max_level=max_level)


def test_forest_invariants():
    m = band_forest(4)
    assert m.E > 4 ** 3 and set(np.unique(m.level)) == {0, 1, 2}
    assert abs(np.prod(m.delta, axis=1).sum() - 1.0) < 1e-14          # leaves tile the box
    nbr = m.neighbors()
    mo = m.mortars()
    assert len(mo) > 0
    # every element face is on exactly one side / mortar; fine quads of a mortar are one level finer
    for row in mo:
        qc, fc, fine = row[0], row[1], row[2:]
        assert np.all(m.level[fine] == m.level[qc] + 1)
        d = fc >> 1
        # fine quads touch the coarse face: their face centres lie on the coarse face plane
        sgn = 1 if fc & 1 else -1
        plane = m.center[qc, d] + sgn * 0.5 * m.delta[qc, d]
        fpl = m.center[fine, d] - sgn * 0.5 * m.delta[fine, d]
        assert np.allclose(np.mod(fpl - plane + 0.5, 1.0) - 0.5, 0.0)
        t1, t2 = [a for a in range(3) if a != d]
        for k in range(4):
            s, t = k & 1, k >> 1
            off1 = m.center[fine[k], t1] - m.center[qc, t1]
            off2 = m.center[fine[k], t2] - m.center[qc, t2]
            assert np.sign(off1) == (1 if s else -1) and np.sign(off2) == (1 if t else -1)
    # conforming neighbours have equal size; 2:1 balance holds across every mortar
    conf = nbr >= 0
    e_idx = np.nonzero(conf)
    assert np.all(m.level[e_idx[0]] == m.level[nbr[conf]])
    assert (nbr <= -2).sum() == 5 * len(mo)


def test_kh_forest_size():
    m = mesh.kh_forest()
    assert 140_000 < m.E < 170_000
    assert len(m.mortars()) > 10_000


def test_mortar_operators():
    pro, prj = orc.mortar_operators()
    x, w = orc.lgl(3)
    # prolongation reproduces cubics on each half; projection preserves the face integral
    p = lambda t: 0.3 - 1.2 * t + 0.7 * t ** 2 + 0.45 * t ** 3   # noqa: E731
    for s, mu in ((0, -0.5), (1, 0.5)):
        np.testing.assert_allclose(pro[s] @ p(x), p(mu + x / 2), atol=1e-14)
    f = [np.cos(3 * (x / 2 - 0.5)), np.sin(2 * (x / 2 + 0.5))]
    coarse = prj[0] @ f[0] + prj[1] @ f[1]
    assert abs(w @ coarse - 0.5 * (w @ f[0] + w @ f[1])) < 1e-14
    np.testing.assert_allclose(prj.sum(axis=(0, 2)), 1.0, atol=1e-14)


@pytest.mark.parametrize("mhd", [False, True])
def test_forest_free_stream(mhd):
    m = band_forest(4)
    if mhd:
        c = abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_HLLD,
                            kappa=5 / 3, mu0=1.0, glm_ch=0.5)
        u1 = setups.mhd_prim2cons(1.3, 0.4, -0.2, 0.3, 0.9, 0.2, 0.3, -0.1, 0.0, 5 / 3)
    else:
        c = abi.default_cfg()
        u1 = setups.prim2cons(1.3, 0.4, -0.2, 0.3, 0.9, 1.4)
    u = np.ascontiguousarray(np.broadcast_to(np.asarray(u1)[:, None, None], (len(u1), m.E, 64)))
    r = orc.Oracle.for_mesh(c, m).rhs(u)
    assert np.max(np.abs(r)) < 1e-12


@pytest.mark.parametrize("sf,ind", [(abi.SURFFLUX_HLLC, abi.IND_NONE), (abi.SURFFLUX_RUSANOV, abi.IND_MODAL)])
def test_forest_conservation(sf, ind):
    m = band_forest(4)
    c = abi.default_cfg(surface_flux=sf, indicator=ind)
    u = setups.smooth_random(m, seed=3)
    o = orc.Oracle.for_mesh(c, m)
    uc, t, n, _ = o.run(u, nsteps=5)
    t0, t1 = o.totals(u), o.totals(uc)
    assert np.all(np.abs(t1 - t0) < 2e-14 * np.maximum(np.abs(t0), 1.0))


def test_forest_convergence():
    """x-wave rho = 1 + 0.2 sin(2 pi x) advected at u = 1 through a refined band: 4th-order-like
    convergence between two forests of the same pattern."""
    errs = []
    for nb in (4, 8):
        m = band_forest(nb, max_level=1, width=0.15)
        x, y, z = m.node_coords(orc.lgl(3)[0])
        one = np.ones_like(x)
        u = np.ascontiguousarray(setups.prim2cons(1 + 0.2 * np.sin(2 * np.pi * x), one, 0 * one, 0 * one, one, 1.4))
        o = orc.Oracle.for_mesh(abi.default_cfg(surface_flux=abi.SURFFLUX_HLLC), m)
        uc, t, n, _ = o.run(u, t_end=0.1)
        exact = 1 + 0.2 * np.sin(2 * np.pi * (x - t))
        errs.append(np.max(np.abs(uc[0] - exact)))
    order = np.log2(errs[0] / errs[1])
    assert order > 3.0, (errs, order)


def test_concat_batch_neighbors():
    f = band_forest(2, max_level=1)
    b = mesh.brick(2)
    m, g = mesh.concat([f, b, b])
    assert m.E == f.E + 2 * b.E and list(np.bincount(g)) == [f.E, b.E, b.E]
    nbr = m.neighbors()
    nf = f.neighbors()
    # the forest part keeps its neighbours and mortar rows; members point into their own block
    assert np.array_equal(nbr[: f.E], nf)
    assert np.array_equal(m.mortars(), f.mortars())
    for i in range(2):
        blk = nbr[f.E + i * b.E: f.E + (i + 1) * b.E]
        assert blk.min() >= f.E + i * b.E and blk.max() < f.E + (i + 1) * b.E


def shocked_coarse_state(m):
    """A state whose coarse mortar elements hold density P(x) P(y) P(z), P through 1, 1e-3, 1e-3, 1 at
    the nodes: admissible at every node, but the prolonged trace dips below zero on the sub-faces."""
    u = setups.smooth_random(m, seed=4)
    x = orc.lgl(3)[0]
    p = np.where(np.abs(np.abs(x) - 1.0) < 1e-12, 1.0, 1e-3)
    rho = np.einsum("k,j,i->kji", p, p, p).ravel()                    # node n = i + 4j + 16k
    qc = np.unique(m.mortars()[:, 0])
    u[0, qc] = rho
    u[1:4, qc] = 0.0
    u[4, qc] = 2.5
    return u, qc


def test_mortar_trace_guard():
    m = band_forest(4)
    u, qc = shocked_coarse_state(m)
    pro, _ = orc.mortar_operators()
    face = u[0, qc[0]].reshape(4, 4, 4)[0]                             # the k = 0 face, [j][i]
    sub = np.einsum("ia,jb,ba->ji", pro[0], pro[0], face)
    assert sub.min() < 0.0                                               # the plain prolongation fails
    c = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1)
    r = orc.Oracle.for_mesh(c, m).rhs(u)
    assert np.all(np.isfinite(r))
    o = orc.Oracle.for_mesh(c, m)
    u2, _, _, _ = o.run(u, nsteps=2)
    assert np.all(np.isfinite(u2))
    np.testing.assert_allclose(o.totals(u2), o.totals(u), rtol=1e-13, atol=1e-13)
