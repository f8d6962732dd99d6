"""Forest adapt (CPU): the new leaf set stays 2:1-balanced and tiles the box, the remap rows point at
the right old elements, and the oracle's payload transfer -- interpolation from an ancestor,
projection of 8 children -- reproduces polynomials it should reproduce and conserves the totals."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def base_forest():
    return mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)


def flags_for(m):
    f = np.zeros(m.E, dtype=np.int32)
    f[m.center[:, 0] < 0.25] = 1
    f[m.center[:, 0] > 0.6] = -1
    return f


def test_adapt_leaf_set_and_remap_rows():
    m = base_forest()
    n, r = mesh.adapt(m, flags_for(m))
    assert abs(np.prod(n.delta, axis=1).sum() - 1.0) < 1e-14
    n.neighbors()
    for row in n.mortars():          # 2:1 across every non-conforming face
        assert np.all(n.level[row[2:]] == n.level[row[0]] + 1)
    kinds = np.bincount(r[:, 0], minlength=3)
    assert kinds[1] > 0 and kinds[2] > 0
    for e, (kind, src, depth, off) in enumerate(r):
        if kind == 0:
            assert np.allclose(n.center[e], m.center[src]) and np.allclose(n.delta[e], m.delta[src])
        elif kind == 1:
            assert np.allclose(n.delta[e] * 2 ** depth, m.delta[src])
            assert np.all(np.abs(n.center[e] - m.center[src]) < 0.5 * m.delta[src])
        else:
            assert np.allclose(n.delta[e], 2 * m.delta[src])
            assert np.allclose(m.center[src:src + 8].mean(axis=0), n.center[e])


def poly_state(m, deg):
    """Admissible state whose variables are polynomials of degree deg in x, y, z."""
    x, y, z = m.node_coords(setups.LGL4)
    rng = np.random.default_rng(deg)
    c = rng.uniform(-1, 1, size=(5, 4))
    p = [c[v, 0] + c[v, 1] * x + c[v, 2] * y ** min(deg, 2) + c[v, 3] * (x * y * z if deg >= 3 else z)
         for v in range(5)]
    return np.ascontiguousarray(np.stack([3.0 + 0.5 * p[0], 0.2 * p[1], 0.2 * p[2], 0.2 * p[3], 20.0 + p[4]]))


def test_remap_reproduces_polynomials():
    m = base_forest()
    n, r = mesh.adapt(m, flags_for(m))
    # refinement and copies are exact for cubics; the LGL projection is exact up to degree 2
    for deg in (2, 3):
        u = poly_state(m, deg)
        got = orc.remap(u, r)
        want = poly_state(n, deg)
        sel = r[:, 0] != 2 if deg == 3 else np.ones(n.E, dtype=bool)
        np.testing.assert_allclose(got[:, sel], want[:, sel], atol=1e-13)


def test_remap_conserves_totals():
    m = base_forest()
    n, r = mesh.adapt(m, flags_for(m))
    u = setups.smooth_random(m, seed=3)
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.kappa = 4, 5, 1.4
    t0 = orc.Oracle(c, m.neighbors(), m.delta, mortars=m.mortars()).totals(u)
    t1 = orc.Oracle(c, n.neighbors(), n.delta, mortars=n.mortars()).totals(orc.remap(u, r))
    np.testing.assert_allclose(t1, t0, rtol=1e-14, atol=1e-14)


def test_inadmissible_refinement_falls_back_to_the_mean():
    """A density profile positive at the nodes whose cubic dips below zero inside the element: its
    children take the parent's mean (all of them, so the family conserves), the rest is untouched."""
    m = base_forest()
    x = setups.LGL4
    i0 = int(np.nonzero(m.level == 0)[0][0])
    u = poly_state(m, 2)
    prof = np.where(np.abs(np.abs(x) - 1.0) < 1e-12, 1.0, 1e-3)       # 1, 1e-3, 1e-3, 1 along x
    u[0, i0] = np.tile(prof, 16)                                        # node n = i + 4j + 16k
    u[1:4, i0] = 0.0
    u[4, i0] = 2.5
    f = np.zeros(m.E, dtype=np.int32)
    f[i0] = 1
    n, r = mesh.adapt(m, f)
    got = orc.remap(u, r)
    kids = np.nonzero((r[:, 0] == 1) & (r[:, 1] == i0))[0]
    assert len(kids) == 8
    wq = orc.lgl(3)[1]
    w = np.einsum("a,b,c->cba", wq, wq, wq).ravel()
    for v in range(5):
        np.testing.assert_allclose(got[v, kids], (w @ u[v, i0]) / 8.0, rtol=1e-14, atol=1e-15)
    plain = orc.remap(poly_state(m, 2), r)
    np.testing.assert_array_equal(got[:, r[:, 0] == 0], plain[:, r[:, 0] == 0])
    assert np.all(got[0] > 0)
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.kappa = 4, 5, 1.4
    t0 = orc.Oracle(c, m.neighbors(), m.delta, mortars=m.mortars()).totals(u)
    t1 = orc.Oracle(c, n.neighbors(), n.delta, mortars=n.mortars()).totals(got)
    np.testing.assert_allclose(t1, t0, rtol=1e-14, atol=1e-14)


def test_coarsening_undone_by_balance_is_dropped():
    """A family flagged for coarsening whose face neighbours refine at the same time would leave a
    level jump of 2: the coarsening is dropped (its 8 leaves are copied), the refinement stays; the
    same family alone coarsens."""
    m = mesh.forest(2, lambda lvl, c, s: np.full(len(c), lvl < 2), max_level=3)
    lev, crd = m.tree["lev"], m.tree["crd"]
    fam = np.nonzero((lev == 2) & np.all(crd >> 1 == 0, axis=1))[0]
    nbr = np.nonzero((lev == 2) & (crd[:, 0] == 2) & (crd[:, 1] < 2) & (crd[:, 2] < 2))[0]
    assert len(fam) == 8 and len(nbr) == 4
    f = np.zeros(m.E, np.int32)
    f[fam] = -1
    f[nbr] = 1
    n, r = mesh.adapt(m, f)
    assert not np.any(r[:, 0] == 2) and np.sum(r[:, 0] == 1) == 32
    assert set(fam) <= set(r[r[:, 0] == 0, 1])
    for row in n.mortars():
        assert np.all(n.level[row[2:]] == n.level[row[0]] + 1)
    f[nbr] = 0
    n2, r2 = mesh.adapt(m, f)
    assert n2.E == m.E - 7 and np.sum(r2[:, 0] == 2) == 1 and r2[r2[:, 0] == 2][0, 1] == fam[0]


def test_inadmissible_coarsening_falls_back_to_the_mean():
    """Children with rough but positive densities whose projection undershoots below zero: the
    coarsened element takes the mean of its 8 children (conservative and admissible)."""
    m = mesh.forest(2, lambda lvl, c, s: np.full(len(c), lvl < 1), max_level=2)
    lev, crd = m.tree["lev"], m.tree["crd"]
    fam = np.nonzero((lev == 1) & np.all(crd >> 1 == 0, axis=1))[0]
    u = np.zeros((5, m.E, 64))
    u[0], u[4] = 1.0, 2.5
    rng = np.random.default_rng(1)
    for c in fam:
        u[0, c] = np.where(rng.random(64) < 0.5, 1e-3, 3.0)
    # the plain projection (sum of the children's L2 projections) is not admissible
    _, prj = orc.mortar_operators()
    plain = sum(np.einsum("ai,bj,ck,kji->cba", prj[c & 1], prj[(c >> 1) & 1], prj[c >> 2],
                          u[0, fam[c]].reshape(4, 4, 4)) for c in range(8))
    assert plain.min() < 0
    f = np.zeros(m.E, np.int32)
    f[fam] = -1
    n, r = mesh.adapt(m, f)
    got = orc.remap(u, r)
    e2 = int(np.nonzero(r[:, 0] == 2)[0][0])
    wq = orc.lgl(3)[1]
    w = np.einsum("a,b,c->cba", wq, wq, wq).ravel()
    for v in range(5):
        np.testing.assert_allclose(got[v, e2], np.mean([w @ u[v, c] / 8.0 for c in fam]), rtol=1e-14, atol=1e-15)
    assert np.all(got[0] > 0)
