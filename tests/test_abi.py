"""CPU tests of the C-ABI library: it loads, exports every entry point include/nemo_gpu.h declares,
its host-built operators equal the oracle's bit for bit, and its argument checks fail cleanly without
touching a GPU.  No compute call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

from nemo_b200 import abi, build, mesh
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return abi.load()


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "nemo_gpu.h")).read()
    return sorted(set(re.findall(r"^int\s+(nemo_gpu_\w+)\s*\(", txt, flags=re.M)))


def test_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(abi.EXPORTS) == syms


def test_operators_bit_identical_to_oracle(lib):
    x, w, D, S, Vi = abi.operators()
    ox, ow, oD, oS, oVi = orc.operators()
    for a, b in ((x, ox), (w, ow), (D, oD), (S, oS), (Vi, oVi)):
        assert np.array_equal(a, b)
    np.testing.assert_allclose(Vi @ np.array([[orc_leg(j, xi) for j in range(4)] for xi in x]), np.eye(4),
                               atol=1e-14)


def test_mortar_operators_bit_identical_to_oracle(lib):
    pro, prj = abi.mortar_operators()
    opro, oprj = orc.mortar_operators()
    assert np.array_equal(pro, opro) and np.array_equal(prj, oprj)


def orc_leg(n, x):
    from numpy.polynomial import legendre
    c = np.zeros(n + 1)
    c[n] = 1
    return legendre.legval(x, c) * np.sqrt(n + 0.5)


def test_sbp_property_of_split_matrix(lib):
    """W S is skew-symmetric (S = 2D - W^-1 B with Q + Q^T = B)."""
    x, w, D, S, Vi = abi.operators()
    WS = np.diag(w) @ S
    assert np.max(np.abs(WS + WS.T)) < 1e-14
    Q = np.diag(w) @ D
    B = np.diag([-1.0, 0, 0, 1.0])
    assert np.max(np.abs(Q + Q.T - B)) < 1e-14


def test_argument_errors_without_gpu(lib):
    bad = abi.default_cfg(n_nodes=5)
    rc = lib.nemo_gpu_init(ctypes.byref(bad))
    assert rc == 1 and "n_nodes" in abi.last_error()
    rc = lib.nemo_gpu_operators(3, None, None, None, None, None)
    assert rc == 1
    m = mesh.brick(2)
    rc = lib.nemo_gpu_upload_state(abi.ptr(np.zeros(10)), 8)
    assert rc == 2   # no mesh yet
    buf = ctypes.create_string_buffer(8)
    assert lib.nemo_gpu_last_error(buf, 8) == 0 and len(buf.value) <= 7
    del m


def test_default_cfg(lib):
    c = abi.default_cfg()
    assert (c.n_nodes, c.n_vars, c.volume_flux, c.surface_flux, c.precision) == (4, 5, 0, 0, 0)
    assert c.kappa == 1.4 and c.alpha_max == 0.5 and c.repair_decr == 0.01


def test_mesh_generator_invariants():
    m = mesh.brick(4, 2, 3)
    nbr = m.neighbors()
    E = m.E
    for e in range(E):
        for f in range(6):
            ne = nbr[e, f]
            assert nbr[ne, f ^ 1] == e
    # Morton order: the first 8 elements of a 4^3 brick form a 2x2x2 block
    m4 = mesh.brick(4)
    c = m4.center[:8]
    assert np.ptp(c, axis=0).max() <= 0.25 + 1e-12
    mb = mesh.brick(3, 3, 3, periodic=(False, True, False))
    nb = mb.neighbors()
    assert (nb[:, 0] == -1).sum() == 9 and (nb[:, 1] == -1).sum() == 9 and (nb[:, 2] >= 0).all()


def test_host_only_cfg_matches_library_defaults(lib):
    """abi.cfg_struct (used where only the oracle runs) equals nemo_gpu_default_cfg field by field."""
    a, b = abi.cfg_struct(), abi.default_cfg()
    for name, _ in abi.NemoCfg._fields_:
        assert getattr(a, name) == getattr(b, name), name


def test_amr_operators_are_the_adapt_interpolation_and_projection(lib):
    """refineMat/coarseMat for hosts' replace callbacks: at q = N the 1D factors are the mortar
    prolongation/projection of the child's half; lower q truncate to Legendre modes 0..q (q = 0:
    the element mean)."""
    R, C = abi.amr_operators(3)
    pro, prj = abi.mortar_operators()
    x, w, D, S, Vi = abi.operators()
    V = np.linalg.inv(Vi)
    for f in range(8):
        for d in range(3):
            s = (f >> d) & 1
            np.testing.assert_allclose(R[3, f, d], pro[s], atol=1e-14)
            np.testing.assert_allclose(C[3, f, d], prj[s], atol=1e-14)
            for q in range(4):
                P = V[:, : q + 1] @ Vi[: q + 1, :]
                np.testing.assert_allclose(R[q, f, d], pro[s] @ P, atol=1e-13)
                np.testing.assert_allclose(C[q, f, d], P @ prj[s], atol=1e-13)
    # refining then projecting back keeps the integral (Gauss-Lobatto quadrature is exact to degree 5
    # on each half) and constants (the projection is not the identity: the quadrature is not exact
    # for the degree-6 products of the projection)
    back = C[3, 0, 0] @ R[3, 0, 0] + C[3, 1, 0] @ R[3, 1, 0]
    np.testing.assert_allclose(w @ back, w, atol=1e-14)
    np.testing.assert_allclose(back @ np.ones(4), np.ones(4), atol=1e-14)
    mean = np.outer(np.ones(4), w / 2.0)
    np.testing.assert_allclose(R[0, 5, 1], mean, atol=1e-14)
    rc = lib.nemo_gpu_amr_operators(4, 4, None, None)
    assert rc == 1 and "qmax" in abi.last_error()


def test_repair_states_needs_init(lib):
    ok = np.zeros(1, dtype=np.int32)
    st = np.zeros((1, 5, 64))
    abi.call("nemo_gpu_finalize")
    rc = lib.nemo_gpu_repair_states(abi.ptr(st), 1, 5 * 64 * 8, abi.ptr(ok))
    assert rc == 2 and "init" in abi.last_error()
