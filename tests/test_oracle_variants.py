"""CPU tests of the oracle's build variants (oracle/Makefile):
  - "count": the same arithmetic with an operation counter; its runs must equal the oracle's bit for
    bit (the counter must not change a single rounding or branch), and its counts must be those of
    hand-countable routines;
  - "libm": log and exp from the C library (the reference's intrinsic arithmetic) instead of the
    shared IEEE-only construction; its runs stay within round-off drift of the oracle's."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def test_counting_build_is_bit_identical_on_a_blended_run():
    c = abi.cfg_struct(indicator=abi.IND_MODAL, positivity=1)
    m = mesh.brick(4, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    a, ta, na, _ = orc.Oracle.for_mesh(c, m, nthreads=2).run(u, nsteps=3)
    oc = orc.Oracle.for_mesh(c, m, nthreads=1, variant="count")
    oc.opcount_reset()
    b, tb, nb, _ = oc.run(u, nsteps=3)
    assert np.array_equal(a, b) and ta == tb and na == nb
    cnt = oc.opcounts()
    assert cnt["add"] > 0 and cnt["mul"] > 0 and cnt["div"] > 0 and cnt["sqrt"] > 0


def test_counting_build_counts_a_logmean_by_hand():
    L = orc.lib("count")
    L.or_opcount_reset()
    L.or_logmean(1.0, 2.0)        # direct branch: x = a/b, |a - b| < eps, (a - b) / log(x)
    out = (orc.ctypes.c_uint64 * 6)()
    L.or_opcount_read(out)
    assert list(out) == [2, 0, 2, 0, 1, 0]
    L.or_opcount_reset()
    L.or_logmean(1.0, 1.00001)    # series branch (|a-b| < 1e-4)
    L.or_opcount_read(out)
    # x = a/b; |a - b| < eps; u = (x(x-2)+1)/(x(x+2)+1); (a+b)(0.5 - u(c1 - u(c2 - c3 u)))
    assert out[2] == 2 and out[4] == 0 and out[0] == 1 + 4 + 4 and out[1] == 2 + 4


def test_libm_build_drifts_only_by_round_off():
    c = abi.cfg_struct(cfl=0.5)
    m = mesh.brick(4)
    u = setups.density_wave(m, seed=1234)
    a, _, _, _ = orc.Oracle.for_mesh(c, m).run(u, nsteps=20)
    b, _, _, _ = orc.Oracle.for_mesh(c, m, variant="libm").run(u, nsteps=20)
    d = np.max(np.abs(a - b) / np.max(np.abs(a), axis=(1, 2), keepdims=True))
    assert 0.0 < d < 1e-9
