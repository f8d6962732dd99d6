"""GPU tests of the entry points behind the Fortran directory's per-quad host shims: the positivity
repair of host-held element states (kernel_validate_mod::kernel_repair) against the oracle's
dgfv_repair_3d, bit for bit, through a strided buffer laid out like the reference's quad array."""
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


def quad_buffer(states, pad=16):
    """states [n][V][64] -> a host buffer with one padded row per element (like quad_t)."""
    n, V, _ = states.shape
    buf = np.zeros((n, V * 64 + pad))
    buf[:, : V * 64] = states.reshape(n, V * 64)
    return buf, (V * 64 + pad) * 8


def run_repair(c, m, states):
    Solver(c, m)   # nemo_gpu_init with the configuration (the mesh is not used by the repair)
    buf, stride = quad_buffer(states)
    ok = np.full(len(states), -1, dtype=np.int32)
    rc = abi.load().nemo_gpu_repair_states(abi.ptr(buf), len(states), stride, abi.ptr(ok))
    V = states.shape[1]
    return rc, buf[:, : V * 64].reshape(states.shape), ok


@pytest.mark.parametrize("mhd", [False, True])
def test_repair_states_bit_exact_with_oracle(mhd):
    m = mesh.brick(2)
    if mhd:
        c = abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD,
                            surface_flux=abi.SURFFLUX_RUSANOV, kappa=5.0 / 3.0, mu0=1.0, positivity=1)
        u = setups.orszag_tang(m)
    else:
        c = abi.default_cfg(positivity=1)
        u = setups.smooth_random(m, seed=4)
    states = np.ascontiguousarray(u.transpose(1, 0, 2))        # [E][V][64]
    bad = [1, 3, 6]
    for e in bad:
        states[e, 4, (7 * e) % 64] = 0.0                         # zero energy: negative pressure at one node
    states[6, 4, 40] = 0.0
    rc, out, ok = run_repair(c, m, states)
    assert rc == 0, abi.last_error()
    assert ok.tolist() == [1] * len(states)
    for e in range(len(states)):
        ref, good = orc.repair(c, states[e])
        assert good
        assert np.array_equal(out[e], ref), e
        if e not in bad:
            assert np.array_equal(out[e], states[e])   # admissible elements are left as they are


def test_repair_states_reports_an_unrepairable_element():
    m = mesh.brick(2)
    c = abi.default_cfg(positivity=1)
    states = np.ascontiguousarray(setups.smooth_random(m, seed=4).transpose(1, 0, 2))
    states[2, 4, :] = 0.0            # every node without internal energy: the mean is inadmissible too
    rc, out, ok = run_repair(c, m, states)
    assert rc == 4 and "inadmissible" in abi.last_error()
    assert ok[2] == 0 and ok.sum() == len(states) - 1
    _, good = orc.repair(c, states[2])
    assert not good
