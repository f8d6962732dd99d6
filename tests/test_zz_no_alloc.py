"""GPU test of nemo_gpu_totals_noalloc, the totals entry point that allocates nothing.

It exists for hosts that cannot allocate device memory when they ask for the conserved totals:
their device arrays belong to their own pool (for example a Fortran/OpenACC data region sized at
start-up) or they run under a fixed device-memory budget where cudaMalloc/cudaFree mid-run would
fail or synchronise the device.  The caller owns the state and the output in device memory; the
library keeps its partial sums in a fixed array of its own.

Checked here through the C-ABI: two calls in a row, on two different states, each equal to what
the allocating entry point (nemo_gpu_totals) returns for the same state -- to the totals tolerance
of the other tests (1e-13 relative), and in fact bit for bit, since both run the same arithmetic.
Also: a partitioned state (owned elements followed by ghost copies, only the owned ones summed), a
9-variable GLM-MHD state, and a state of exactly the 65536 elements the fixed scratch holds.
This file is collected last so that a stop at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver

pytestmark = pytest.mark.gpu


def totals_allocating(c, m, u, n_owned=None):
    s = Solver(c, m)
    s.upload(u)
    if n_owned is not None:
        abi.call("nemo_gpu_set_owned", int(n_owned))
    out = s.totals()[: int(c.n_vars)]
    s.finalize()
    return out


def totals_noalloc(m, u, nelems=None):
    """nemo_gpu_totals_noalloc on caller-owned device copies of u [V][E][64] and the element sizes."""
    import torch
    lib = abi.load()
    V = u.shape[0]
    u_dev = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    d_dev = torch.from_numpy(np.ascontiguousarray(m.delta)).cuda()
    out_dev = torch.full((V,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.nemo_gpu_totals_noalloc(ctypes.c_void_p(u_dev.data_ptr()), ctypes.c_void_p(d_dev.data_ptr()),
                                     m.E, m.E if nelems is None else nelems, V,
                                     ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_uint64(stream))
    assert rc == 0, abi.last_error()
    torch.cuda.synchronize()
    return out_dev.cpu().numpy()


def same_totals(got, ref):
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.array_equal(got, ref)


def test_totals_noalloc_matches_allocating_entry_point_twice():
    import torch
    m1 = mesh.brick(8)
    u1 = setups.smooth_random(m1, seed=21)
    m2 = mesh.brick(16, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u2 = setups.sedov(m2, sigma=0.05)
    c = abi.default_cfg()
    refs = [totals_allocating(c, m1, u1), totals_allocating(c, m2, u2)]

    for (m, u), ref in zip(((m1, u1), (m2, u2)), refs):
        same_totals(totals_noalloc(m, u), ref)


def test_totals_noalloc_partitioned_state_sums_owned_elements_only():
    # the first 300 of 512 elements are owned, the rest stand for ghost copies of other ranks
    m = mesh.brick(8)
    u = setups.smooth_random(m, seed=5)
    ref = totals_allocating(abi.default_cfg(), m, u, n_owned=300)
    same_totals(totals_noalloc(m, u, nelems=300), ref)
    full = totals_allocating(abi.default_cfg(), m, u)
    assert not np.array_equal(ref, full)


def test_totals_noalloc_mhd_nine_variables():
    m = mesh.brick(8)
    u = setups.orszag_tang(m)
    c = abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD,
                        surface_flux=abi.SURFFLUX_RUSANOV, kappa=5.0 / 3.0, mu0=1.0)
    same_totals(totals_noalloc(m, u), totals_allocating(c, m, u))


def test_totals_noalloc_at_the_scratch_limit():
    m = mesh.brick(64, 32, 32)    # 65536 elements, the whole fixed scratch (168 MB of state)
    assert m.E == 65536
    u = setups.smooth_random(m, seed=7)
    same_totals(totals_noalloc(m, u), totals_allocating(abi.default_cfg(), m, u))


def test_totals_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = abi.load()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = lib.nemo_gpu_totals_noalloc(p, p, 65537, 65537, 5, p, ctypes.c_uint64(0))
    assert rc == 1 and "65536" in abi.last_error()
    rc = lib.nemo_gpu_totals_noalloc(p, p, 8, 8, 10, p, ctypes.c_uint64(0))
    assert rc == 1 and "nvars" in abi.last_error()
    rc = lib.nemo_gpu_totals_noalloc(p, p, 7, 8, 5, p, ctypes.c_uint64(0))
    assert rc == 1 and "elem_stride" in abi.last_error()
