"""GPU test of nemo_gpu_totals_noalloc, the totals entry point that allocates nothing.

It exists for hosts that cannot allocate device memory when they ask for the conserved totals:
their device arrays belong to their own pool (for example a Fortran/OpenACC data region sized at
start-up) or they run under a fixed device-memory budget where cudaMalloc/cudaFree mid-run would
fail or synchronise the device.  The caller owns the state and the output in device memory; the
library keeps its partial sums in a fixed array of its own.

Checked here through the C-ABI: two calls in a row, on two different states, each equal to what
the allocating entry point (nemo_gpu_totals) returns for the same state -- to the totals tolerance
of the other tests (1e-13 relative), and in fact bit for bit, since both run the same arithmetic.
This file is collected last so that a stop at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver

pytestmark = pytest.mark.gpu


def totals_allocating(c, m, u):
    s = Solver(c, m)
    s.upload(u)
    out = s.totals()
    s.finalize()
    return out


def test_totals_noalloc_matches_allocating_entry_point_twice():
    import torch
    m1 = mesh.brick(8)
    u1 = setups.smooth_random(m1, seed=21)
    m2 = mesh.brick(16, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u2 = setups.sedov(m2, sigma=0.05)
    c = abi.default_cfg()
    refs = [totals_allocating(c, m1, u1), totals_allocating(c, m2, u2)]

    lib = abi.load()
    stream = torch.cuda.current_stream().cuda_stream
    for (m, u), ref in zip(((m1, u1), (m2, u2)), refs):
        u_dev = torch.from_numpy(np.ascontiguousarray(u)).cuda()          # [V][E][64], caller-owned
        d_dev = torch.from_numpy(np.ascontiguousarray(m.delta)).cuda()    # [E][3]
        out_dev = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.nemo_gpu_totals_noalloc(ctypes.c_void_p(u_dev.data_ptr()), ctypes.c_void_p(d_dev.data_ptr()),
                                         m.E, 5, ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_uint64(stream))
        assert rc == 0, abi.last_error()
        torch.cuda.synchronize()
        got = out_dev.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
        assert np.array_equal(got, ref)


def test_totals_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = abi.load()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = lib.nemo_gpu_totals_noalloc(p, p, 65537, 5, p, ctypes.c_uint64(0))
    assert rc == 1 and "65536" in abi.last_error()
    rc = lib.nemo_gpu_totals_noalloc(p, p, 8, 10, p, ctypes.c_uint64(0))
    assert rc == 1 and "nvars" in abi.last_error()
