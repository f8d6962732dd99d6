"""GPU tests of the asynchronous path through the C-ABI: nemo_gpu_upload_state_async,
nemo_gpu_run_async and nemo_gpu_download_state_async (two staging slots each way).  States streamed through
the library this way give, bit for bit, what the synchronous calls give, each download matching its
own upload even when the uploads of later states are already in flight."""
import ctypes

import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


def pinned_aos(u):
    import torch
    t = torch.empty(u.size, dtype=torch.float64, pin_memory=True)
    t.numpy()[:] = np.ascontiguousarray(u.transpose(1, 0, 2)).ravel()
    return t


def serial(s, u, nsteps):
    s.upload(u)
    s.run(nsteps=nsteps)
    return s.download()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_FP32])
def test_streamed_states_match_the_synchronous_calls(precision):
    import torch
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    ua = setups.sedov(m, sigma=0.05)
    ub = setups.sedov(m, sigma=0.08)
    s = Solver(abi.default_cfg(precision=precision, indicator=abi.IND_MODAL, positivity=1), m)
    ref_a, ref_b = serial(s, ua, 3), serial(s, ub, 3)
    row = 5 * 64 * 8
    ins = [pinned_aos(ua), pinned_aos(ub), pinned_aos(ua)]
    outs = [torch.zeros(ua.size, dtype=torch.float64, pin_memory=True) for _ in ins]
    for hin, hout in zip(ins, outs):
        s.upload_async(hin.data_ptr(), row)
        s.run_async(3)
        s.download_async(hout.data_ptr(), row)
    s.sync()
    got = [o.numpy().reshape(m.E, 5, 64).transpose(1, 0, 2) for o in outs]
    assert np.array_equal(got[0], ref_a)
    assert np.array_equal(got[1], ref_b)
    assert np.array_equal(got[2], ref_a)
    # the library state after the stream is the last state's result, and a synchronous run continues it
    assert np.array_equal(s.download(), ref_a)


def test_run_async_needs_a_state_and_rejects_timing_mode():
    m = mesh.brick(4)
    s = Solver(abi.default_cfg(), m)
    with pytest.raises(abi.NemoError):
        s.run_async(1)
    s.upload(setups.density_wave(m, seed=1))
    abi.call("nemo_gpu_set_timing", 1)
    with pytest.raises(abi.NemoError):
        s.run_async(1)
    abi.call("nemo_gpu_set_timing", 0)
    s.run_async(2)
    s.sync()
    t, _ = s.status()
    assert t > 0
