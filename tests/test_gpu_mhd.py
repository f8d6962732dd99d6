"""GPU parity of the GLM-MHD stage kernels against the FP64 oracle: the plain path bit for bit
(rhs, host-driven stages, device-driven steps with the per-step GLM cleaning speed, blended runs),
the FP32 form within FP32 tolerances."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
K = 5.0 / 3.0


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


def mcfg(**kw):
    base = dict(n_vars=9, eqn=abi.EQN_MHD, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_RUSANOV,
                kappa=K, mu0=1.0, glm_ch=0.7, glm_alpha=0.3)
    base.update(kw)
    return abi.default_cfg(**base)


def rel_linf(a, b):
    return max(np.max(np.abs(a[v] - b[v])) / max(np.max(np.abs(b[v])), 1e-300) for v in range(a.shape[0]))


@pytest.mark.parametrize("vf,sf", [(abi.VOLFLUX_EC_MHD, abi.SURFFLUX_RUSANOV), (abi.VOLFLUX_CENTRAL, abi.SURFFLUX_RUSANOV),
                                   (abi.VOLFLUX_EC_MHD, abi.SURFFLUX_HLLD)])
def test_mhd_rhs_bit_exact(vf, sf):
    m = mesh.brick(4)
    u = setups.orszag_tang(m)
    u[8] = 0.01 * np.sin(3.0 * u[0] * np.arange(m.E)[:, None])     # a nonzero psi field
    c = mcfg(volume_flux=vf, surface_flux=sf)
    s = Solver(c, m)
    s.upload(u)
    r = s.rhs()
    ref = orc.Oracle(c, m.neighbors(), m.delta).rhs(u)
    assert np.array_equal(r, ref), rel_linf(r, ref)


def test_mhd_run_bit_exact_with_device_glm():
    m = mesh.brick(4)
    u = setups.orszag_tang(m)
    c = mcfg()
    s = Solver(c, m)
    s.upload(u)
    t, n = s.run(nsteps=5)
    uc, tc, nc, _ = orc.Oracle(c, m.neighbors(), m.delta).run(u, nsteps=5)
    assert n == nc == 5 and t == tc
    assert np.array_equal(s.download(), uc)


@pytest.mark.parametrize("sf", [abi.SURFFLUX_RUSANOV, abi.SURFFLUX_HLLD])
def test_mhd_blended_run_bit_exact(sf):
    m = mesh.brick(4)
    u = setups.orszag_tang(m)
    c = mcfg(indicator=abi.IND_MODAL, positivity=1, surface_flux=sf)
    s = Solver(c, m)
    s.upload(u)
    o = orc.Oracle(c, m.neighbors(), m.delta)
    assert np.array_equal(s.alpha(), o.alpha(u))
    t, n = s.run(nsteps=4)
    uc, tc, nc, _ = o.run(u, nsteps=4)
    assert np.array_equal(s.download(), uc)


@pytest.mark.parametrize("sf", [abi.SURFFLUX_RUSANOV, abi.SURFFLUX_HLLD])
def test_mhd_fp32_form_close_to_oracle(sf):
    m = mesh.brick(8)
    u = setups.orszag_tang(m)
    c = mcfg(precision=abi.PREC_FP32, surface_flux=sf)
    s = Solver(c, m)
    s.upload(u)
    o = orc.Oracle(c, m.neighbors(), m.delta)
    r, ref = s.rhs(), o.rhs(u)
    # relative to the largest rhs entry: the rotated-out components (B_z, m_z) and psi of this
    # z-independent, discretely divergence-free state have FP64 rhs at round-off level only
    assert np.max(np.abs(r - ref)) / np.max(np.abs(ref)) < 1e-5
    t, n = s.run(nsteps=10)
    uc, tc, nc, _ = o.run(u, nsteps=10)
    got = s.download()
    assert np.sum(np.abs(got[0] - uc[0])) / np.sum(np.abs(uc[0])) < 1e-6


def test_hlld_requires_unit_mu0():
    m = mesh.brick(2)
    with pytest.raises(abi.NemoError, match="mu0"):
        Solver(mcfg(surface_flux=abi.SURFFLUX_HLLD, mu0=2.0), m)


def test_mhd_fp32_learned_indicator_close_to_fp64():
    """FP32 form with the learned indicator (parallel 16-lane feature sums) against the plain FP64
    form with the same BF16 network, which equals the oracle bit for bit."""
    from nemo_b200 import learned
    m = mesh.brick(8)
    u = setups.orszag_tang(m)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_FP32):
        s = Solver(mcfg(precision=prec, indicator=abi.IND_LEARNED, positivity=1, surface_flux=abi.SURFFLUX_HLLD), m)
        learned.install()
        s.upload(u)
        out[prec] = (s.alpha(), None)
        s.run(nsteps=5)
        out[prec] = (out[prec][0], s.download())
        s.finalize()
    a64, u64 = out[abi.PREC_FP64]
    a32, u32 = out[abi.PREC_FP32]
    assert np.max(np.abs(a32 - a64)) < 1e-3
    assert np.sum(np.abs(u32[0] - u64[0])) / np.sum(np.abs(u64[0])) < 1e-6
