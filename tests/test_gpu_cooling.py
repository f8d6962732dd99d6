"""Barotropic cooling on the GPU: applied after every stage inside the stage kernels, the plain FP64
path equals the oracle bit for bit over a run, the FP32 form stays within FP32 tolerance, and the
configuration is checked at init."""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
KAP = 5.0 / 3.0


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


def ccfg(**kw):
    base = dict(kappa=KAP, indicator=abi.IND_MODAL, positivity=1, source=abi.SOURCE_BAROTROPIC_COOLING,
                dens_critical=1.0, k_isothermal=1.0, k_adiabatic=1.0)
    base.update(kw)
    return abi.default_cfg(**base)


def test_cooled_run_bit_exact():
    m = mesh.brick(6)
    u = setups.smooth_random(m, seed=6, kappa=KAP)
    c = ccfg()
    s = Solver(c, m)
    s.upload(u)
    t, n = s.run(nsteps=5)
    ref, tr, nr, _ = orc.Oracle(c, m.neighbors(), m.delta).run(u, nsteps=5)
    assert n == nr == 5 and t == tr
    assert np.array_equal(s.download(), ref)


def test_cooled_fp32_form_close():
    m = mesh.brick(6)
    u = setups.smooth_random(m, seed=6, kappa=KAP)
    s = Solver(ccfg(precision=abi.PREC_FP32), m)
    s.upload(u)
    s.run(nsteps=5)
    got = s.download()
    ref, _, _, _ = orc.Oracle(ccfg(), m.neighbors(), m.delta).run(u, nsteps=5)
    for v in (0, 4):
        assert np.sum(np.abs(got[v] - ref[v])) / np.sum(np.abs(ref[v])) < 1e-6


def test_cooling_configuration_checks():
    m = mesh.brick(2)
    with pytest.raises(abi.NemoError, match="dens_critical"):
        Solver(ccfg(k_adiabatic=0.0), m)
    with pytest.raises(abi.NemoError, match="Euler"):
        Solver(ccfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_RUSANOV,
                    mu0=1.0), m)
