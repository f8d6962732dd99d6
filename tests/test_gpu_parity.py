"""GPU parity: the CUDA path (through the C-ABI) against the FP64 oracle on the same seeded inputs.

Tolerance of the plain FP64 path: 1e-12 relative L-infinity (per variable, relative to the
variable's max magnitude); conserved totals to round-off.  The plain path is compiled without
FMA contraction and evaluates the oracle's expressions in the same order, so most differences
are zero (log and exp are the same IEEE-only construction on both sides).
"""
import numpy as np
import pytest

from nemo_b200 import abi, mesh, setups
from nemo_b200.solver import Solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-12
KAPPA = 1.4


def cfg(**kw):
    return abi.default_cfg(**kw)


def rel_linf(a, b):
    """max over variables of max|a-b| / max|b|."""
    out = 0.0
    for v in range(a.shape[0]):
        scale = max(np.max(np.abs(b[v])), 1e-300)
        out = max(out, np.max(np.abs(a[v] - b[v])) / scale)
    return out


def make(c, m, groups=None):
    s = Solver(c, m, groups)
    o = orc.Oracle(c, m.neighbors(), m.delta)
    return s, o


@pytest.fixture(autouse=True)
def _fin():
    yield
    try:
        abi.call("nemo_gpu_finalize")
    except Exception:
        pass


@pytest.mark.parametrize("nx,vf,sf", [(4, 0, 0), (4, 1, 0), (4, 0, 1), (8, 0, 0)])
def test_rhs_parity_density_wave(nx, vf, sf):
    m = mesh.brick(nx)
    u = setups.density_wave(m, seed=nx)
    s, o = make(cfg(volume_flux=vf, surface_flux=sf), m)
    s.upload(u)
    r_gpu, r_cpu = s.rhs(), o.rhs(u)
    assert rel_linf(r_gpu, r_cpu) <= TOL
    assert np.array_equal(s.download(), u)


@pytest.mark.parametrize("vf,sf", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_rhs_parity_distinct_velocities(vf, sf):
    """All three momentum components differ, so every rotation of the direction wrappers matters."""
    m = mesh.brick(4)
    u = setups.smooth_random(m, seed=7)
    s, o = make(cfg(volume_flux=vf, surface_flux=sf), m)
    s.upload(u)
    r_gpu, r_cpu = s.rhs(), o.rhs(u)
    assert rel_linf(r_gpu, r_cpu) <= TOL
    assert np.array_equal(r_gpu, r_cpu)      # the plain path is bit-exact


def test_stage_by_stage_bit_exact():
    m = mesh.brick(4)
    u = setups.smooth_random(m, seed=8)
    s, o = make(cfg(), m)
    s.upload(u)
    dt, _ = o.timestep(u)
    uc, reg = u.copy(), np.zeros_like(u)
    for st in range(5):
        o.stage(uc, reg, st, dt)
        s.stage(st + 1, dt)
        assert np.array_equal(s.download(), uc), st


def test_rhs_parity_ragged_and_open_boundaries():
    """E = 105 (not a multiple of the 8-element tile) and non-periodic faces (mirrored states)."""
    m = mesh.brick(3, 5, 7, periodic=(False, True, False))
    u = setups.density_wave(m, seed=5)
    s, o = make(cfg(), m)
    s.upload(u)
    assert rel_linf(s.rhs(), o.rhs(u)) <= TOL


def test_rhs_parity_blended_sedov():
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    c = cfg(indicator=abi.IND_MODAL, positivity=1)
    s, o = make(c, m)
    s.upload(u)
    a_gpu, a_cpu = s.alpha(), o.alpha(u)
    assert np.max(np.abs(a_gpu - a_cpu)) <= 1e-12
    assert a_cpu.max() > 0
    assert rel_linf(s.rhs(), o.rhs(u, alpha=a_cpu)) <= TOL


def test_stage_sequence_parity_fixed_dt():
    m = mesh.brick(4)
    u = setups.density_wave(m, seed=9)
    s, o = make(cfg(), m)
    s.upload(u)
    dt, _ = o.timestep(u)
    uc, reg = u.copy(), np.zeros_like(u)
    for _ in range(3):
        s.step(dt)
        for st in range(5):
            o.stage(uc, reg, st, dt)
    assert rel_linf(s.download(), uc) <= TOL


def test_run_parity_100_steps_config1_small():
    """The benchmark's smooth case (config 1 form) on 4^3 elements, 100 steps, device dt."""
    m = mesh.brick(4)
    u = setups.density_wave(m, seed=1234)
    s, o = make(cfg(cfl=0.5), m)
    s.upload(u)
    t_gpu, n_gpu = s.run(nsteps=100)
    uc, t_cpu, n_cpu, nbad = o.run(u, nsteps=100)
    assert n_gpu == n_cpu == 100
    assert abs(t_gpu - t_cpu) <= 1e-14 * t_cpu
    assert rel_linf(s.download(), uc) <= TOL
    # conservation to round-off on the periodic mesh
    tot0, tot1 = o.totals(u), s.totals()
    assert np.max(np.abs(tot1 - tot0)) <= 1e-13 * np.max(np.abs(tot0))
    np.testing.assert_array_equal(s.totals(), o.totals(s.download()))


def test_run_parity_sedov_blended_to_t_end():
    m = mesh.brick(8, lo=(-0.5,) * 3, hi=(0.5,) * 3)
    u = setups.sedov(m, sigma=0.05)
    c = cfg(indicator=abi.IND_MODAL, positivity=1, cfl=0.5)
    s, o = make(c, m)
    s.upload(u)
    t_end = 2e-3
    t_gpu, n_gpu = s.run(t_end=t_end)
    uc, t_cpu, n_cpu, nbad = o.run(u, t_end=t_end)
    assert n_gpu == n_cpu and abs(t_gpu - t_end) < 1e-15 and abs(t_cpu - t_end) < 1e-15
    assert rel_linf(s.download(), uc) <= TOL
    assert s.status()[1] == nbad == 0


def test_calc_timestep_parity():
    m = mesh.brick(4)
    u = setups.density_wave(m, seed=3)
    s, o = make(cfg(cfl=0.5), m)
    s.upload(u)
    dt_g, lm_g = s.calc_timestep()
    dt_c, lm_c = o.timestep(u)
    assert dt_g == dt_c and lm_g == lm_c


def test_repair_path_parity():
    """A stage whose update leaves inadmissible nodes: the GPU repair equals the oracle's."""
    m = mesh.brick(4)
    x = m.node_coords(setups.LGL4)[0]
    one = np.ones_like(x)
    u = np.ascontiguousarray(setups.prim2cons(one, np.where(x < 0.5, -3.0, 3.0), 0 * one, 0 * one, 0.05 * one,
                                              KAPPA))
    c = cfg(positivity=1)
    s, o = make(c, m)
    s.upload(u)
    dt, _ = o.timestep(u)
    uc, reg = u.copy(), np.zeros_like(u)
    nb_c = o.stage(uc, reg, 0, 32 * dt)
    nb_g = s.stage(1, 32 * dt)
    assert nb_c == nb_g == 0
    assert rel_linf(s.download(), uc) <= TOL
    # a step size at which the repair cannot succeed: counted and reported as ERR_REPAIR
    s.upload(u)
    uc, reg = u.copy(), np.zeros_like(u)
    nb_c = o.stage(uc, reg, 0, 64 * dt)
    with pytest.raises(abi.NemoError) as ei:
        s.stage(1, 64 * dt)
    assert ei.value.code == 4 and nb_c > 0
    assert s.status()[1] == nb_c


def test_hook_mainloop_matches_run():
    """The reference-named hook path (driver mainloop) gives the same state as nemo_gpu_run."""
    from nemo_b200.solver import Runtime
    m = mesh.brick(4)
    u = setups.density_wave(m, seed=2)
    s, o = make(cfg(), m)
    s.upload(u)
    rt = s.mainloop(Runtime(), stop_time=1e9, max_steps=5)
    a = s.download()
    s.upload(u)
    s.run(nsteps=5)
    assert rt.ok and rt.nsteps == 5
    assert rel_linf(a, s.download()) <= TOL


def test_upload_strided_like_quad_array():
    """Upload from a host array with a per-element stride larger than the state (quad_t layout)."""
    m = mesh.brick(2)
    u = setups.density_wave(m, seed=4)
    s, _ = make(cfg(), m)
    pad = 37  # doubles of other quad_t members after each element's state
    host = np.zeros((m.E, 5 * 64 + pad))
    host[:, :320] = u.transpose(1, 0, 2).reshape(m.E, 320)
    s.upload_aos(host.ctypes.data, host.strides[0])
    assert np.array_equal(s.download(), u)


def test_error_paths():
    m = mesh.brick(2)
    s, _ = make(cfg(), m)
    with pytest.raises(abi.NemoError) as ei:
        s.rhs()                                   # no state yet
    assert ei.value.code == 2
    with pytest.raises(abi.NemoError):
        s.stage(7, 1e-3)
    bad = m.side_faceid.copy()
    bad[0, 1] = bad[0, 0]                         # same face on both halves
    import ctypes
    rc = abi.load().nemo_gpu_set_mesh(m.E, abi.ptr(m.delta), abi.ptr(m.center), m.S, abi.ptr(m.side_quads),
                                      abi.ptr(bad), abi.ptr(m.side_nquads), abi.ptr(m.boundary))
    assert rc == 1
    del ctypes
