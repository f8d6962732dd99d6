"""Host-side mirror of the reference's kernel/timedisc hook interface, on top of the C-ABI.

The reference's driver (source/driver_mod.f90:62-150) calls, per time step,
    hook_calc_timestep  -> kernel_timestep_mod::hook_calc_timestep_200   (dt from the CFL bound)
    hook_evolve         -> timedisc_evolve_mod::hook_evolve_500          (5 LSRK stages, each
                            hook_pre_rk_timestep_300 [face fluxes] + hook_mid_rk_timestep_500
                            [rkstep_cb: kernel_evolve + register update])
and hook_analyze for conserved totals.  `Solver` is the GPU module: the same hooks with the same
meaning, each a call into libnemo_gpu.so.  Errors come back as NemoError (the reference's
raise_error path); nothing here computes physics on the CPU.

States on the Python side are structure-of-arrays float64 u[V, E, n^3] (Fortran node order).
"""
import ctypes

import numpy as np

from . import abi
from .abi import call

# LSRK 5-4 (Kennedy-Carpenter 2N) coefficients as the reference's timedisc_const_mod
# (source/timedisc/rungekutta/low-storage/4-5/timedisc_const_mod.f90:5-29).
nstages = 5
a_rk = np.array([0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                 -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0])
b_rk = np.array([0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                 2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0])
c_rk = np.array([1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                 1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                 2277821191437.0 / 14882151754819.0])
dt_coeffs = b_rk


class Runtime:
    """The fields of the reference's runtime_t the hooks read and write (source/runtime_mod.f90)."""

    def __init__(self, simtime=0.0):
        self.simtime = simtime
        self.timestep = 0.0
        self.maxtimestep = 0.0
        self.rkstage = 0
        self.rktimestep = 0.0
        self.rksimtime = simtime
        self.nsteps = 0
        self.ok = True
        self.message = ""


class Solver:
    """One GPU spatial-operator instance (the library holds one per process)."""

    def __init__(self, cfg, mesh, groups=None):
        self.cfg = cfg
        self.mesh = mesh
        self.V = int(cfg.n_vars)
        self.E = mesh.E
        self.n = 4
        call("nemo_gpu_init", ctypes.byref(cfg))
        call("nemo_gpu_set_mesh", mesh.E, abi.ptr(mesh.delta), abi.ptr(mesh.center), mesh.S,
             abi.ptr(mesh.side_quads), abi.ptr(mesh.side_faceid), abi.ptr(mesh.side_nquads),
             abi.ptr(mesh.boundary))
        if groups is not None:
            g = np.ascontiguousarray(groups, dtype=np.int32)
            call("nemo_gpu_set_groups", int(g.max()) + 1, abi.ptr(g))
        self.nodes, self.weights = abi.operators()[:2]

    # ---- state transfer (SoA numpy <-> the library's per-element Fortran layout) -------------
    def upload(self, u):
        u = np.asarray(u, dtype=np.float64)
        assert u.shape == (self.V, self.E, self.n ** 3), u.shape
        aos = np.ascontiguousarray(u.transpose(1, 0, 2))
        call("nemo_gpu_upload_state", abi.ptr(aos), self.V * self.n ** 3 * 8)

    def upload_async(self, aos, stride_bytes):
        """Asynchronous upload from a pinned host buffer laid out like the reference's quad array
        (nemo_gpu_upload_state_async): taken in stream order by the steps enqueued after it."""
        call("nemo_gpu_upload_state_async", ctypes.c_void_p(aos), int(stride_bytes))

    def run_async(self, nsteps):
        """Enqueue nsteps device-dt steps without waiting (nemo_gpu_run_async)."""
        call("nemo_gpu_run_async", int(nsteps))

    def download_async(self, aos, stride_bytes):
        """Start the device->host copy of the state after the enqueued steps into a pinned host buffer
        laid out like the reference's quad array (nemo_gpu_download_state_async)."""
        call("nemo_gpu_download_state_async", ctypes.c_void_p(aos), int(stride_bytes))

    def sync(self):
        """Wait for everything enqueued (steps and copies); raise what the device reported."""
        call("nemo_gpu_sync")

    def upload_aos(self, aos, stride_bytes):
        """Upload from a host buffer laid out like the reference's quad array (per-element stride)."""
        call("nemo_gpu_upload_state", ctypes.c_void_p(aos), int(stride_bytes))

    def download(self):
        aos = np.empty((self.E, self.V, self.n ** 3))
        call("nemo_gpu_download_state", abi.ptr(aos), self.V * self.n ** 3 * 8)
        return np.ascontiguousarray(aos.transpose(1, 0, 2))

    # ---- hooks ---------------------------------------------------------------------------------
    def calc_timestep(self, cfl=None):
        dt, lm = ctypes.c_double(), ctypes.c_double()
        call("nemo_gpu_calc_timestep", float(cfl if cfl is not None else self.cfg.cfl), ctypes.byref(dt),
             ctypes.byref(lm))
        return dt.value, lm.value

    def stage(self, stage, dt, t_stage=0.0):
        nbad = ctypes.c_int32(0)
        call("nemo_gpu_stage", int(stage), float(dt), float(t_stage), ctypes.byref(nbad))
        return nbad.value

    def step(self, dt):
        call("nemo_gpu_step", float(dt))

    def run(self, nsteps=0, t_end=0.0):
        t, s = ctypes.c_double(), ctypes.c_int64()
        call("nemo_gpu_run", int(nsteps), float(t_end), ctypes.byref(t), ctypes.byref(s))
        return t.value, s.value

    def rhs(self):
        aos = np.empty((self.E, self.V, self.n ** 3))
        call("nemo_gpu_rhs", abi.ptr(aos))
        return np.ascontiguousarray(aos.transpose(1, 0, 2))

    def alpha(self):
        a = np.empty(self.E)
        call("nemo_gpu_alpha", abi.ptr(a))
        return a

    def autotune(self, nsteps=3):
        """Pick the stage schedule by timing (FP32 Euler form); returns (mode, ctas, ms per step of
        each candidate)."""
        mode, ctas = ctypes.c_int32(), ctypes.c_int32()
        ms = np.zeros(8)
        call("nemo_gpu_autotune", int(nsteps), ctypes.byref(mode), ctypes.byref(ctas), abi.ptr(ms))
        return mode.value, ctas.value, ms

    def set_schedule(self, mode, ctas=0):
        call("nemo_gpu_set_schedule", int(mode), int(ctas))

    def amr_flags(self, refine_threshold, coarsen_threshold):
        """Adapt flags of the current state from the device density probe (nemo_gpu_amr_flags)."""
        f = np.empty(self.E, dtype=np.int32)
        call("nemo_gpu_amr_flags", float(refine_threshold), float(coarsen_threshold), abi.ptr(f))
        return f

    def adapt(self, flags, min_level=0):
        """One forest adapt step (mesh.adapt): new mesh, state remapped on the device; returns the
        new mesh and its remap rows."""
        from . import mesh as mesh_mod
        new, remap = mesh_mod.adapt(self.mesh, flags, min_level=min_level)
        remap = np.ascontiguousarray(remap, dtype=np.int32)
        if new.E == self.E and not np.any(remap[:, 0]):   # nothing changed
            return self.mesh, remap
        call("nemo_gpu_adapt", new.E, abi.ptr(new.delta), abi.ptr(new.center), new.S, abi.ptr(new.side_quads),
             abi.ptr(new.side_faceid), abi.ptr(new.side_nquads), abi.ptr(new.boundary), abi.ptr(remap))
        self.mesh, self.E = new, new.E
        return new, remap

    def run_amr(self, nsteps, every, refine_threshold, coarsen_threshold, min_level=0):
        """nsteps steps with an adapt before every `every`-th (hook_pre_timestep_300 of the Sedov setup,
        source/setups/euler/3d/sedov/setup_amr_mod.f90:7-21): device density flags, host forest
        rebuild, device remap.  Returns (t, number of elements after each adapt)."""
        sizes, done, t = [], 0, 0.0
        while done < nsteps:
            self.adapt(self.amr_flags(refine_threshold, coarsen_threshold), min_level=min_level)
            sizes.append(self.E)
            k = min(every, nsteps - done)
            t, _ = self.run(nsteps=k)
            done += k
        return t, sizes

    def totals(self):
        out = np.zeros(10)
        call("nemo_gpu_totals", abi.ptr(out))
        return out[: self.V]

    def status(self):
        t, nb = ctypes.c_double(), ctypes.c_int64()
        call("nemo_gpu_status", ctypes.byref(t), ctypes.byref(nb))
        return t.value, nb.value

    def finalize(self):
        call("nemo_gpu_finalize")

    # reference-named hooks ------------------------------------------------------------------------
    def hook_calc_timestep_200(self, rt, cfl=None):
        """kernel_timestep_mod::hook_calc_timestep_200 (source/kernel/mcfv/3d/kernel_timestep_mod.f90:17-58)."""
        rt.maxtimestep, _ = self.calc_timestep(cfl)
        return rt.maxtimestep

    def hook_pre_rk_timestep_300(self, rt):
        """Face fill + face flux (kernel_hooks_mod.f90:7-20): fused into the stage kernel; no-op."""

    def hook_mid_rk_timestep_500(self, rt):
        """rkstep_cb over all quads (timedisc_hooks_mod.f90:19-58): one fused stage launch."""
        try:
            self.stage(rt.rkstage, rt.timestep, rt.rksimtime)
        except abi.NemoError as exc:
            rt.ok, rt.message = False, str(exc)

    def hook_evolve_500(self, rt):
        """The stage loop of timedisc_evolve_mod::hook_evolve_500 (timedisc_evolve_mod.f90:20-84)."""
        for stage in range(1, nstages + 1):
            rt.rkstage = stage
            rt.rktimestep = rt.timestep * dt_coeffs[stage - 1]
            rt.rksimtime = rt.simtime + rt.rktimestep
            self.hook_pre_rk_timestep_300(rt)
            self.hook_mid_rk_timestep_500(rt)
            if not rt.ok:
                return

    def mainloop(self, rt, stop_time, max_steps=None):
        """driver_mod::mainloop (source/driver_mod.f90:62-150) without I/O: dt, clamp, evolve."""
        while rt.simtime < stop_time and (max_steps is None or rt.nsteps < max_steps):
            self.hook_calc_timestep_200(rt)
            rt.timestep = min(rt.maxtimestep, stop_time - rt.simtime)
            self.hook_evolve_500(rt)
            if not rt.ok:
                break
            rt.simtime = rt.simtime + rt.timestep
            rt.nsteps += 1
        return rt
