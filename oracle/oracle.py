"""ctypes wrapper of the CPU FP64 oracle (liboracle.so, built from nemo_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's
CPU-baseline leg, never by the nemo_b200 package.  See nemo_oracle.cpp for what the oracle
restates and how far its parity with the reference is pinned.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


# Build variants of the oracle (oracle/Makefile): "" the oracle, "libm" with the C library's log/exp
# (the reference's intrinsic arithmetic), "count" with the algorithmic operation counter, "fma" with
# the C library's log/exp and FMA contraction (an optimising build of the reference).
VARIANTS = {"": "liboracle.so", "libm": "liboracle_libm.so", "count": "liboracle_count.so",
            "fma": "liboracle_fma.so"}
_VLIB = {}


def build(force=False):
    srcs = [os.path.join(_HERE, f) for f in ("nemo_oracle.cpp", "opcount.cpp", "Makefile")]
    newest = max(os.path.getmtime(f) for f in srcs)
    sos = [os.path.join(_HERE, f) for f in VARIANTS.values()]
    if force or any(not os.path.exists(so) or os.path.getmtime(so) < newest for so in sos):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return sos[0]


def lib(variant=""):
    """The oracle's shared library (variant "" / "libm" / "count", see VARIANTS)."""
    global _LIB
    if variant:
        if variant not in _VLIB:
            _VLIB[variant] = _load(os.path.join(_HERE, VARIANTS[variant]))
        return _VLIB[variant]
    if _LIB is None:
        _LIB = _load(os.path.join(_HERE, VARIANTS[""]))
    return _LIB


def _load(so):
    if not os.path.exists(so):
        build()
    L = ctypes.CDLL(so)
    L.or_logmean.restype = ctypes.c_double
    L.or_logmean.argtypes = [ctypes.c_double, ctypes.c_double]
    L.or_pressure.restype = ctypes.c_double
    L.or_pressure.argtypes = [_dp, ctypes.c_double]
    L.or_flux.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double]
    L.or_riemann.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double]
    L.or_twopoint.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double]
    L.or_lgl.argtypes = [ctypes.c_int, _dp, _dp]
    L.or_operators.argtypes = [_dp] * 5
    L.or_mortar_operators.argtypes = [_dp, _dp]
    L.or_set_mortars.argtypes = [ctypes.c_int64, ctypes.c_void_p]
    L.or_remap.argtypes = [ctypes.c_int, ctypes.c_int64, _dp, ctypes.c_int64, ctypes.c_void_p, ctypes.c_double,
                           ctypes.c_double, _dp]
    L.or_rk_coeffs.argtypes = [_dp] * 3
    L.or_alpha.argtypes = [ctypes.c_void_p, ctypes.c_int64, _ip, _dp, _dp, _dp, ctypes.c_int]
    L.or_rhs.argtypes = [ctypes.c_void_p, ctypes.c_int64, _ip, _dp, _dp, ctypes.c_void_p, _dp,
                         ctypes.c_int]
    L.or_timestep.restype = ctypes.c_double
    L.or_timestep.argtypes = [ctypes.c_void_p, ctypes.c_int64, _dp, _dp, _dp]
    L.or_stage.restype = ctypes.c_int64
    L.or_stage.argtypes = [ctypes.c_void_p, ctypes.c_int64, _ip, _dp, ctypes.c_int,
                           ctypes.c_double, _dp, _dp, ctypes.c_int]
    L.or_run.restype = ctypes.c_int64
    L.or_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, _ip, _dp, _dp, ctypes.c_int64,
                         ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
    L.or_totals.argtypes = [ctypes.c_void_p, ctypes.c_int64, _dp, _dp, _dp]
    L.or_max_threads.restype = ctypes.c_int
    L.or_log.restype = ctypes.c_double
    L.or_log.argtypes = [ctypes.c_double]
    L.or_exp.restype = ctypes.c_double
    L.or_exp.argtypes = [ctypes.c_double]
    L.or_set_mlp.argtypes = [_dp, _dp, _dp]
    L.or_mhd_flux.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.or_mhd_riemann.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.or_mhd_twopoint.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double]
    L.or_mhd_nc.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double]
    L.or_mhd_pressure.restype = ctypes.c_double
    L.or_mhd_pressure.argtypes = [_dp, ctypes.c_double, ctypes.c_double]
    L.or_timestep2.restype = ctypes.c_double
    L.or_timestep2.argtypes = [ctypes.c_void_p, ctypes.c_int64, _dp, _dp, _dp, _dp]
    L.or_features.argtypes = [ctypes.c_void_p, ctypes.c_int64, _dp, _dp, ctypes.c_void_p, ctypes.c_int]
    L.or_mlp_alpha.restype = ctypes.c_double
    L.or_mlp_alpha.argtypes = [ctypes.c_void_p, _dp]
    L.or_repair.restype = ctypes.c_int
    L.or_repair.argtypes = [ctypes.c_void_p, _dp]
    if hasattr(L, "or_opcount_read"):
        L.or_opcount_read.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
    return L


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def nthreads_default():
    return int(lib().or_max_threads())


def operators():
    n = 4
    x, w = np.zeros(n), np.zeros(n)
    D, S, Vi = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    lib().or_operators(_p(x), _p(w), _p(D), _p(S), _p(Vi))
    return x, w, D, S, Vi


def mortar_operators():
    """(prolongation [2,4,4], projection [2,4,4]) of the 2:1 mortar, lower/upper half."""
    pro, prj = np.zeros((2, 4, 4)), np.zeros((2, 4, 4))
    lib().or_mortar_operators(_p(pro), _p(prj))
    return pro, prj


def amr_flags(u, refine_threshold, coarsen_threshold):
    """Density probes of the Sedov setup (source/setups/euler/3d/sedov/setup_amr_mod.f90:23-65) per
    element: +1 if any node's density > refine_threshold, else -1 if none > coarsen_threshold, else 0."""
    dmax = np.asarray(u)[0].max(axis=1)
    return np.where(dmax > refine_threshold, 1, np.where(dmax > coarsen_threshold, 0, -1)).astype(np.int32)


def remap(u, remap_rows, kappa=1.4, mu0=1.0):
    """State [V, E_old, 64] -> [V, E_new, 64] by adapt remap rows (mesh.adapt); inadmissible
    transferred elements fall back to the conservative means (V = 9: GLM-MHD admissibility)."""
    u = _f64(u)
    r = np.ascontiguousarray(remap_rows, dtype=np.int32)
    out = np.zeros((u.shape[0], len(r), 64))
    lib().or_remap(u.shape[0], u.shape[1], _p(u), len(r), r.ctypes.data, float(kappa), float(mu0), _p(out))
    return out


def lgl(N):
    x, w = np.zeros(N + 1), np.zeros(N + 1)
    lib().or_lgl(N, _p(x), _p(w))
    return x, w


def rk_coeffs():
    a, b, c = np.zeros(5), np.zeros(5), np.zeros(5)
    lib().or_rk_coeffs(_p(a), _p(b), _p(c))
    return a, b, c


def set_mlp(w, lo, hi):
    """Weights (1505, FP64 values of the BF16-rounded weights the GPU uses) and input bounds."""
    w, lo, hi = _f64(w), _f64(lo), _f64(hi)
    lib().or_set_mlp(_p(w), _p(lo), _p(hi))


def features(cfg, u):
    u = _f64(u)
    E = u.shape[1]
    f = np.zeros((E, 12))
    a = np.zeros(E)
    lib().or_features(ctypes.byref(cfg), E, _p(u), _p(f), a.ctypes.data, nthreads_default())
    return f, a


def mlp_alpha(cfg, feat):
    feat = _f64(feat)
    return lib().or_mlp_alpha(ctypes.byref(cfg), _p(feat))


def mhd_flux(d, u, kappa=5 / 3, mu0=1.0, ch=0.0):
    u = _f64(u)
    f = np.zeros(9)
    lib().or_mhd_flux(d, _p(u), _p(f), kappa, mu0, ch)
    return f


def mhd_riemann(d, uL, uR, kappa=5 / 3, mu0=1.0, ch=0.0, kind=1):
    """MHD surface flux in direction d: kind 1 Rusanov, 2 HLLD (mu0 = 1)."""
    uL, uR = _f64(uL), _f64(uR)
    f = np.zeros(9)
    lib().or_mhd_riemann(kind, d, _p(uL), _p(uR), _p(f), kappa, mu0, ch)
    return f


def mhd_twopoint(kind, d, u, v, kappa=5 / 3, mu0=1.0, ch=0.0):
    u, v = _f64(u), _f64(v)
    f = np.zeros(9)
    lib().or_mhd_twopoint(kind, d, _p(u), _p(v), _p(f), kappa, mu0, ch)
    return f


def mhd_nc(d, ui, ul, ur, kappa=5 / 3, mu0=1.0):
    ui, ul, ur = _f64(ui), _f64(ul), _f64(ur)
    f = np.zeros(9)
    lib().or_mhd_nc(d, _p(ui), _p(ul), _p(ur), _p(f), kappa, mu0)
    return f


def repair(cfg, st):
    """Positivity repair of one element st[V,64] (copy returned) and whether it succeeded."""
    st = _f64(st).copy()
    ok = lib().or_repair(ctypes.byref(cfg), _p(st))
    return st, bool(ok)


def logmean(a, b):
    return lib().or_logmean(float(a), float(b))


def pressure(u, kappa=1.4):
    u = _f64(u)
    return lib().or_pressure(_p(u), kappa)


def flux(d, u, kappa=1.4):
    u = _f64(u)
    f = np.zeros(5)
    lib().or_flux(d, _p(u), _p(f), kappa)
    return f


def riemann(kind, d, uL, uR, kappa=1.4):
    uL, uR = _f64(uL), _f64(uR)
    f = np.zeros(5)
    lib().or_riemann(kind, d, _p(uL), _p(uR), _p(f), kappa)
    return f


def twopoint(kind, d, u, v, kappa=1.4):
    u, v = _f64(u), _f64(v)
    f = np.zeros(5)
    lib().or_twopoint(kind, d, _p(u), _p(v), _p(f), kappa)
    return f


class Oracle:
    """Oracle bound to one configuration and mesh (nbr = per-element face neighbours with the mortar
    encoding of Mesh.neighbors(); mortars = Mesh.mortars() for a 2:1 forest)."""

    def __init__(self, cfg, nbr, delta, nthreads=None, mortars=None, variant=""):
        self.lib = lib(variant)              # "": the oracle; "libm" / "count": its build variants
        self.cfg = cfg                       # a nemo_b200.abi.NemoCfg (ctypes struct)
        self.nbr = np.ascontiguousarray(nbr, dtype=np.int32)
        self.delta = _f64(delta)
        self.E = self.nbr.shape[0]
        self.V = int(cfg.n_vars)
        self.nthreads = nthreads or int(self.lib.or_max_threads())
        self.mortars = np.ascontiguousarray(np.zeros((0, 6)) if mortars is None else mortars, dtype=np.int32)
        if (self.nbr <= -2).any() and len(self.mortars) == 0:
            raise ValueError("mesh has mortar faces: pass mortars=mesh.mortars()")

    @classmethod
    def for_mesh(cls, cfg, mesh, nthreads=None, variant=""):
        return cls(cfg, mesh.neighbors(), mesh.delta, nthreads=nthreads, mortars=mesh.mortars(), variant=variant)

    def _c(self):
        self.lib.or_set_mortars(len(self.mortars), self.mortars.ctypes.data)
        return ctypes.byref(self.cfg)

    def alpha(self, u):
        u = _f64(u)
        a = np.zeros(self.E)
        self.lib.or_alpha(self._c(), self.E, _p(self.nbr, _ip), _p(self.delta), _p(u), _p(a), self.nthreads)
        return a

    def rhs(self, u, alpha=None):
        u = _f64(u)
        r = np.zeros_like(u)
        ap = None
        if alpha is not None:
            alpha = _f64(alpha)
            ap = alpha.ctypes.data
        self.lib.or_rhs(self._c(), self.E, _p(self.nbr, _ip), _p(self.delta), _p(u), ap, _p(r), self.nthreads)
        return r

    def timestep(self, u):
        u = _f64(u)
        lm = ctypes.c_double(0)
        dt = self.lib.or_timestep(self._c(), self.E, _p(self.delta), _p(u), ctypes.byref(lm))
        return dt, lm.value

    def timestep2(self, u):
        """dt, max wave speed, max velocity component (MHD cleaning speed inputs)."""
        u = _f64(u)
        lm, vm = ctypes.c_double(0), ctypes.c_double(0)
        dt = self.lib.or_timestep2(self._c(), self.E, _p(self.delta), _p(u), ctypes.byref(lm), ctypes.byref(vm))
        return dt, lm.value, vm.value

    def stage(self, u, reg, stage, dt):
        """In place on u and reg (float64 C-contiguous); stage is 0-based."""
        return self.lib.or_stage(self._c(), self.E, _p(self.nbr, _ip), _p(self.delta), stage, dt, _p(u), _p(reg),
                              self.nthreads)

    def run(self, u, nsteps=0, t_end=0.0, t0=0.0):
        u = _f64(u).copy()
        t = ctypes.c_double(t0)
        nbad = ctypes.c_int64(0)
        steps = self.lib.or_run(self._c(), self.E, _p(self.nbr, _ip), _p(self.delta), _p(u), int(nsteps),
                             float(t_end), ctypes.byref(t), ctypes.byref(nbad), self.nthreads)
        return u, t.value, int(steps), int(nbad.value)

    def totals(self, u):
        u = _f64(u)
        out = np.zeros(10)
        self.lib.or_totals(self._c(), self.E, _p(self.delta), _p(u), _p(out))
        return out[: self.V]

    def opcounts(self):
        """Counted operations since the last reset (variant "count" only): dict by kind."""
        out = (ctypes.c_uint64 * 6)()
        self.lib.or_opcount_read(out)
        return dict(zip(("add", "mul", "div", "sqrt", "log", "exp"), [int(x) for x in out]))

    def opcount_reset(self):
        self.lib.or_opcount_reset()
