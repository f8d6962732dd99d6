"""ctypes binding of the C-ABI in include/nemo_gpu.h (libnemo_gpu.so, built in-tree).

There is no CPU fallback: if the library is missing or fails to load, every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnemo_gpu.so")

EQN_EULER, EQN_MHD = 0, 1
VOLFLUX_CHANDRASHEKAR, VOLFLUX_CENTRAL, VOLFLUX_EC_MHD = 0, 1, 2
SURFFLUX_HLLC, SURFFLUX_RUSANOV, SURFFLUX_HLLD = 0, 1, 2
PREC_FP64, PREC_FP32 = 0, 1
IND_NONE, IND_MODAL, IND_LEARNED = 0, 1, 2
SOURCE_NONE, SOURCE_BAROTROPIC_COOLING = 0, 1

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_STATE", 3: "ERR_CUDA", 4: "ERR_REPAIR", 5: "ERR_NONFINITE"}

# Every entry point declared in include/nemo_gpu.h (checked by the CPU tests against the header).
EXPORTS = [
    "nemo_gpu_default_cfg", "nemo_gpu_init", "nemo_gpu_operators", "nemo_gpu_set_mesh",
    "nemo_gpu_set_groups", "nemo_gpu_upload_state", "nemo_gpu_download_state",
    "nemo_gpu_calc_timestep", "nemo_gpu_stage", "nemo_gpu_step", "nemo_gpu_run", "nemo_gpu_rhs",
    "nemo_gpu_alpha", "nemo_gpu_totals", "nemo_gpu_status", "nemo_gpu_finalize",
    "nemo_gpu_last_error", "nemo_gpu_set_timing", "nemo_gpu_kernel_timing", "nemo_gpu_stream",
    "nemo_gpu_totals_noalloc", "nemo_gpu_set_mlp", "nemo_gpu_features", "nemo_gpu_indicator_stats",
    "nemo_gpu_mlp_train", "nemo_gpu_mlp_grad", "nemo_gpu_mlp_forward", "nemo_gpu_mortar_operators",
    "nemo_gpu_autotune", "nemo_gpu_set_schedule", "nemo_gpu_set_owned", "nemo_gpu_pack_elements",
    "nemo_gpu_unpack_elements", "nemo_gpu_adapt", "nemo_gpu_amr_flags",
    "nemo_gpu_checkpoint_begin", "nemo_gpu_checkpoint_wait", "nemo_gpu_set_time",
    "nemo_gpu_pack_faces", "nemo_gpu_unpack_faces", "nemo_gpu_measure_peaks", "nemo_gpu_amr_operators",
    "nemo_gpu_repair_states", "nemo_gpu_upload_state_async", "nemo_gpu_upload_wait", "nemo_gpu_run_async",
    "nemo_gpu_sync", "nemo_gpu_set_interior", "nemo_gpu_stage_interior", "nemo_gpu_stage_boundary",
    "nemo_gpu_glm_speeds", "nemo_gpu_set_glm", "nemo_gpu_download_state_async",
]


class NemoError(RuntimeError):
    def __init__(self, func, code, msg):
        super().__init__(f"{func} -> {STATUS.get(code, code)}: {msg}")
        self.code = code


class NemoCfg(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int32), ("n_vars", ctypes.c_int32), ("eqn", ctypes.c_int32),
        ("volume_flux", ctypes.c_int32), ("surface_flux", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("indicator", ctypes.c_int32), ("alpha_smoothing", ctypes.c_int32), ("positivity", ctypes.c_int32),
        ("non_conservative", ctypes.c_int32), ("source", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("kappa", ctypes.c_double), ("mu0", ctypes.c_double), ("cfl", ctypes.c_double),
        ("alpha_max", ctypes.c_double), ("alpha_min", ctypes.c_double), ("repair_decr", ctypes.c_double),
        ("glm_ch", ctypes.c_double), ("glm_alpha", ctypes.c_double), ("dens_critical", ctypes.c_double),
        ("k_isothermal", ctypes.c_double), ("k_adiabatic", ctypes.c_double), ("reserved", ctypes.c_double),
    ]


_LIB = None
_dp = ctypes.POINTER(ctypes.c_double)


def load(path=LIB_PATH):
    """Load libnemo_gpu.so; raises if it is absent (build it with nemo_b200.build.build())."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} not found: the CUDA library is required (no CPU fallback); "
                           "build it with python -m nemo_b200.build")
    L = ctypes.CDLL(path)
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    vp = ctypes.c_void_p
    sig = {
        "nemo_gpu_default_cfg": [ctypes.POINTER(NemoCfg)],
        "nemo_gpu_init": [ctypes.POINTER(NemoCfg)],
        "nemo_gpu_operators": [i32, vp, vp, vp, vp, vp],
        "nemo_gpu_set_mesh": [i64, vp, vp, i64, vp, vp, vp, vp],
        "nemo_gpu_set_groups": [i32, vp],
        "nemo_gpu_upload_state": [vp, i64],
        "nemo_gpu_download_state": [vp, i64],
        "nemo_gpu_calc_timestep": [dbl, ctypes.POINTER(dbl), ctypes.POINTER(dbl)],
        "nemo_gpu_stage": [i32, dbl, dbl, ctypes.POINTER(i32)],
        "nemo_gpu_step": [dbl],
        "nemo_gpu_run": [i64, dbl, ctypes.POINTER(dbl), ctypes.POINTER(i64)],
        "nemo_gpu_rhs": [vp],
        "nemo_gpu_alpha": [vp],
        "nemo_gpu_totals": [vp],
        "nemo_gpu_status": [ctypes.POINTER(dbl), ctypes.POINTER(i64)],
        "nemo_gpu_finalize": [],
        "nemo_gpu_last_error": [ctypes.c_char_p, i32],
        "nemo_gpu_set_timing": [i32],
        "nemo_gpu_kernel_timing": [ctypes.POINTER(dbl), ctypes.POINTER(i64), ctypes.POINTER(dbl),
                                   ctypes.POINTER(i64)],
        "nemo_gpu_stream": [ctypes.POINTER(ctypes.c_uint64)],
        "nemo_gpu_measure_peaks": [vp],
        "nemo_gpu_amr_operators": [i32, i32, vp, vp],
        "nemo_gpu_repair_states": [vp, i64, i64, vp],
        "nemo_gpu_upload_state_async": [vp, i64],
        "nemo_gpu_upload_wait": [],
        "nemo_gpu_run_async": [i64],
        "nemo_gpu_sync": [],
        "nemo_gpu_set_interior": [i64],
        "nemo_gpu_stage_interior": [i32, dbl],
        "nemo_gpu_stage_boundary": [i32, dbl, ctypes.POINTER(i32)],
        "nemo_gpu_glm_speeds": [ctypes.POINTER(dbl), ctypes.POINTER(dbl)],
        "nemo_gpu_set_glm": [dbl, dbl],
        "nemo_gpu_download_state_async": [vp, i64],
        "nemo_gpu_totals_noalloc": [vp, vp, i64, i64, i32, vp, ctypes.c_uint64],
        "nemo_gpu_set_mlp": [vp, i32, vp, vp],
        "nemo_gpu_features": [vp, vp],
        "nemo_gpu_indicator_stats": [ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(dbl)],
        "nemo_gpu_mlp_train": [vp, vp, i64, vp, ctypes.c_float, i32, i32, ctypes.c_float, ctypes.c_uint64, vp],
        "nemo_gpu_mlp_grad": [vp, vp, i64, vp, ctypes.c_float, vp, vp],
        "nemo_gpu_mlp_forward": [vp, i64, vp, ctypes.c_float, vp],
        "nemo_gpu_mortar_operators": [i32, vp, vp],
        "nemo_gpu_autotune": [i32, ctypes.POINTER(i32), ctypes.POINTER(i32), vp],
        "nemo_gpu_set_schedule": [i32, i32],
        "nemo_gpu_set_owned": [i64],
        "nemo_gpu_pack_elements": [vp, i64, vp],
        "nemo_gpu_unpack_elements": [vp, i64, vp],
        "nemo_gpu_adapt": [i64, vp, vp, i64, vp, vp, vp, vp, vp],
        "nemo_gpu_amr_flags": [dbl, dbl, vp],
        "nemo_gpu_checkpoint_begin": [vp, i64, vp],
        "nemo_gpu_checkpoint_wait": [ctypes.POINTER(dbl), ctypes.POINTER(i64)],
        "nemo_gpu_set_time": [dbl, i64],
        "nemo_gpu_pack_faces": [vp, vp, i64, vp],
        "nemo_gpu_unpack_faces": [vp, vp, i64, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    _LIB = L
    return L


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().nemo_gpu_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def call(name, *args):
    rc = getattr(load(), name)(*args)
    if rc != 0:
        raise NemoError(name, rc, last_error())
    return rc


def default_cfg(**kw):
    c = NemoCfg()
    call("nemo_gpu_default_cfg", ctypes.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def measure_peaks():
    """Measured FP64 / FP32 FMA peaks of the current device: dict with TFLOP/s, SM count and clock."""
    out = np.zeros(4)
    call("nemo_gpu_measure_peaks", out.ctypes.data)
    return {"fp64_tflops": float(out[0]), "fp32_tflops": float(out[1]), "sms": int(out[2]),
            "sm_max_mhz": float(out[3])}


def amr_operators(qmax=3):
    """(refine, coarsen) as [q][f][d][i][j] numpy arrays (the C side writes the Fortran layout
    (n, n, 3, 8, 0:qmax), i fastest)."""
    n = 4
    r = np.zeros((qmax + 1) * 8 * 3 * n * n)
    c = np.zeros_like(r)
    call("nemo_gpu_amr_operators", n, int(qmax), r.ctypes.data, c.ctypes.data)
    shape = (qmax + 1, 8, 3, n, n)   # C order of the Fortran (i, j, d, f, q) array is (q, f, d, j, i)
    return r.reshape(shape).transpose(0, 1, 2, 4, 3), c.reshape(shape).transpose(0, 1, 2, 4, 3)


def cfg_struct(**kw):
    """A NemoCfg with the defaults of nemo_gpu_default_cfg, built without loading the library (for
    callers that only drive the oracle)."""
    c = NemoCfg(n_nodes=4, n_vars=5, eqn=EQN_EULER, volume_flux=VOLFLUX_CHANDRASHEKAR, surface_flux=SURFFLUX_HLLC,
                precision=PREC_FP64, indicator=IND_NONE, alpha_smoothing=1, positivity=0, kappa=1.4, mu0=1.0,
                cfl=0.5, alpha_max=0.5, alpha_min=0.001, repair_decr=0.01)
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def operators():
    n = 4
    x, w = np.zeros(n), np.zeros(n)
    D, S, Vi = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    call("nemo_gpu_operators", n, x.ctypes.data, w.ctypes.data, D.ctypes.data, S.ctypes.data, Vi.ctypes.data)
    return x, w, D, S, Vi


def mortar_operators():
    """(prolongation [2,4,4], projection [2,4,4]) of the 2:1 mortar, lower/upper half."""
    pro, prj = np.zeros((2, 4, 4)), np.zeros((2, 4, 4))
    call("nemo_gpu_mortar_operators", 4, pro.ctypes.data, prj.ctypes.data)
    return pro, prj


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data)
