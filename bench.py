"""Benchmark of the spatial-operator hot path: DOF-updates/s per RK stage on one B200.

Workload (default): the shocked Euler case with DG/FV blending -- Sedov-type blast on 32^3
elements, N = 3 (2,097,152 nodes, 5 variables), gamma 1.4, ambient rho 1, p 1e-5, E0 = 1 in a
Gaussian of width 0.05, modal-energy indicator with alpha in [0, 0.5], positivity repair, periodic
box, LSRK 5-4 at CFL 0.5.  One "step" is one full time step (5 RK stages + the device CFL
reduction); one DOF-update is one node with all 5 variables advanced through one stage.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Multi-GPU (torchrun): every rank advances its own replica of the workload (independent runs; the
element-partitioned halo exchange is not built), the timed region is bracketed by barriers and the
max over ranks is reported; value is the whole-job DOF-updates/s.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (elements per direction, setup, indicator)
    "sedov32": dict(nx=32, setup="sedov", indicator=1, positivity=1,
                    desc="Sedov blast 32^3 elements N=3 (2.1M nodes), DG/FV blending, FP64"),
    "sedov64": dict(nx=64, setup="sedov", indicator=1, positivity=1,
                    desc="Sedov blast 64^3 elements N=3 (16.8M nodes), learned indicator vs the modal one, FP64"),
    "wave16": dict(nx=16, setup="wave", indicator=0, positivity=0,
                   desc="periodic density wave 16^3 elements N=3 (262k nodes), EC volume + HLLC, FP64"),
    "batch": dict(nx=24, setup="batch", indicator=1, positivity=1, t_end=0.05,
                  desc="batched uneven workload: Kelvin-Helmholtz forest on 24^3 base elements with 0-2 "
                       "levels of refinement at the shear layers (2:1 mortars) + 256 independent 8^3 "
                       "Gaussian-blob runs (amplitudes U[0.1,1]), N=3, one element list, per-run time steps"),
    "ot64": dict(nx=64, setup="orszag_tang", indicator=1, positivity=1, mhd=True, t_end=0.1,
                 desc="GLM-MHD Orszag-Tang 64^3 elements N=3 (16.8M nodes, 9 variables), gamma 5/3, "
                      "b0 = 1/sqrt(4 pi), HLLD surface + EC volume, DG/FV blending"),
}


def nvars(wl):
    return 9 if WORKLOADS[wl].get("mhd") else 5


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_state(wl):
    """(mesh, state, groups or None)."""
    from nemo_b200 import mesh, setups
    w = WORKLOADS[wl]
    if w["setup"] == "batch":
        m, g, f, one, amps = mesh.batched_workload(nb=w["nx"])
        u = np.concatenate([setups.kelvin_helmholtz(f)] + [setups.gaussian_blob(one, a) for a in amps], axis=1)
        return m, np.ascontiguousarray(u), g
    if w["setup"] == "sedov":
        m = mesh.brick(w["nx"], lo=(-0.5,) * 3, hi=(0.5,) * 3)
        u = setups.sedov(m, sigma=0.05)
    elif w["setup"] == "orszag_tang":
        m = mesh.brick(w["nx"])
        u = setups.orszag_tang(m)
    else:
        m = mesh.brick(w["nx"])
        u = setups.density_wave(m, seed=1234)
    return m, u, None


def make_cfg(wl, precision=0, learned=False):
    from nemo_b200 import abi
    w = WORKLOADS[wl]
    ind = abi.IND_LEARNED if (learned and w["indicator"]) else w["indicator"]
    if w.get("mhd"):
        return abi.default_cfg(indicator=ind, positivity=w["positivity"], cfl=0.5, precision=precision,
                               eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD,
                               surface_flux=abi.SURFFLUX_HLLD, kappa=5.0 / 3.0, mu0=1.0)
    return abi.default_cfg(indicator=ind, positivity=w["positivity"], cfl=0.5, precision=precision)


def make_solver(wl, m, precision, learned=False, groups=None):
    from nemo_b200.solver import Solver
    s = Solver(make_cfg(wl, precision, learned), m, groups)
    if learned and WORKLOADS[wl]["indicator"]:
        from nemo_b200 import learned as lm
        lm.install()
    return s


def timed_run(s, steps, stream, dist, torch, ctypes, abi):
    """K steps with per-kernel CUDA events on the library stream; returns (ms, stage_ms, stage_n,
    total_ms, total_n, t_sim, steps_done)."""
    abi.call("nemo_gpu_set_timing", 1)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t_sim, nst = s.run(nsteps=steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    st_ms, st_n, tot_ms, tot_n = (ctypes.c_double(), ctypes.c_int64(), ctypes.c_double(), ctypes.c_int64())
    abi.call("nemo_gpu_kernel_timing", ctypes.byref(st_ms), ctypes.byref(st_n), ctypes.byref(tot_ms),
             ctypes.byref(tot_n))
    abi.call("nemo_gpu_set_timing", 0)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, st_ms.value, st_n.value, tot_ms.value, tot_n.value, t_sim, nst


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        import tempfile
        fd, self.out = tempfile.mkstemp(prefix="nemo_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv",
                                          "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.out) as f:
            for line in f.read().splitlines()[1:]:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        try:
            os.remove(self.out)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1].split()[0]) for r in rows]
        mx = float(rows[0][2].split()[0])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def cpu_baseline(wl, u, m, nthreads=None, sample_stages=5):
    """The oracle (C++ FP64 restatement, OpenMP) on the host cores, on a bounded sample of the same
    workload: sample_stages RK stages of the full state (one common time step for all elements)."""
    from oracle import oracle as orc
    c = make_cfg(wl)
    o = orc.Oracle.for_mesh(c, m, nthreads=nthreads)
    uu, reg = u.copy(), np.zeros_like(u)
    dt, _ = o.timestep(uu)
    o.stage(uu, reg, 0, dt)  # untimed warm-up stage (page-in)
    uu, reg = u.copy(), np.zeros_like(u)
    t0 = time.perf_counter()
    for s in range(sample_stages):
        o.stage(uu, reg, s % 5, dt)
    el = time.perf_counter() - t0
    dof = m.E * 64 * sample_stages
    return {"value": dof / el, "unit": "DOF-updates/s", "cores": o.nthreads, "kind": "port",
            "sample": f"{sample_stages} RK stages of the full {WORKLOADS[wl]['desc']} state, "
                      f"{o.nthreads} OpenMP threads, {el:.2f} s"}


def accuracy_check(wl, m, u, abi, Solver, t_end=0.05, groups=None):  # noqa: C901
    """All forms to t_end.  The chosen form (FP32 bulk + learned indicator) against the FP64 form of
    the same method (learned indicator evaluated in FP64 from the same BF16 weights; that plain
    path reproduces the FP64 oracle bit for bit, see tests/test_gpu_learned.py), and both against
    the plain FP64 modal-indicator run."""
    import ctypes
    res = {}
    for key, prec, learned in (("fp64_modal", abi.PREC_FP64, False), ("fp64_learned", abi.PREC_FP64, True),
                               ("fp32_learned", abi.PREC_FP32, True)):
        s = make_solver(wl, m, prec, learned, groups)
        s.upload(u)
        if prec == abi.PREC_FP32:
            s.autotune(nsteps=2)
        t0 = time.perf_counter()
        t, n = s.run(t_end=t_end)
        el = time.perf_counter() - t0
        fb, jn, mae = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        abi.call("nemo_gpu_indicator_stats", ctypes.byref(fb), ctypes.byref(jn), ctypes.byref(mae))
        uf = s.download()
        res[key] = dict(rho=uf[0], t=t, steps=n, wall=el, nbad=s.status()[1], fallback=fb.value,
                        judged=jn.value, judge_mae=mae.value)
        if WORKLOADS[wl].get("mhd"):
            res[key]["divb"] = divb(m, uf, abi)
        s.finalize()

    def l1(a, b):
        return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))

    r = res
    return {"t_end": t_end, "steps": {k: v["steps"] for k, v in r.items()},
            "rel_l1_density_chosen_vs_fp64_same_method": l1(r["fp32_learned"]["rho"], r["fp64_learned"]["rho"]),
            "rel_linf_density_chosen_vs_fp64_same_method": float(
                np.max(np.abs(r["fp32_learned"]["rho"] - r["fp64_learned"]["rho"])) / np.max(np.abs(r["fp64_learned"]["rho"]))),
            "rel_l1_density_learned_vs_modal_fp64": l1(r["fp64_learned"]["rho"], r["fp64_modal"]["rho"]),
            "indicator_judge": {k: {"fallback_elements": v["fallback"], "judged_elements": v["judged"],
                                    "mean_abs_alpha_learned_minus_modal": v["judge_mae"]}
                                for k, v in r.items() if k != "fp64_modal"},
            "repair_failures": {k: v["nbad"] for k, v in r.items()},
            "wall_s_to_t_end": {k: v["wall"] for k, v in r.items()},
            **({"div_b_l2_linf": {"t0": divb(m, u, abi), **{k: v["divb"] for k, v in r.items()}}}
               if WORKLOADS[wl].get("mhd") else {})}


def divb(m, u, abi):
    from nemo_b200 import setups
    _, w, D, _, _ = abi.operators()
    return setups.divergence_b(m, u, D, w)


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU implementation of the path.  The Fortran reference
    cannot be built here (no Fortran compiler / MPI / p4est / HDF5), so this times the C++ FP64
    restatement of it (oracle/) on all host cores; each step is one full time step (5 stages)."""
    if rank != 0:
        return
    from oracle import oracle as orc
    orc.build()
    m, u, groups = make_state(args.workload)
    c = make_cfg(args.workload)
    o = orc.Oracle.for_mesh(c, m)
    uu = u.copy()
    for _ in range(args.warmup):
        uu, _, _, _ = o.run(uu, nsteps=1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        uu, _, _, _ = o.run(uu, nsteps=1)
    el = time.perf_counter() - t0
    val = m.E * 64 * 5 * args.steps / el
    line = {
        "impl": "reference", "metric": "DOF-updates/s per RK stage", "value": val, "unit": "DOF-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "elements": m.E, "nodes": m.E * 64,
                   "stages_per_step": 5},
        "cpu_baseline": {"value": val, "unit": "DOF-updates/s", "cores": o.nthreads, "kind": "port",
                         "sample": f"{args.steps} full time steps, {o.nthreads} OpenMP threads; the Fortran "
                                   "reference is unbuildable here, this is its C++ FP64 restatement"},
        "e2e": {"value": val, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["pid"] = {"cpu": o.nthreads * 1e6 / val, "unit": PID_UNIT, "note": PID_NOTE}
    print(json.dumps(line), flush=True)


PID_UNIT = "us per node-stage per device (GPU) or per core (CPU)"
PID_NOTE = ("performance index of the reference's driver (source/driver_mod.f90:83): wall time x processing "
            "units / (nodes x time steps x RK stages); for one device 1e6 / (DOF-updates/s per device)")


def pid_block(value, e2e, value64, cpu):
    """The reference's performance index for each measured form (lower is better)."""
    out = {"chosen": 1e6 / value, "plain_fp64": 1e6 / value64, "unit": PID_UNIT, "note": PID_NOTE}
    if e2e:
        out["e2e"] = 1e6 / e2e
    if cpu:
        out["cpu_baseline"] = cpu["cores"] * 1e6 / cpu["value"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sedov32", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the run to t_end that checks the L1 error")
    ap.add_argument("--schedule", default="auto", choices=["auto", "grid", "persistent"],
                    help="FP32 stage schedule: autotuned (default) or fixed (profiling runs)")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference" or os.environ.get("NEMO_BENCH_ALLOW_SHORT")

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from nemo_b200 import abi
    from nemo_b200.solver import Solver
    import ctypes

    m, u, groups = make_state(args.workload)
    dof_per_step = m.E * 64 * 5
    V = nvars(args.workload)
    mhd = bool(WORKLOADS[args.workload].get("mhd"))

    # ---- the plain FP64 form (the comparison point of the metric)
    s = Solver(make_cfg(args.workload, abi.PREC_FP64), m, groups)
    s.upload(u)
    stream_ptr = ctypes.c_uint64()
    abi.call("nemo_gpu_stream", ctypes.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    s.run(nsteps=args.warmup)
    ms64, st64, n64, tot64, ntot64, _, _ = timed_run(s, args.steps, stream, dist, torch, ctypes, abi)
    value64 = world * dof_per_step * args.steps / (ms64 * 1e-3)
    s.finalize()

    # ---- the chosen form: FP32 bulk + learned indicator, FP64 state/register/update/repair/reductions
    s = make_solver(args.workload, m, abi.PREC_FP32, learned=True, groups=groups)
    s.upload(u)
    if args.schedule == "auto":
        tune_mode, tune_ctas, tune_ms = s.autotune(nsteps=3)   # restores the state it times
    else:
        import torch as _t
        nsm = _t.cuda.get_device_properties(local).multi_processor_count
        tune_mode, tune_ctas, tune_ms = (0, 0, [-1.0] * 5) if args.schedule == "grid" else (1, 4 * nsm, [-1.0] * 5)
        s.set_schedule(tune_mode, tune_ctas)
    abi.call("nemo_gpu_stream", ctypes.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    s.run(nsteps=args.warmup)
    with ClockSampler(local) as clk:
        ms, st_ms_v, st_n_v, tot_ms_v, tot_n_v, t_sim, nst = timed_run(s, args.steps, stream, dist, torch, ctypes,
                                                                        abi)
    value = world * dof_per_step * args.steps / (ms * 1e-3)

    # ---- roofline of the stage kernel (HBM): algorithmic bytes per launch / avg launch time
    bytes_per_launch = sum(m.E * 64 * V * 8 * (3 if st == 0 else 4) for st in range(5)) / 5.0
    avg_stage_s = st_ms_v * 1e-3 / max(st_n_v, 1)
    peak, peak_kind = load_peaks()
    achieved = bytes_per_launch / avg_stage_s / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(args.workload)

    e2e_val, e2e_steps, nbytes = None, 0, u.nbytes
    if not args.no_e2e:
        # ---- end to end through the C-ABI: pinned host state in, one step, state out (every step)
        host_in = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
        host_out = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
        host_in.numpy()[:] = np.ascontiguousarray(u.transpose(1, 0, 2)).ravel()
        row = V * 64 * 8
        for _ in range(2):  # warm-up
            s.upload_aos(host_in.data_ptr(), row)
            s.run(nsteps=1)
            abi.call("nemo_gpu_download_state", ctypes.c_void_p(host_out.data_ptr()), row)
        e2e_steps = max(3, min(args.steps, 10))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            s.upload_aos(host_in.data_ptr(), row)
            s.run(nsteps=1)
            abi.call("nemo_gpu_download_state", ctypes.c_void_p(host_out.data_ptr()), row)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([e2e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e_val = world * dof_per_step * e2e_steps / (e2e_ms * 1e-3)

    s.finalize()
    accuracy = None
    if not args.no_accuracy and WORKLOADS[args.workload]["setup"] in ("sedov", "orszag_tang", "batch"):
        accuracy = accuracy_check(args.workload, m, u, abi, Solver, t_end=WORKLOADS[args.workload].get("t_end", 0.05),
                                  groups=groups)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload, u, m)

    if rank == 0:
        line = {
            "metric": "DOF-updates/s per RK stage",
            "value": value,
            "unit": "DOF-updates/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 flux bulk, f64 state/register/update",
            "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "elements": m.E, "nodes": m.E * 64,
                       "stages_per_step": 5,
                       "form": "chosen: FP32 bulk + FP64 accumulation, learned indicator with modal fallback",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "schedule": {"chosen": "persistent" if tune_mode == 1 else "grid", "persistent_ctas": tune_ctas,
                                    "autotune_ms_per_step": {"grid": tune_ms[0], "persistent_1_per_sm": tune_ms[1],
                                                             "persistent_2_per_sm": tune_ms[2],
                                                             "persistent_3_per_sm": tune_ms[3],
                                                             "persistent_4_per_sm": tune_ms[4]}},
                       "groups": int(groups.max()) + 1 if groups is not None else 1,
                       "l2": f"working set (u in/out + register, 3 x {u.nbytes / 1e6:.0f} MB) larger than L2"},
            "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "k_stage_mhd<float>" if mhd else "k_stage_euler32",
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "avg_launch_ms": avg_stage_s * 1e3},
            "e2e": None if e2e_val is None else {
                    "value": e2e_val, "unit": "DOF-updates/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes,
                    "note": "per step: upload of the full state from pinned host memory, one time step, "
                            "download of the full state"},
            "gpu_launches": int(tot_n_v),
            "sim": {"t": t_sim, "steps": nst},
            "plain_fp64": {"value": value64, "unit": "DOF-updates/s", "ms_per_step": ms64 / args.steps,
                           "avg_stage_ms": st64 / max(n64, 1),
                           "kernel": "k_stage_mhd<double>" if mhd else "k_stage_euler64",
                           "speedup_of_chosen_form": value / value64},
            "accuracy": accuracy,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        line["pid"] = pid_block(value / world, None if e2e_val is None else e2e_val / world, value64 / world, cpu)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
