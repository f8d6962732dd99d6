"""Algorithmic flops per DOF-update of the bench workloads, from the counting build of the oracle.

MEASUREMENT INFRASTRUCTURE (run here, on the host; its output is committed): the oracle compiled
with an operation counter (oracle/opcount.cpp) runs one full time step -- the CFL reduction, five
RK stages with their indicator, mortar, element and update work -- from each workload's initial
state, single-threaded, and the counted + - * / sqrt log exp (1 flop each; the oracle has no FMA)
are divided by the DOF-updates of that step (nodes x 5 stages).  The result is frozen in
profiles/roofline.json, which bench.py reads to grade the stage kernels against the arithmetic
roofline.  The metric's unit follows the reference's performance index (source/driver_mod.f90:83:
node updates per RK stage).

    python -m oracle.count_flops [workload ...]
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

OUT = os.path.join(ROOT, "profiles", "roofline.json")


def count(wl):
    import bench
    m, u, groups = bench.make_state(wl)
    c = bench.make_cfg(wl, host_only=True)
    o = orc.Oracle.for_mesh(c, m, nthreads=1, variant="count")
    o.opcount_reset()
    t0 = time.perf_counter()
    o.run(u, nsteps=1)
    el = time.perf_counter() - t0
    cnt = o.opcounts()
    dof = m.E * 64 * 5
    return {"flops_per_dof_update": sum(cnt.values()) / dof,
            "by_kind_per_dof_update": {k: v / dof for k, v in cnt.items()},
            "elements": int(m.E), "dof_updates_counted": int(dof),
            "sample": "one time step (CFL reduction + 5 RK stages) from the initial state, single-threaded",
            "count_seconds": round(el, 1), "variables": int(c.n_vars)}


def main(argv):
    import bench
    orc.build()
    wls = argv or ["wave16", "sedov32", "batch", "ot64"]
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data["convention"] = ("algorithmic flops of the FP64 oracle: + - * / sqrt log exp count 1 each (no FMA: "
                          "contraction is off), comparisons/fabs/fmin/fmax/conversions 0; per DOF-update = one "
                          "node with all variables advanced through one RK stage")
    data.setdefault("workloads", {})
    for wl in wls:
        r = count(wl)
        r["workload"] = bench.WORKLOADS[wl]["desc"]
        data["workloads"][wl] = r
        print(wl, json.dumps(r), flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
