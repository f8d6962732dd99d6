"""The reference arm of bench.py (the oracle on the host cores) prints one JSON line with the keys
the benchmark contract asks for; a small workload keeps it to seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "wave16",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "DOF-updates/s per RK stage" and line["unit"] == "DOF-updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "DOF-updates/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "workload" in line["config"]
    # the reference driver's performance index: microseconds per node-stage per core
    assert abs(line["pid"]["cpu"] - cb["cores"] * 1e6 / line["value"]) < 1e-9 * line["pid"]["cpu"]


def test_reference_arm_does_not_load_the_cuda_library():
    """The reference arm runs the oracle only: libnemo_gpu.so must not be mapped into its process."""
    code = (
        "import sys, types; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'wave16', '--steps', '1',"
        " '--warmup', '0']; sys.path.insert(0, '.'); import bench; bench.main();"
        " maps = open('/proc/self/maps').read(); print('LOADED' if 'libnemo_gpu.so' in maps else 'CLEAN')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
