"""Build libnemo_gpu.so in-tree with nvcc for sm_100a (no JIT, no torch extension cache).

The plain FP64 kernels are compiled with -fmad=false (every + - * / one IEEE operation) and the
host code with -ffp-contract=off; the FP32-bulk kernels keep FMA contraction.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnemo_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr"]
# per-source extra flags
SOURCES = {
    "nemo_gpu.cu": [],
    "control.cu": ["-fmad=false"],
    "stage_fp64.cu": ["-fmad=false"],
    "stage_fp32.cu": ["--use_fast_math"],
    "noalloc.cu": ["-fmad=false"],
    "mlp.cu": ["--use_fast_math"],
    "mortar.cu": ["-fmad=false"],
    "peaks.cu": [],
}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "nemo_gpu.h"))
    objs, jobs = [], []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc()] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append((src, cmd))

    # the translation units are independent: compile them concurrently (the stage kernels dominate)
    def run(job):
        src, cmd = job
        return src, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for src, r in pool.map(run, jobs):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
            if ptxas_info or verbose:
                print(r.stderr, file=sys.stderr)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
