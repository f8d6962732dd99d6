"""Learned shock indicator: training data, training driver and weights file.

The network (12 -> 32 SiLU -> 32 SiLU -> 1 sigmoid, alpha in [0, alpha_max]) maps per-element
modal-energy features to the DG/FV blending coefficient; it is trained on the GPU by the library's
own forward/backward/Adam kernels (nemo_gpu_mlp_train) on element snapshots labelled by the plain
modal indicator, then evaluated inside the stage kernels with the modal indicator as fallback and
judge (include/nemo_gpu.h).  Data: seeded random 3D Riemann and blast problems with density and
pressure ratios log-uniform in [1, 100], advanced with the FP32 form and the modal indicator, and
sampled at a few times each.
"""
import ctypes
import json
import os

import numpy as np

from . import abi, mesh, setups
from .abi import call

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "indicator_mlp.json")
MLP_NW = 32 * 12 + 32 + 32 * 32 + 32 + 32 + 1


def init_weights(seed=0):
    """Glorot-uniform weights, zero biases, packed as W1 b1 W2 b2 W3 b3."""
    rng = np.random.default_rng(seed)

    def glorot(o, i):
        lim = np.sqrt(6.0 / (i + o))
        return rng.uniform(-lim, lim, size=(o, i))

    parts = [glorot(32, 12).ravel(), np.zeros(32), glorot(32, 32).ravel(), np.zeros(32), glorot(1, 32).ravel(),
             np.array([-2.0])]
    return np.concatenate(parts).astype(np.float32)


def random_problem(m, rng, kappa=1.4):
    """A seeded random 3D Riemann problem (planar interface, random normal) or blast (Gaussian
    pressure bump) on the unit periodic box, density and pressure ratios log-uniform in [1, 100]."""
    x, y, z = m.node_coords(setups.LGL4)
    ratio_r = np.exp(rng.uniform(0, np.log(100.0)))
    ratio_p = np.exp(rng.uniform(0, np.log(100.0)))
    if rng.uniform() < 0.5:
        nvec = rng.normal(size=3)
        nvec /= np.linalg.norm(nvec)
        c = rng.uniform(0.3, 0.7, size=3)
        side = ((x - c[0]) * nvec[0] + (y - c[1]) * nvec[1] + (z - c[2]) * nvec[2]) > 0
        width = rng.uniform(0.0, 0.02)
        if width > 0:
            s = 0.5 * (1 + np.tanh(((x - c[0]) * nvec[0] + (y - c[1]) * nvec[1] + (z - c[2]) * nvec[2]) / width))
        else:
            s = side.astype(float)
        rho = 1.0 + (ratio_r - 1.0) * s
        p = 1.0 + (ratio_p - 1.0) * s
        vel = [rng.uniform(-0.5, 0.5) * np.ones_like(x) for _ in range(3)]
    else:
        c = rng.uniform(0.3, 0.7, size=3)
        sig = rng.uniform(0.03, 0.12)
        r2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
        g = np.exp(-0.5 * r2 / sig ** 2)
        rho = 1.0 + (ratio_r - 1.0) * g * rng.uniform(0, 1)
        p = 1.0 + (ratio_p - 1.0) * g
        vel = [np.zeros_like(x)] * 3
    return np.ascontiguousarray(setups.prim2cons(rho, vel[0], vel[1], vel[2], p, kappa))


def generate_dataset(nproblems=200, nx=16, steps=(0, 4, 12), seed=2024, max_zero_frac=None):
    """Features and modal-indicator labels of element snapshots (the library must be loadable on a
    GPU).  Returns (feat [n,12] float32, alpha [n] float32)."""
    from .solver import Solver
    m = mesh.brick(nx)
    cfg = abi.default_cfg(precision=abi.PREC_FP32, indicator=abi.IND_MODAL, positivity=1, cfl=0.5)
    s = Solver(cfg, m)
    rng = np.random.default_rng(seed)
    feats, labels = [], []
    f = np.empty((m.E, 12), dtype=np.float32)
    a = np.empty(m.E)
    for _ in range(nproblems):
        u = random_problem(m, rng)
        s.upload(u)
        done = 0
        for st in steps:
            if st > done:
                s.run(nsteps=st - done)
                done = st
            call("nemo_gpu_features", abi.ptr(f), abi.ptr(a))
            feats.append(f.copy())
            labels.append(a.astype(np.float32))
    s.finalize()
    feat = np.concatenate(feats)
    alpha = np.concatenate(labels)
    ok = np.all(np.isfinite(feat), axis=1) & np.isfinite(alpha)
    feat, alpha = feat[ok], alpha[ok]
    if max_zero_frac is None:
        sel = rng.permutation(len(alpha))
        return np.ascontiguousarray(feat[sel]), np.ascontiguousarray(alpha[sel])
    # cap the share of the dominant alpha = 0 label
    zero = np.nonzero(alpha == 0)[0]
    nz = np.nonzero(alpha != 0)[0]
    keep_zero = min(len(zero), int(max_zero_frac / (1 - max_zero_frac) * max(len(nz), 1)))
    sel = np.concatenate([nz, rng.choice(zero, size=keep_zero, replace=False)])
    rng.shuffle(sel)
    return np.ascontiguousarray(feat[sel]), np.ascontiguousarray(alpha[sel])


def train(feat, alpha, epochs=30, batch=4096, lr=3e-3, seed=7, alpha_max=0.5, w0=None):
    w = init_weights(seed) if w0 is None else np.array(w0, dtype=np.float32)
    loss = np.zeros(epochs, dtype=np.float32)
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    alpha = np.ascontiguousarray(alpha, dtype=np.float32)
    call("nemo_gpu_mlp_train", abi.ptr(feat), abi.ptr(alpha), len(alpha), abi.ptr(w), ctypes.c_float(alpha_max),
         epochs, batch, ctypes.c_float(lr), ctypes.c_uint64(seed), abi.ptr(loss))
    return w, loss


def forward(feat, w, alpha_max=0.5):
    feat = np.ascontiguousarray(feat, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    out = np.empty(len(feat), dtype=np.float32)
    call("nemo_gpu_mlp_forward", abi.ptr(feat), len(feat), abi.ptr(w), ctypes.c_float(alpha_max), abi.ptr(out))
    return out


def input_bounds(feat, margin=0.05):
    """Per-input bounds of the normalised training inputs (x = feat/10 + 1), widened by margin."""
    x = feat / 10.0 + 1.0
    return (x.min(axis=0) - margin).astype(np.float32), (x.max(axis=0) + margin).astype(np.float32)


def save(w, lo, hi, meta, path=WEIGHTS):
    with open(path, "w") as f:
        json.dump({"weights": [float(v) for v in w], "lo": [float(v) for v in lo], "hi": [float(v) for v in hi],
                   "meta": meta}, f)


def load(path=WEIGHTS):
    with open(path) as f:
        d = json.load(f)
    return (np.array(d["weights"], dtype=np.float32), np.array(d["lo"], dtype=np.float32),
            np.array(d["hi"], dtype=np.float32), d.get("meta", {}))


def bf16_round(w):
    """The FP64 values of the BF16-rounded weights (nearest, ties to even) that nemo_gpu_set_mlp keeps."""
    b = np.asarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def install(path=WEIGHTS):
    """Load the trained network into the library (after nemo_gpu_init)."""
    w, lo, hi, _ = load(path)
    call("nemo_gpu_set_mlp", abi.ptr(w), MLP_NW, abi.ptr(lo), abi.ptr(hi))
    return w, lo, hi


def main(out=None, nproblems=200, epochs=40):
    """Generate the data set, train, and write the weights file (run on a GPU)."""
    import time
    t0 = time.time()
    feat, alpha = generate_dataset(nproblems=nproblems)
    t1 = time.time()
    w, loss = train(feat, alpha, epochs=epochs)
    t2 = time.time()
    lo, hi = input_bounds(feat)
    pred = forward(feat, w)
    mae = float(np.mean(np.abs(np.where(pred < 0.001, 0.0, pred) - alpha)))
    meta = {"samples": int(len(alpha)), "problems": nproblems, "epochs": epochs, "final_loss": float(loss[-1]),
            "first_loss": float(loss[0]), "train_mae": mae, "data_s": t1 - t0, "train_s": t2 - t1,
            "label_frac_nonzero": float(np.mean(alpha > 0))}
    save(w, lo, hi, meta, out or WEIGHTS)
    print(json.dumps(meta))
    return w, lo, hi, meta


if __name__ == "__main__":
    import sys
    main(out=sys.argv[1] if len(sys.argv) > 1 else None)
