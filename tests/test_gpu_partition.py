"""The partitioned GPU path: two processes share the GPU, each advances its element range of a 2:1
forest through the CUDA library with ghosts refreshed before every stage (library pack/unpack,
gloo host buffers) and the all-reduced time step; the owned elements must equal the FP64 oracle's
single-process run bit for bit.  (On a multi-GPU node the same code runs one process per GPU with
NCCL device buffers.)  The processes never wait on each other inside a kernel: every exchange goes
through the host between launches."""
import os
import socket

import numpy as np
import pytest

from nemo_b200 import abi, mesh, partition, setups
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def band_forest(nb=4):
    return mesh.forest(nb, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)


def blast_state(m):
    x, y, z = m.node_coords(setups.LGL4)
    u = setups.smooth_random(m, seed=2)
    u[4] += 5.0 * np.exp(-((x - 0.45) ** 2 + (y - 0.5) ** 2 + (z - 0.55) ** 2) / 0.01)
    return np.ascontiguousarray(u)


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir, nsteps, precision, faces):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = blast_state(m)
        part = partition.partition(m, world)[rank]
        cfg = abi.default_cfg(indicator=abi.IND_MODAL, positivity=1, precision=precision)
        run = partition.PartitionedRun(cfg, part, dist, faces=faces)
        run.upload(np.ascontiguousarray(u[:, part.glob]))
        run.run(nsteps)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), run.download_owned())
        run.s.finalize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision,faces", [(abi.PREC_FP64, True), (abi.PREC_FP64, False), (abi.PREC_FP32, True)])
def test_two_process_partition_matches_oracle(precision, faces, tmp_path):
    """Ghost refresh by faces (the default) or whole elements."""
    import torch.multiprocessing as tmp
    nsteps = 3
    tmp.spawn(_worker, args=(2, _port(), str(tmp_path), nsteps, precision, faces), nprocs=2, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(2)], axis=1)
    m = band_forest()
    u = blast_state(m)
    ref, _, _, _ = orc.Oracle.for_mesh(abi.default_cfg(indicator=abi.IND_MODAL, positivity=1), m).run(u, nsteps=nsteps)
    if precision == abi.PREC_FP64:
        assert np.array_equal(got, ref)
    else:
        assert np.sum(np.abs(got[0] - ref[0])) / np.sum(np.abs(ref[0])) < 1e-6
