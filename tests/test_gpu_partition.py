"""The partitioned GPU path: two processes share the GPU, each advances its element range of a 2:1
forest through the CUDA library with ghosts refreshed before every stage (library pack/unpack,
gloo host buffers) and the all-reduced time step; the owned elements must equal the FP64 oracle's
single-process run bit for bit.  (On a multi-GPU node the same code runs one process per GPU with
NCCL device buffers.)  The processes never wait on each other inside a kernel: every exchange goes
through the host between launches (the interior part of a stage is enqueued before the host waits
for the exchange, the boundary part after it)."""
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


def mhd_cfg(**kw):
    return abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_HLLD,
                           kappa=5.0 / 3.0, mu0=1.0, indicator=abi.IND_MODAL, positivity=1, **kw)


def _worker(rank, world, port, out_dir, nsteps, precision, faces, overlap=True, mhd=False):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = np.ascontiguousarray(setups.orszag_tang(m)) if mhd else blast_state(m)
        part = partition.partition(m, world)[rank]
        cfg = mhd_cfg(precision=precision) if mhd else abi.default_cfg(indicator=abi.IND_MODAL, positivity=1,
                                                                         precision=precision)
        run = partition.PartitionedRun(cfg, part, dist, faces=faces, overlap=overlap)
        run.upload(np.ascontiguousarray(u[:, part.glob]))
        run.run(nsteps)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), run.download_owned())
        run.s.finalize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision,faces,overlap", [(abi.PREC_FP64, True, True), (abi.PREC_FP64, False, True),
                                                     (abi.PREC_FP64, True, False), (abi.PREC_FP32, True, True)])
def test_two_process_partition_matches_oracle(precision, faces, overlap, tmp_path):
    """Ghost refresh by faces (the default) or whole elements; each stage split into the interior
    part (while the exchange is in flight) and the partition-boundary part, or run whole."""
    import torch.multiprocessing as tmp
    nsteps = 3
    tmp.spawn(_worker, args=(2, _port(), str(tmp_path), nsteps, precision, faces, overlap), nprocs=2, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(2)], axis=1)
    m = band_forest()
    u = blast_state(m)
    ref, _, _, _ = orc.Oracle.for_mesh(abi.default_cfg(indicator=abi.IND_MODAL, positivity=1), m).run(u, nsteps=nsteps)
    if precision == abi.PREC_FP64:
        assert np.array_equal(got, ref)
    else:
        assert np.sum(np.abs(got[0] - ref[0])) / np.sum(np.abs(ref[0])) < 1e-6


def test_two_process_mhd_partition_matches_oracle(tmp_path):
    """GLM-MHD with HLLD on a 2:1 forest: Δt all-reduced, λmax and vmax all-reduced into the global
    cleaning speed; bit-exact with the single-process oracle run."""
    import torch.multiprocessing as tmp
    nsteps = 2
    tmp.spawn(_worker, args=(2, _port(), str(tmp_path), nsteps, abi.PREC_FP64, True, True, True), nprocs=2, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(2)], axis=1)
    m = band_forest()
    ref, _, _, _ = orc.Oracle.for_mesh(mhd_cfg(), m).run(setups.orszag_tang(m), nsteps=nsteps)
    assert np.array_equal(got, ref)
