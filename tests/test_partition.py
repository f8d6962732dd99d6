"""Element partition with ghost exchange (CPU): partition invariants, and the oracle advanced on
2 and 3 gloo ranks -- each rank its own share plus ghosts refreshed before every stage, the time
step an all-reduce minimum -- reproduces the single-process oracle run bit for bit, on a 2:1
forest with blending and positivity repair."""
import os
import socket

import numpy as np
import pytest

from nemo_b200 import abi, mesh, partition, setups
from oracle import oracle as orc


def band_forest(nb=4):
    return mesh.forest(nb, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)


def blast_state(m):
    x, y, z = m.node_coords(setups.LGL4)
    u = setups.smooth_random(m, seed=2)
    u[4] += 5.0 * np.exp(-((x - 0.45) ** 2 + (y - 0.5) ** 2 + (z - 0.55) ** 2) / 0.01)
    return np.ascontiguousarray(u)


@pytest.mark.parametrize("nranks", [2, 3])
def test_partition_invariants(nranks):
    m = band_forest()
    parts = partition.partition(m, nranks)
    owned = np.concatenate([np.sort(p.glob[: p.n_owned]) for p in parts])
    assert np.array_equal(owned, np.arange(m.E))
    gnbr = m.neighbors()
    for p in parts:
        lnbr = p.mesh.neighbors()          # a valid local mesh (every face on one side)
        lm = p.mesh.mortars()
        # interior elements come first and read no ghost: no ghost neighbour, no ghost mortar quad
        assert 0 < p.n_interior < p.n_owned
        inner = lnbr[: p.n_interior]
        assert np.all(inner < p.n_owned)
        for row in lm:
            quads = row[[0, 2, 3, 4, 5]]
            if np.any(quads < p.n_interior):
                assert np.all(quads < p.n_owned)
        # both owned blocks keep the element order
        assert np.all(np.diff(p.glob[: p.n_interior]) > 0) and np.all(np.diff(p.glob[p.n_interior: p.n_owned]) > 0)
        for e in range(p.n_owned):
            for f in range(6):
                if lnbr[e, f] >= 0:
                    assert p.glob[lnbr[e, f]] == gnbr[p.glob[e], f]
                else:
                    assert (lnbr[e, f] == -1) == (gnbr[p.glob[e], f] == -1)
        for row in lm:   # local mortars are global mortars
            g = p.glob[row[[0, 2, 3, 4, 5]]]
            gm = m.mortars()
            assert any(gr[0] == g[0] and gr[1] == row[1] and np.array_equal(gr[2:], g[1:]) for gr in gm)
        for peer, idx in p.send.items():
            assert np.array_equal(p.glob[idx], parts[peer].glob[parts[peer].recv[p.rank]])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir, nsteps):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = blast_state(m)
        part = partition.partition(m, world)[rank]
        cfg = abi.NemoCfg()   # built by hand: the CUDA library is not loaded on CPU ranks
        cfg.n_nodes, cfg.n_vars, cfg.eqn = 4, 5, abi.EQN_EULER
        cfg.volume_flux, cfg.surface_flux, cfg.precision = 0, 0, 0
        cfg.indicator, cfg.alpha_smoothing, cfg.positivity = abi.IND_MODAL, 1, 1
        cfg.kappa, cfg.mu0, cfg.cfl, cfg.alpha_max, cfg.alpha_min, cfg.repair_decr = 1.4, 1.0, 0.5, 0.5, 0.001, 0.01
        lm = part.mesh
        o = orc.Oracle.for_mesh(cfg, lm, nthreads=1)
        ul = np.ascontiguousarray(u[:, part.glob])
        reg = np.zeros_like(ul)
        V = ul.shape[0]
        own = part.n_owned

        def get_rows(idx):
            return torch.from_numpy(np.ascontiguousarray(ul[:, idx].transpose(1, 0, 2)).reshape(len(idx), -1))

        def set_rows(idx, buf):
            ul[:, idx] = buf.numpy().reshape(len(idx), V, 64).transpose(1, 0, 2)

        def make_buffer(n):
            return torch.empty((n, V * 64), dtype=torch.float64)

        for _ in range(nsteps):
            partition.exchange(part, dist, get_rows, set_rows, make_buffer)
            dt_loc = orc.lib().or_timestep(o._c(), own, orc._p(np.ascontiguousarray(lm.delta[:own])),
                                           orc._p(np.ascontiguousarray(ul[:, :own])), None)
            dt = torch.tensor([dt_loc], dtype=torch.float64)
            dist.all_reduce(dt, op=dist.ReduceOp.MIN)
            for st in range(5):
                if st > 0:
                    partition.exchange(part, dist, get_rows, set_rows, make_buffer)
                o.stage(ul, reg, st, float(dt.item()))
        order = np.argsort(part.glob[:own])   # owned elements in global order
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), ul[:, :own][:, order])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_oracle_run_matches_single_process(world, tmp_path):
    import torch.multiprocessing as tmp
    orc.build()
    nsteps = 3
    tmp.spawn(_worker, args=(world, _free_port(), str(tmp_path), nsteps), nprocs=world, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)], axis=1)
    m = band_forest()
    u = blast_state(m)
    c = abi.NemoCfg()
    c.n_nodes, c.n_vars, c.eqn = 4, 5, abi.EQN_EULER
    c.indicator, c.alpha_smoothing, c.positivity = abi.IND_MODAL, 1, 1
    c.kappa, c.mu0, c.cfl, c.alpha_max, c.alpha_min, c.repair_decr = 1.4, 1.0, 0.5, 0.5, 0.001, 0.01
    ref, _, n, _ = orc.Oracle.for_mesh(c, m).run(u, nsteps=nsteps)
    assert n == nsteps
    assert np.array_equal(got, ref)


def _face_nodes(f):
    """Node indices of face f (the library's face order: j = a + 4 b over the tangential axes)."""
    d, end = f >> 1, (3 if f & 1 else 0)
    out = []
    for j in range(16):
        a, b = j & 3, j >> 2
        out.append([end + 4 * a + 16 * b, a + 4 * end + 16 * b, a + 4 * b + 16 * end][d])
    return np.array(out)


@pytest.mark.parametrize("nranks", [2, 3])
def test_face_plan(nranks):
    """Every trace a rank reads from a ghost is in its face plan, sender and receiver list the same
    (global element, face) in the same order, and the plan moves far less than whole elements."""
    m = band_forest()
    parts = partition.partition(m, nranks)
    for p in parts:
        lnbr = p.mesh.neighbors()
        need = set()
        for e in range(p.n_owned):               # conforming neighbours of owned elements
            for f in range(6):
                n = lnbr[e, f]
                if n >= p.n_owned:
                    need.add((int(p.glob[n]), f ^ 1))
        for row in p.mesh.mortars():            # every quad of a local mortar
            qc, fc = int(row[0]), int(row[1])
            if qc >= p.n_owned:
                need.add((int(p.glob[qc]), fc))
            for q in row[2:]:
                if q >= p.n_owned:
                    need.add((int(p.glob[q]), fc ^ 1))
        got = {(int(p.glob[i]), int(f)) for idx, fs in p.recv_f.values() for i, f in zip(idx, fs)}
        assert need <= got
        for peer, (idx, fs) in p.send_f.items():
            ridx, rfs = parts[peer].recv_f[p.rank]
            assert np.array_equal(p.glob[idx], parts[peer].glob[ridx]) and np.array_equal(fs, rfs)
            assert np.all(idx < p.n_owned)
        nf = sum(len(v[0]) for v in p.send_f.values())
        ne = sum(len(v) for v in p.send.values())
        assert nf * (5 * 16 + 1) < 0.35 * ne * (5 * 64 + 1)


def _face_worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = blast_state(m)
        alpha = np.linspace(0.0, 0.5, m.E)
        part = partition.partition(m, world)[rank]
        ul = np.zeros((u.shape[0], len(part.glob), 64))
        ul[:, : part.n_owned] = u[:, part.glob[: part.n_owned]]
        al = np.zeros(len(part.glob))
        al[: part.n_owned] = alpha[part.glob[: part.n_owned]]
        V = u.shape[0]

        def get_rows(ent):
            idx, fs = ent
            rows = [np.concatenate([ul[:, i][:, _face_nodes(f)].ravel(), [al[i]]]) for i, f in zip(idx, fs)]
            return torch.from_numpy(np.array(rows))

        def set_rows(ent, buf):
            b = buf.numpy()
            for k, (i, f) in enumerate(zip(*ent)):
                ul[:, i, _face_nodes(f)] = b[k, : V * 16].reshape(V, 16)
                al[i] = b[k, -1]

        partition.exchange(part, dist, get_rows, set_rows,
                           lambda n: torch.empty((n, V * 16 + 1), dtype=torch.float64), faces=True)
        ok = True
        for idx, fs in part.recv_f.values():
            for i, f in zip(idx, fs):
                g = part.glob[i]
                ok = ok and np.array_equal(ul[:, i, _face_nodes(f)], u[:, g, _face_nodes(f)]) and al[i] == alpha[g]
        np.save(os.path.join(out_dir, f"ok{rank}.npy"), np.array([ok]))
    finally:
        dist.destroy_process_group()


def test_face_exchange_gloo(tmp_path):
    import torch.multiprocessing as tmp
    tmp.spawn(_face_worker, args=(3, _free_port(), str(tmp_path)), nprocs=3, join=True)
    assert all(bool(np.load(tmp_path / f"ok{r}.npy")[0]) for r in range(3))


def mhd_cfg():
    c = abi.cfg_struct(eqn=abi.EQN_MHD, n_vars=9, volume_flux=abi.VOLFLUX_EC_MHD, surface_flux=abi.SURFFLUX_HLLD,
                       kappa=5.0 / 3.0, mu0=1.0, indicator=abi.IND_MODAL, positivity=1)
    return c


def _mhd_worker(rank, world, port, out_dir, nsteps):
    """GLM-MHD on gloo ranks: the oracle stage on the rank's share, Δt all-reduced (MIN), the wave and
    velocity maxima all-reduced (MAX) into the cleaning speed of every rank, the ghost exchange
    posted before and finished after the interior work of each stage (begin / end)."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = np.ascontiguousarray(setups.orszag_tang(m))
        part = partition.partition(m, world)[rank]
        cfg = mhd_cfg()
        lm = part.mesh
        o = orc.Oracle.for_mesh(cfg, lm, nthreads=1)
        ul = np.ascontiguousarray(u[:, part.glob])
        reg = np.zeros_like(ul)
        V, own = ul.shape[0], part.n_owned

        def get_rows(idx):
            return torch.from_numpy(np.ascontiguousarray(ul[:, idx].transpose(1, 0, 2)).reshape(len(idx), -1))

        def set_rows(idx, buf):
            ul[:, idx] = buf.numpy().reshape(len(idx), V, 64).transpose(1, 0, 2)

        def make_buffer(n):
            return torch.empty((n, V * 64), dtype=torch.float64)

        delta_own = np.ascontiguousarray(lm.delta[:own])
        for _ in range(nsteps):
            partition.exchange(part, dist, get_rows, set_rows, make_buffer)
            lmx, vmx = orc.ctypes.c_double(), orc.ctypes.c_double()
            dt_loc = orc.lib().or_timestep2(o._c(), own, orc._p(delta_own), orc._p(np.ascontiguousarray(ul[:, :own])),
                                            orc.ctypes.byref(lmx), orc.ctypes.byref(vmx))
            lmax, vmax = lmx.value, vmx.value
            dt = torch.tensor([dt_loc], dtype=torch.float64)
            dist.all_reduce(dt, op=dist.ReduceOp.MIN)
            sp = torch.tensor([lmax, vmax], dtype=torch.float64)
            dist.all_reduce(sp, op=dist.ReduceOp.MAX)
            cfg.glm_ch = 2.0 * abs(float(sp[0]) - float(sp[1]))
            cfg.glm_alpha = cfg.glm_ch / 0.18
            for st in range(5):
                if st > 0:
                    h = partition.exchange_begin(part, dist, get_rows, make_buffer)
                    partition.exchange_end(h, set_rows)
                o.stage(ul, reg, st, float(dt.item()))
        order = np.argsort(part.glob[:own])
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), ul[:, :own][:, order])
    finally:
        dist.destroy_process_group()


def test_partitioned_mhd_oracle_run_matches_single_process(tmp_path):
    import torch.multiprocessing as tmp
    orc.build()
    nsteps = 2
    tmp.spawn(_mhd_worker, args=(2, _free_port(), str(tmp_path), nsteps), nprocs=2, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(2)], axis=1)
    m = band_forest()
    u = setups.orszag_tang(m)
    ref, _, n, _ = orc.Oracle.for_mesh(mhd_cfg(), m).run(u, nsteps=nsteps)
    assert n == nsteps
    assert np.array_equal(got, ref)


def _overlap_worker(rank, world, port, out_dir):
    """exchange_begin posts the transfers; work between begin and end; exchange_end delivers the
    same traces as a back-to-back exchange."""
    import time
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = band_forest()
        u = blast_state(m)
        part = partition.partition(m, world)[rank]
        V = u.shape[0]
        ul = np.zeros((V, len(part.glob), 64))
        ul[:, : part.n_owned] = u[:, part.glob[: part.n_owned]]

        def get_rows(ent):
            idx, fs = ent
            return torch.from_numpy(np.array([ul[:, i][:, _face_nodes(f)].ravel() for i, f in zip(idx, fs)]))

        def set_rows(ent, buf):
            b = buf.numpy()
            for k, (i, f) in enumerate(zip(*ent)):
                ul[:, i, _face_nodes(f)] = b[k].reshape(V, 16)

        h = partition.exchange_begin(part, dist, get_rows, lambda n: torch.empty((n, V * 16), dtype=torch.float64),
                                     faces=True)
        time.sleep(0.05 * (rank + 1))           # "interior work" of uneven length on the ranks
        partition.exchange_end(h, set_rows)
        ok = all(np.array_equal(ul[:, i, _face_nodes(f)], u[:, part.glob[i], _face_nodes(f)])
                 for idx, fs in part.recv_f.values() for i, f in zip(idx, fs))
        np.save(os.path.join(out_dir, f"ok{rank}.npy"), np.array([ok]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_begin_end_with_work_between(world, tmp_path):
    import torch.multiprocessing as tmp
    tmp.spawn(_overlap_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    assert all(bool(np.load(tmp_path / f"ok{r}.npy")[0]) for r in range(world))
