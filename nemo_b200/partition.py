"""Element partition of a mesh over processes, with ghost copies of the face neighbours.

The reference partitions its quads over MPI ranks along the p4est space-filling curve and exchanges
the payloads of the partition-boundary quads every stage (source/mesh/p4est/mesh_utils_mod.f90:
623-675 for the exchange, :1014- for the partition); the time step is an MPI_Allreduce minimum
(source/kernel/mcfv/3d/kernel_timestep_mod.f90:48-52).  Here rank r takes a contiguous range of the
element list (Morton order, so the ranges are compact), and its local mesh is those elements followed
by ghost copies of every element that shares a side with one of them (conforming neighbours and the
other quads of a 2:1 mortar).  Before every RK stage each rank sends the current state and raw
blending coefficient of the owned elements that other ranks hold as ghosts; the ghosts' remaining
faces become boundary sides (they are never advanced, only read).  Each element's update only reads
its own state and its neighbours' traces, so every owned element evolves exactly as in the unsplit
run.

One exchange per stage, point to point (torch.distributed isend/irecv: NCCL with device buffers on
GPUs, gloo with host buffers on CPUs), and one minimum reduction of the time step per step.  A
ghost is only read through the traces on the faces that the rank's sides touch (its conforming
neighbours' faces and the mortars it belongs to) and through its raw blending coefficient, so the
exchange moves those faces: one row of V x 16 trace values + the coefficient per (ghost, face),
a quarter of the element's payload for a ghost with one shared face (the reference exchanges
whole payloads).  The whole-element form is kept beside it.
"""
from dataclasses import dataclass, field

import numpy as np

from .mesh import Mesh


@dataclass
class Part:
    """One rank's share: local mesh (owned elements first: those that read no ghost data, then the
    partition-boundary ones; then the ghosts), global id of each local element, and the exchange
    plan (local element indices, matched in order between sender and receiver)."""
    rank: int
    mesh: Mesh
    n_owned: int
    glob: np.ndarray                                  # [E_local] global element ids
    n_interior: int = 0                               # owned elements [0, n_interior) read no ghost
    send: dict = field(default_factory=dict)          # peer -> local owned indices to send
    recv: dict = field(default_factory=dict)          # peer -> local ghost indices to fill
    send_f: dict = field(default_factory=dict)        # peer -> (local owned indices, face ids) to send
    recv_f: dict = field(default_factory=dict)        # peer -> (local ghost indices, face ids) to fill
    ghost_faces: list = field(default_factory=list)   # (global element, face) read from ghosts


def owner_ranges(E, nranks):
    """Contiguous, balanced element ranges [lo_r, hi_r) along the element order."""
    b = [(E * r) // nranks for r in range(nranks + 1)]
    return [(b[r], b[r + 1]) for r in range(nranks)]


def partition(mesh, nranks, interior_first=True):
    """Split mesh over nranks ranks; returns [Part] (one per rank).  With interior_first, each rank's
    owned elements are ordered so that those whose sides touch no ghost come first (n_interior of
    them, in element order), then the partition-boundary ones: a stage can then advance the interior
    while the ghost traces are in flight."""
    E = mesh.E
    ranges = owner_ranges(E, nranks)
    owner = np.empty(E, dtype=np.int64)
    for r, (lo, hi) in enumerate(ranges):
        owner[lo:hi] = r
    # quads of every side (1, 2 or 5 of them), -1 where unused
    sq = np.asarray(mesh.side_quads, dtype=np.int64)
    nq = np.asarray(mesh.side_nquads, dtype=np.int64)
    valid = np.arange(4)[None, None, :] < nq[:, :, None]
    qv = np.where(valid, sq, -1)
    fid = np.asarray(mesh.side_faceid, dtype=np.int64)
    parts = []
    for r, (lo, hi) in enumerate(ranges):
        mine = (qv >= lo) & (qv < hi)
        sides = np.nonzero(mine.any(axis=(1, 2)))[0]
        qs = qv[sides]
        ghost_q = (qs >= 0) & ((qs < lo) | (qs >= hi))
        other = qs[ghost_q]
        need = np.unique(other)                 # ghosts, ascending (= by owner, then id)
        owned = np.arange(lo, hi)
        n_int = hi - lo
        if interior_first:
            # owned quads on a side that also holds a ghost (a conforming neighbour or another quad
            # of a 2:1 mortar) read ghost data
            touch = ghost_q.any(axis=(1, 2))
            bq = qs[touch]
            bq = np.unique(bq[(bq >= lo) & (bq < hi)])
            is_b = np.zeros(hi - lo, dtype=bool)
            is_b[bq - lo] = True
            owned = np.concatenate([owned[~is_b], owned[is_b]])
            n_int = int((~is_b).sum())
        glob = np.concatenate([owned, need]).astype(np.int64)
        loc = np.full(E, -1, dtype=np.int64)
        loc[glob] = np.arange(len(glob))
        Q = np.where(qs >= 0, loc[np.maximum(qs, 0)], -1).astype(np.int32)
        F = fid[sides].astype(np.int8)
        NQ = nq[sides].astype(np.int8)
        B = np.asarray(mesh.boundary, dtype=np.int32)[sides]
        # (local element, face) pairs on the included sides
        vmask = qs >= 0
        ce = Q.astype(np.int64)[vmask]
        cf = np.broadcast_to(F.astype(np.int64)[:, :, None], qs.shape)[vmask]
        nown, nloc = hi - lo, len(glob)
        cov = np.zeros((nloc, 6), dtype=bool)
        cov[ce, cf] = True
        # faces of ghosts that no included side covers: boundary sides (mirrored state, never used)
        gi, gf = np.nonzero(~cov[nown:])
        gi = gi + nown
        if len(gi):
            qb = np.full((len(gi), 2, 4), -1, dtype=np.int32)
            qb[:, 0, 0] = gi
            Q = np.concatenate([Q, qb])
            F = np.concatenate([F, np.stack([gf, gf ^ 1], axis=1).astype(np.int8)])
            NQ = np.concatenate([NQ, np.tile(np.array([1, 0], dtype=np.int8), (len(gi), 1))])
            B = np.concatenate([B, (1 + gf).astype(np.int32)])
        local = Mesh(mesh.delta[glob], mesh.center[glob], Q, F, NQ, B, level=mesh.level[glob])
        part = Part(rank=r, mesh=local, n_owned=nown, glob=glob, n_interior=n_int)
        # ghost faces on the included sides: the traces this rank reads from other ranks' elements
        hi_i, hi_f = np.nonzero(cov[nown:])
        part.ghost_faces = [(int(glob[i + nown]), int(f)) for i, f in zip(hi_i, hi_f)]
        parts.append(part)
    # local index of every global element on its owner
    local_of = []
    for pr in parts:
        lo_map = np.full(E, -1, dtype=np.int64)
        lo_map[pr.glob[: pr.n_owned]] = np.arange(pr.n_owned)
        local_of.append(lo_map)
    # exchange plan: rank r receives its ghosts owned by p; p sends them in the same (global) order
    for r, pr in enumerate(parts):
        ghosts = pr.glob[pr.n_owned:]
        for p in range(nranks):
            sel = np.nonzero(owner[ghosts] == p)[0]
            if len(sel) == 0:
                continue
            pr.recv[p] = (pr.n_owned + sel).astype(np.int32)
            parts[p].send[r] = local_of[p][ghosts[sel]].astype(np.int32)
    # face plan: rank r receives its ghost faces owned by p; p sends them in the same (global) order
    for r, pr in enumerate(parts):
        loc = {int(g): i for i, g in enumerate(pr.glob)}
        for p in range(nranks):
            ent = [(g, f) for g, f in pr.ghost_faces if owner[g] == p]
            if not ent:
                continue
            gids = np.array([g for g, _ in ent], dtype=np.int64)
            fids = np.array([f for _, f in ent], dtype=np.int32)
            pr.recv_f[p] = (np.array([loc[int(g)] for g in gids], dtype=np.int32), fids)
            parts[p].send_f[r] = (local_of[p][gids].astype(np.int32), fids.copy())
    return parts


def exchange_begin(part, dist, get_rows, make_buffer, faces=False):
    """Post one ghost refresh: get_rows(entries) -> buffer of those local entries (taken now),
    make_buffer(n) -> an empty receive buffer for n entries.  Entries are element index arrays, or
    (element, face) array pairs with faces=True.  Sends and receives are posted together
    (batch_isend_irecv), so no ordering between peers is needed; returns a handle for
    exchange_end.  Work that reads no ghost can run between the two calls."""
    ops, incoming = [], []
    send, recv = (part.send_f, part.recv_f) if faces else (part.send, part.recv)
    count = (lambda ent: len(ent[0])) if faces else len
    for peer, idx in sorted(send.items()):
        ops.append(dist.P2POp(dist.isend, get_rows(idx), peer))
    for peer, idx in sorted(recv.items()):
        buf = make_buffer(count(idx))
        incoming.append((idx, buf))
        ops.append(dist.P2POp(dist.irecv, buf, peer))
    reqs = dist.batch_isend_irecv(ops) if ops else []
    return reqs, incoming


def exchange_end(handle, set_rows, device_sync=None):
    """Finish a ghost refresh: wait for the transfers, then set_rows(entries, buffer) for every
    received buffer.  device_sync: called after the waits when the receive buffers are device
    memory written on the communication library's stream (NCCL), before they are read elsewhere."""
    reqs, incoming = handle
    for req in reqs:
        req.wait()
    if device_sync and reqs:
        device_sync()
    for idx, buf in incoming:
        set_rows(idx, buf)


def exchange(part, dist, get_rows, set_rows, make_buffer, faces=False):
    """One ghost refresh, begin and end back to back (see exchange_begin / exchange_end)."""
    exchange_end(exchange_begin(part, dist, get_rows, make_buffer, faces=faces), set_rows)


class PartitionedRun:
    """Advance one rank's share on its GPU.  Per stage: the owned traces that other ranks read are
    packed by the library and sent (the ghost faces by default, whole elements with faces=False);
    while they are in flight the library advances the owned elements that read no ghost
    (nemo_gpu_stage_interior); once the ghosts are refreshed it advances the partition-boundary
    elements (nemo_gpu_stage_boundary).  Δt is the all-reduce minimum of the ranks' CFL bounds; for
    GLM-MHD the wave and velocity maxima are all-reduced too and set the cleaning speed
    c_h = 2 |λmax − vmax| and damping c_h / 0.18 of every rank (source/kernel/mcfv/3d/
    kernel_timestep_mod.f90:48-52, :338-344).  overlap=False runs each stage whole after the
    refresh (the reference's order)."""

    def __init__(self, cfg, part, dist, host_buffers=None, faces=True, overlap=True):
        import torch
        from . import abi
        from .solver import Solver
        if cfg.eqn not in (abi.EQN_EULER, abi.EQN_MHD):
            raise ValueError("unknown equations")
        self.torch, self.abi, self.dist, self.part = torch, abi, dist, part
        self.cfg = cfg
        self.mhd = cfg.eqn == abi.EQN_MHD
        self.faces = faces
        self.overlap = overlap
        self.s = Solver(cfg, part.mesh)
        abi.call("nemo_gpu_set_owned", int(part.n_owned))
        abi.call("nemo_gpu_set_interior", int(part.n_interior if overlap else 0))
        self.row = cfg.n_vars * (16 if faces else 64) + 1
        # gloo moves host tensors, NCCL device tensors
        self.host = (dist.get_backend() != "nccl") if host_buffers is None else host_buffers
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.idx_dev = {}
        plans = (part.send_f, part.recv_f) if faces else (part.send, part.recv)
        for d in plans:
            for peer, ent in d.items():
                if faces:
                    self.idx_dev[id(ent)] = (torch.as_tensor(ent[0], dtype=torch.int32, device=dev),
                                             torch.as_tensor(ent[1], dtype=torch.int32, device=dev))
                else:
                    self.idx_dev[id(ent)] = torch.as_tensor(ent, dtype=torch.int32, device=dev)
        self.bytes_per_exchange = sum(
            (len(e[0]) if faces else len(e)) for e in plans[0].values()) * self.row * 8
        self.order = np.argsort(part.glob[: part.n_owned], kind="stable")   # local owned -> global order

    def _get(self, ent):
        t, vp = self.torch, self.abi.ctypes.c_void_p
        n = len(ent[0]) if self.faces else len(ent)
        buf = t.empty((n, self.row), dtype=t.float64, device=self.dev)
        if self.faces:
            i, f = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_pack_faces", vp(i.data_ptr()), vp(f.data_ptr()), n, vp(buf.data_ptr()))
        else:
            i = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_pack_elements", vp(i.data_ptr()), n, vp(buf.data_ptr()))
        return buf.cpu() if self.host else buf

    def _set(self, ent, buf):
        vp = self.abi.ctypes.c_void_p
        if self.host:
            b = buf.to(self.dev)
            self.torch.cuda.current_stream().synchronize()   # the copy is on torch's stream
        else:
            b = buf.contiguous()
        if self.faces:
            i, f = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_unpack_faces", vp(i.data_ptr()), vp(f.data_ptr()), len(ent[0]), vp(b.data_ptr()))
        else:
            i = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_unpack_elements", vp(i.data_ptr()), len(ent), vp(b.data_ptr()))

    def _buf(self, n):
        t = self.torch
        return t.empty((n, self.row), dtype=t.float64, device="cpu" if self.host else self.dev)

    def _device_sync(self):
        # NCCL writes the receive buffers on its own stream; req.wait() orders torch's current
        # stream after it, and the library reads them on its stream: wait for torch's stream
        if not self.host:
            self.torch.cuda.current_stream().synchronize()

    def upload(self, u_local):
        self.s.upload(u_local)

    def exchange_begin(self):
        return exchange_begin(self.part, self.dist, self._get, self._buf, faces=self.faces)

    def exchange_end(self, handle):
        exchange_end(handle, self._set, self._device_sync)

    def exchange(self):
        self.exchange_end(self.exchange_begin())

    def timestep(self):
        """Δt of the step (all ranks), and for GLM-MHD the global cleaning speed set on every rank."""
        t = self.torch
        dev = "cpu" if self.host else self.dev
        dt_loc, lmax = self.s.calc_timestep(self.cfg.cfl)
        dt = t.tensor([dt_loc], dtype=t.float64, device=dev)
        self.dist.all_reduce(dt, op=self.dist.ReduceOp.MIN)
        if self.mhd:
            lm, vm = self.abi.ctypes.c_double(), self.abi.ctypes.c_double()
            self.abi.call("nemo_gpu_glm_speeds", self.abi.ctypes.byref(lm), self.abi.ctypes.byref(vm))
            sp = t.tensor([lm.value, vm.value], dtype=t.float64, device=dev)
            self.dist.all_reduce(sp, op=self.dist.ReduceOp.MAX)
            lmax_g, vmax_g = (float(x) for x in sp.cpu())
            ch = 2.0 * abs(lmax_g - vmax_g)
            self.abi.call("nemo_gpu_set_glm", ch, ch / 0.18)
        return float(dt.item())

    def step(self):
        self.exchange()   # ghosts' state and raw blending coefficients for the CFL bound and stage 1
        dt = self.timestep()
        nb = self.abi.ctypes.c_int32()
        for st in range(1, 6):
            h = self.exchange_begin() if st > 1 else None
            self.abi.call("nemo_gpu_stage_interior", st, dt)       # reads no ghost: overlaps the transfer
            if h is not None:
                self.exchange_end(h)
            self.abi.call("nemo_gpu_stage_boundary", st, dt, self.abi.ctypes.byref(nb))
        return dt

    def run(self, nsteps):
        return [self.step() for _ in range(nsteps)]

    def download_owned(self):
        """The owned elements' state, [V][n_owned][64] in global element order."""
        return self.s.download()[:, : self.part.n_owned][:, self.order]
