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
    """One rank's share: local mesh (owned elements first), global id of each local element, and
    the exchange plan (local element indices, matched in order between sender and receiver)."""
    rank: int
    mesh: Mesh
    n_owned: int
    glob: np.ndarray                                  # [E_local] global element ids
    send: dict = field(default_factory=dict)          # peer -> local owned indices to send
    recv: dict = field(default_factory=dict)          # peer -> local ghost indices to fill
    send_f: dict = field(default_factory=dict)        # peer -> (local owned indices, face ids) to send
    recv_f: dict = field(default_factory=dict)        # peer -> (local ghost indices, face ids) to fill
    ghost_faces: list = field(default_factory=list)   # (global element, face) read from ghosts


def owner_ranges(E, nranks):
    """Contiguous, balanced element ranges [lo_r, hi_r) along the element order."""
    b = [(E * r) // nranks for r in range(nranks + 1)]
    return [(b[r], b[r + 1]) for r in range(nranks)]


def partition(mesh, nranks):
    """Split mesh over nranks ranks; returns [Part] (one per rank)."""
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
        other = qs[(qs >= 0) & ((qs < lo) | (qs >= hi))]
        need = np.unique(other)                 # ghosts, ascending (= by owner, then id)
        glob = np.concatenate([np.arange(lo, hi), need]).astype(np.int64)
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
        part = Part(rank=r, mesh=local, n_owned=nown, glob=glob)
        # ghost faces on the included sides: the traces this rank reads from other ranks' elements
        hi_i, hi_f = np.nonzero(cov[nown:])
        part.ghost_faces = [(int(glob[i + nown]), int(f)) for i, f in zip(hi_i, hi_f)]
        parts.append(part)
    # exchange plan: rank r receives its ghosts owned by p; p sends them in the same (global) order
    for r, pr in enumerate(parts):
        ghosts = pr.glob[pr.n_owned:]
        for p in range(nranks):
            sel = np.nonzero(owner[ghosts] == p)[0]
            if len(sel) == 0:
                continue
            pr.recv[p] = (pr.n_owned + sel).astype(np.int32)
            lo_p = ranges[p][0]
            parts[p].send[r] = (ghosts[sel] - lo_p).astype(np.int32)
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
            parts[p].send_f[r] = ((gids - ranges[p][0]).astype(np.int32), fids.copy())
    return parts


def exchange(part, dist, get_rows, set_rows, make_buffer, faces=False):
    """One ghost refresh: get_rows(entries) -> buffer of those local entries, set_rows(entries,
    buffer); make_buffer(n) -> an empty receive buffer for n entries.  Entries are element index
    arrays, or (element, face) array pairs with faces=True.  Sends and receives are posted together
    (batch_isend_irecv) so no ordering between peers is needed."""
    ops, incoming = [], []
    send, recv = (part.send_f, part.recv_f) if faces else (part.send, part.recv)
    count = (lambda ent: len(ent[0])) if faces else len
    for peer, idx in sorted(send.items()):
        ops.append(dist.P2POp(dist.isend, get_rows(idx), peer))
    for peer, idx in sorted(recv.items()):
        buf = make_buffer(count(idx))
        incoming.append((idx, buf))
        ops.append(dist.P2POp(dist.irecv, buf, peer))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for idx, buf in incoming:
        set_rows(idx, buf)


class PartitionedRun:
    """Advance one rank's share on its GPU: ghosts refreshed before every stage through the library's
    pack/unpack entry points (the ghost faces by default, whole elements with faces=False),
    Δt = all-reduce minimum of the ranks' CFL bounds.  Euler only (the GLM cleaning speed of MHD
    would need its own all-reduce of λmax and vmax)."""

    def __init__(self, cfg, part, dist, host_buffers=None, faces=True):
        import torch
        from . import abi
        from .solver import Solver
        if cfg.eqn != abi.EQN_EULER:
            raise ValueError("partitioned runs support the Euler equations only")
        if cfg.n_vars != 5:
            raise ValueError("n_vars must be 5")
        self.torch, self.abi, self.dist, self.part = torch, abi, dist, part
        self.cfg = cfg
        self.faces = faces
        self.s = Solver(cfg, part.mesh)
        abi.call("nemo_gpu_set_owned", int(part.n_owned))
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
        b = (buf.to(self.dev) if self.host else buf).contiguous()
        if self.faces:
            i, f = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_unpack_faces", vp(i.data_ptr()), vp(f.data_ptr()), len(ent[0]), vp(b.data_ptr()))
        else:
            i = self.idx_dev[id(ent)]
            self.abi.call("nemo_gpu_unpack_elements", vp(i.data_ptr()), len(ent), vp(b.data_ptr()))

    def _buf(self, n):
        t = self.torch
        return t.empty((n, self.row), dtype=t.float64, device="cpu" if self.host else self.dev)

    def upload(self, u_local):
        self.s.upload(u_local)

    def exchange(self):
        exchange(self.part, self.dist, self._get, self._set, self._buf, faces=self.faces)

    def step(self):
        t = self.torch
        self.exchange()   # ghosts' raw blending coefficients for the CFL-independent first stage
        dt_loc, _ = self.s.calc_timestep(self.cfg.cfl)
        dt = t.tensor([dt_loc], dtype=t.float64, device="cpu" if self.host else self.dev)
        self.dist.all_reduce(dt, op=self.dist.ReduceOp.MIN)
        dt = float(dt.item())
        for st in range(1, 6):
            if st > 1:
                self.exchange()
            self.s.stage(st, dt)
        return dt

    def run(self, nsteps):
        return [self.step() for _ in range(nsteps)]

    def download_owned(self):
        return self.s.download()[:, : self.part.n_owned]
