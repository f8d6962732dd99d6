"""Element meshes in the reference's side form.

The reference takes its connectivity from p4est through p4wrap (source/mesh/p4est/mesh_utils_mod.f90:
160-441): a list of quads with delta/center and a list of sides, each side joining the quads on its two
halves (nquads 1, or 4 on the fine half of a 2:1 non-conforming face) with the face id each quad sees.
p4est is not available here, so this module generates the same structures for uniform bricks (periodic
or not) and for statically refined, 2:1-balanced forests, with elements in Morton (Z) order so that
consecutive elements are spatially compact (2x2x2 blocks of eight on a uniform brick).
"""
import numpy as np

NOR, SOU, WES, EAS, FRO, BAC = range(6)


def _part1by2(x):
    x = np.asarray(x, dtype=np.int64) & 0x1FFFFF
    x = (x | (x << 32)) & 0x1F00000000FFFF
    x = (x | (x << 16)) & 0x1F0000FF0000FF
    x = (x | (x << 8)) & 0x100F00F00F00F00F
    x = (x | (x << 4)) & 0x10C30C30C30C30C3
    x = (x | (x << 2)) & 0x1249249249249249
    return x


def morton3(ix, iy, iz):
    return _part1by2(ix) | (_part1by2(iy) << 1) | (_part1by2(iz) << 2)


class Mesh:
    """delta/center [E,3]; sides: quads [S,2,4] (0-based, -1 unused), faceid [S,2], nquads [S,2],
    boundary [S] (0 interior, 1+face id at the domain boundary)."""

    def __init__(self, delta, center, side_quads, side_faceid, side_nquads, boundary, level=None):
        self.delta = np.ascontiguousarray(delta, dtype=np.float64)
        self.center = np.ascontiguousarray(center, dtype=np.float64)
        self.side_quads = np.ascontiguousarray(side_quads, dtype=np.int32)
        self.side_faceid = np.ascontiguousarray(side_faceid, dtype=np.int8)
        self.side_nquads = np.ascontiguousarray(side_nquads, dtype=np.int8)
        self.boundary = np.ascontiguousarray(boundary, dtype=np.int32)
        self.E = self.delta.shape[0]
        self.S = self.side_quads.shape[0]
        self.level = level if level is not None else np.zeros(self.E, dtype=np.int8)

    def neighbors(self):
        """Conforming face neighbours [E,6] (-1 at a domain boundary); raises on mortars."""
        nbr = np.full((self.E, 6), -2, dtype=np.int32)
        for s in range(self.S):
            nq = self.side_nquads[s]
            if nq[0] > 1 or nq[1] > 1:
                raise ValueError("neighbors(): mesh has non-conforming sides")
            q0, q1 = self.side_quads[s, 0, 0], self.side_quads[s, 1, 0]
            f0, f1 = int(self.side_faceid[s, 0]), int(self.side_faceid[s, 1])
            if nq[1] == 0:
                nbr[q0, f0] = -1
            else:
                nbr[q0, f0] = q1
                nbr[q1, f1] = q0
        if (nbr == -2).any():
            raise ValueError("neighbors(): element face without a side")
        return nbr

    def node_coords(self, nodes):
        """Node coordinates [3,E,n^3] for Gauss-Lobatto nodes on [-1,1] (quad_get_coords,
        source/mesh/p4est/quad_utils_mod.f90:176-206)."""
        n = len(nodes)
        xi = np.asarray(nodes)
        i = np.arange(n ** 3) % n
        j = (np.arange(n ** 3) // n) % n
        k = np.arange(n ** 3) // (n * n)
        out = np.empty((3, self.E, n ** 3))
        for d, ii in enumerate((i, j, k)):
            out[d] = self.center[:, d:d + 1] + 0.5 * xi[ii][None, :] * self.delta[:, d:d + 1]
        return out


def brick(nx, ny=None, nz=None, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), periodic=(True, True, True)):
    """Uniform nx*ny*nz brick, Morton-ordered elements, one side per element face pair."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    order = np.argsort(morton3(ix, iy, iz), kind="stable")
    ix, iy, iz = ix[order], iy[order], iz[order]
    E = nx * ny * nz
    eid = np.empty((nx, ny, nz), dtype=np.int64)
    eid[ix, iy, iz] = np.arange(E)
    dx = (hi - lo) / np.array([nx, ny, nz])
    delta = np.tile(dx, (E, 1))
    center = lo + (np.stack([ix, iy, iz], axis=1) + 0.5) * dx
    dims = (nx, ny, nz)
    idx = (ix, iy, iz)
    Q, F, NQ, B = [], [], [], []
    for d in range(3):
        plus_face, minus_face = 2 * d + 1, 2 * d
        up = list(idx)
        up[d] = idx[d] + 1
        at_edge = up[d] == dims[d]
        up[d] = np.where(at_edge, 0, up[d])
        nb = eid[up[0], up[1], up[2]]
        inner = ~at_edge | bool(periodic[d])
        e_in = np.nonzero(inner)[0]
        q = np.full((len(e_in), 2, 4), -1, dtype=np.int32)
        q[:, 0, 0] = e_in
        q[:, 1, 0] = nb[e_in]
        Q.append(q); F.append(np.tile([plus_face, minus_face], (len(e_in), 1)))
        NQ.append(np.tile([1, 1], (len(e_in), 1))); B.append(np.zeros(len(e_in), dtype=np.int32))
        if not periodic[d]:
            for face, sel in ((plus_face, np.nonzero(at_edge)[0]), (minus_face, np.nonzero(idx[d] == 0)[0])):
                q = np.full((len(sel), 2, 4), -1, dtype=np.int32)
                q[:, 0, 0] = sel
                Q.append(q); F.append(np.tile([face, face ^ 1], (len(sel), 1)))
                NQ.append(np.tile([1, 0], (len(sel), 1))); B.append(np.full(len(sel), 1 + face, dtype=np.int32))
    quads, fids, nqs, bnd = (np.concatenate(Q), np.concatenate(F), np.concatenate(NQ), np.concatenate(B))
    return Mesh(delta, center, quads, fids, nqs, bnd)


def ensemble(members, nx):
    """members independent periodic nx^3 bricks on [0,1]^3, stacked; returns (mesh, group_of_elem)."""
    one = brick(nx)
    E1, S1 = one.E, one.S
    quads = np.concatenate([np.where(one.side_quads >= 0, one.side_quads + m * E1, -1) for m in range(members)])
    mesh = Mesh(np.tile(one.delta, (members, 1)), np.tile(one.center, (members, 1)), quads,
                np.tile(one.side_faceid, (members, 1)), np.tile(one.side_nquads, (members, 1)),
                np.tile(one.boundary, members))
    groups = np.repeat(np.arange(members, dtype=np.int32), E1)
    return mesh, groups
