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

    def _mortar_sides(self):
        return np.nonzero((self.side_nquads == 4).any(axis=1))[0]

    def mortars(self):
        """2:1 mortars [M,6] = (coarse quad, coarse face, fine quads 0..3) in side order; fine quad
        k = s + 2 t sits at half s of the face's first tangential axis and half t of the second."""
        sel = self._mortar_sides()
        out = np.empty((len(sel), 6), dtype=np.int32)
        for m, s in enumerate(sel):
            c = 0 if self.side_nquads[s, 0] == 1 else 1
            out[m, 0] = self.side_quads[s, c, 0]
            out[m, 1] = self.side_faceid[s, c]
            out[m, 2:] = self.side_quads[s, 1 - c, :]
        return out

    def neighbors(self):
        """Face neighbours [E,6]: the conforming neighbour, -1 at a domain boundary, and for a face on
        a 2:1 mortar -2 - slot, where slot = 5 m for the coarse face of mortar m (in side order) and
        5 m + 1 + k for its fine quad k -- the row of that face's flux in the mortar flux buffer."""
        nbr = np.full((self.E, 6), np.iinfo(np.int32).min, dtype=np.int32)
        conf = (self.side_nquads[:, 0] == 1) & (self.side_nquads[:, 1] == 1) & (self.boundary == 0)
        q0, q1 = self.side_quads[conf, 0, 0], self.side_quads[conf, 1, 0]
        f0, f1 = self.side_faceid[conf, 0].astype(np.int64), self.side_faceid[conf, 1].astype(np.int64)
        nbr[q0, f0] = q1
        nbr[q1, f1] = q0
        bnd = (self.side_nquads[:, 1] == 0) | ((self.boundary > 0) & (self.side_nquads[:, 0] == 1))
        nbr[self.side_quads[bnd, 0, 0], self.side_faceid[bnd, 0].astype(np.int64)] = -1
        for m, s in enumerate(self._mortar_sides()):
            c = 0 if self.side_nquads[s, 0] == 1 else 1
            nbr[self.side_quads[s, c, 0], self.side_faceid[s, c]] = -2 - 5 * m
            for k in range(4):
                nbr[self.side_quads[s, 1 - c, k], self.side_faceid[s, 1 - c]] = -2 - (5 * m + 1 + k)
        if (nbr == np.iinfo(np.int32).min).any():
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


def _children(lev, crd, mask):
    """Leaves with the masked ones replaced by their 8 children (child c = sx + 2 sy + 4 sz)."""
    c = np.arange(8)
    kids = np.stack([c & 1, (c >> 1) & 1, c >> 2], axis=1)
    c2 = (2 * crd[mask][:, None, :] + kids[None]).reshape(-1, 3)
    l2 = np.repeat(lev[mask] + 1, 8)
    return np.concatenate([lev[~mask], l2]), np.concatenate([crd[~mask], c2])


def _balance(nb, max_level, lev, crd):
    """2:1 face balance on the finest grid: a leaf whose face neighbour is two or more levels finer is
    split, until none is (level of each finest cell and of its six neighbours, maximum per leaf)."""
    nf = nb << max_level
    while True:
        levgrid = np.empty((nf, nf, nf), dtype=np.int64)
        owner = np.empty((nf, nf, nf), dtype=np.int64)
        for lv in np.unique(lev):   # paint the finest cells of all leaves of one level at once
            sel = np.nonzero(lev == lv)[0]
            s = 1 << (max_level - int(lv))
            o = np.arange(s)
            off = np.stack(np.meshgrid(o, o, o, indexing="ij"), axis=-1).reshape(-1, 3)
            cells = crd[sel][:, None, :] * s + off[None]
            levgrid[cells[..., 0], cells[..., 1], cells[..., 2]] = lv
            owner[cells[..., 0], cells[..., 1], cells[..., 2]] = sel[:, None]
        nbmax = levgrid.copy()
        for d in range(3):
            for sh in (1, -1):
                nbmax = np.maximum(nbmax, np.roll(levgrid, sh, axis=d))
        leafmax = np.zeros(len(lev), dtype=np.int64)
        np.maximum.at(leafmax, owner.ravel(), nbmax.ravel())
        bad = leafmax > lev + 1
        if not bad.any():
            return lev, crd
        lev, crd = _children(lev, crd, bad)


def forest(nb, refine, max_level=2, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """Statically refined periodic forest on an nb^3 base brick (one octree per base element).

    refine(level, center[n,3], size[n]) -> bool[n] marks leaves of that level to split into 8; it is
    called for level 0, 1, ..., max_level-1 in turn.  The forest is then 2:1 face-balanced (a leaf whose
    face neighbour is two or more levels finer is split, repeatedly), the leaves are put in Morton order
    of their anchors on the finest grid (the p4est order), and the sides are built: conforming sides as
    in brick(), and one side per 2:1 non-conforming face with the coarse quad on one half and the four
    fine quads (k = s + 2 t over the face's two tangential axes, lower axis first) on the other.  The
    returned mesh keeps its leaves (mesh.tree: level and integer coordinates) for adapt()."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    g = np.stack(np.meshgrid(np.arange(nb), np.arange(nb), np.arange(nb), indexing="ij"), -1).reshape(-1, 3)
    lev = np.zeros(len(g), dtype=np.int64)
    crd = g.astype(np.int64)
    for level in range(max_level):
        at = lev == level
        if not at.any():
            continue
        size = (hi - lo)[None, :] / (nb << lev[at])[:, None]
        cen = lo + (crd[at] + 0.5) * size
        mask = np.zeros(len(lev), dtype=bool)
        mask[at] = np.asarray(refine(level, cen, size), dtype=bool)
        if mask.any():
            lev, crd = _children(lev, crd, mask)
    lev, crd = _balance(nb, max_level, lev, crd)
    return forest_mesh(nb, max_level, lev, crd, lo, hi)


def forest_mesh(nb, max_level, lev, crd, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """The mesh of a 2:1-balanced leaf set (level, integer coordinates at that level): Morton order of
    the anchors on the finest grid, sides as described in forest()."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    nf = nb << max_level
    lev = np.asarray(lev, dtype=np.int64)
    crd = np.asarray(crd, dtype=np.int64)
    anchor = crd << (max_level - lev)[:, None]
    order = np.argsort(morton3(anchor[:, 0], anchor[:, 1], anchor[:, 2]), kind="stable")
    lev, crd = lev[order], crd[order]
    E = len(lev)
    size = (hi - lo)[None, :] / (nb << lev)[:, None]
    cen = lo + (crd + 0.5) * size

    key_scale = np.int64(nf)
    def key(l, c):
        return ((l * key_scale + c[:, 0]) * key_scale + c[:, 1]) * key_scale + c[:, 2]

    keys = key(lev, crd)
    srt = np.argsort(keys)
    skeys = keys[srt]

    def find(l, c):
        n_l = nb << l
        c = np.mod(c, n_l[:, None])
        k = key(l, c)
        pos = np.searchsorted(skeys, k)
        pos = np.minimum(pos, len(skeys) - 1)
        hit = skeys[pos] == k
        return np.where(hit, srt[pos], -1)

    Q, F, NQ = [], [], []
    eidx = np.arange(E)
    for d in range(3):
        t1, t2 = [a for a in range(3) if a != d]
        unit = np.zeros(3, dtype=np.int64)
        unit[d] = 1
        # + side: conforming or finer neighbour
        nbc = find(lev, crd + unit)
        conf = nbc >= 0
        q = np.full((conf.sum(), 2, 4), -1, dtype=np.int32)
        q[:, 0, 0], q[:, 1, 0] = eidx[conf], nbc[conf]
        Q.append(q); F.append(np.tile([2 * d + 1, 2 * d], (len(q), 1))); NQ.append(np.tile([1, 1], (len(q), 1)))
        for sign in (1, -1):
            base = 2 * (crd + sign * unit)
            if sign == -1:
                base[:, d] += 1
            kids = []
            for k in range(4):
                off = np.zeros(3, dtype=np.int64)
                off[t1], off[t2] = k & 1, k >> 1
                kids.append(find(lev + 1, base + off))
            kids = np.stack(kids, 1)
            fine = (kids >= 0).all(axis=1) & (lev < max_level)
            if sign == 1:
                fine &= ~conf
            sel = np.nonzero(fine)[0]
            q = np.full((len(sel), 2, 4), -1, dtype=np.int32)
            if sign == 1:   # coarse on the minus half, fine quads see their minus face
                q[:, 0, 0] = sel
                q[:, 1, :] = kids[sel]
                F.append(np.tile([2 * d + 1, 2 * d], (len(sel), 1))); NQ.append(np.tile([1, 4], (len(sel), 1)))
            else:           # fine quads on the minus half, coarse sees its minus face
                q[:, 0, :] = kids[sel]
                q[:, 1, 0] = sel
                F.append(np.tile([2 * d + 1, 2 * d], (len(sel), 1))); NQ.append(np.tile([4, 1], (len(sel), 1)))
            Q.append(q)
    quads, fids, nqs = np.concatenate(Q), np.concatenate(F), np.concatenate(NQ)
    mesh = Mesh(size, cen, quads, fids, nqs, np.zeros(len(quads), dtype=np.int32), level=lev.astype(np.int8))
    mesh.tree = dict(nb=nb, max_level=max_level, lev=lev, crd=crd, lo=lo, hi=hi)
    return mesh


def kh_forest(nb=24, max_level=2, seed=7, band=(0.06, 0.05)):
    """Forest for the Kelvin-Helmholtz layer on [-1,1]^3 (shear interfaces at y = +-0.25): leaves
    whose centre lies within band[level] of the seeded, sinusoidally displaced interface are split --
    the finite-difference |grad rho| of the layer exceeds the threshold there."""
    rng = np.random.default_rng(seed)
    kx, kz = rng.integers(1, 4, size=2)
    ph = rng.uniform(0, 2 * np.pi, size=2)

    def refine(level, c, size):
        shift = 0.02 * np.sin(np.pi * kx * c[:, 0] + ph[0]) * np.sin(np.pi * kz * c[:, 2] + ph[1])
        dist = np.abs(np.abs(c[:, 1] - shift) - 0.25)
        return dist < band[min(level, len(band) - 1)] + 0.5 * size[:, 1]

    return forest(nb, refine, max_level=max_level, lo=(-1.0,) * 3, hi=(1.0,) * 3)


def concat(meshes):
    """Independent meshes side by side in one element list (a batch): element ids of mesh i are
    offset by the element count of the meshes before it.  Returns (mesh, group_of_element) with
    group i = mesh i; each group keeps its own time step and simulation time on the device."""
    off = np.cumsum([0] + [m.E for m in meshes])
    quads = np.concatenate([np.where(m.side_quads >= 0, m.side_quads + off[i], -1) for i, m in enumerate(meshes)])
    mesh = Mesh(np.concatenate([m.delta for m in meshes]), np.concatenate([m.center for m in meshes]), quads,
                np.concatenate([m.side_faceid for m in meshes]), np.concatenate([m.side_nquads for m in meshes]),
                np.concatenate([m.boundary for m in meshes]), level=np.concatenate([m.level for m in meshes]))
    groups = np.concatenate([np.full(m.E, i, dtype=np.int32) for i, m in enumerate(meshes)])
    return mesh, groups


def batched_workload(nb=24, members=256, member_nx=8, seed=11):
    """The batched uneven workload: the Kelvin-Helmholtz forest (group 0) and `members` independent
    periodic member_nx^3 bricks (groups 1..members) in one element list.  Returns (mesh, groups,
    forest, member_mesh, amplitudes) with the Gaussian-blob amplitudes drawn from U[0.1, 1]."""
    f = kh_forest(nb=nb)
    one = brick(member_nx)
    mesh, groups = concat([f] + [one] * members)
    amps = np.random.default_rng(seed).uniform(0.1, 1.0, size=members)
    return mesh, groups, f, one, amps


def adapt(mesh, flags, min_level=0):
    """One adapt step of a forest mesh (made by forest() or adapt()), as mesh_adapt
    (source/mesh/p4est/mesh_utils_mod.f90:879-1010): coarsen, refine, then restore the 2:1 balance.

    flags[E]: +1 refine (below max_level), -1 coarsen (only complete families of 8 sibling leaves above
    min_level that are all flagged), 0 keep.  The new leaf set is 2:1-balanced again (balance may
    refine further, and a coarsening that balance would undo is dropped).  Returns (new mesh, remap) with remap[E_new, 4]
    int32 rows (kind, src, depth, offsets) for nemo_gpu_adapt:
      kind 0: copy of old element src;
      kind 1: refinement of old element src, an ancestor `depth` levels up; offsets = ox | oy << 8 |
              oz << 16 locate the new element inside it (0 <= o < 2^depth);
      kind 2: projection of the 8 old children src .. src + 7 (child c = sx + 2 sy + 4 sz).
    The data movement mirrors kernel_amr_refine / kernel_amr_coarsen
    (source/kernel/dgsem/weakform/2d/kernel_amr_mod.f90:12-73) in 3D.  Unlike the reference's
    one-level walk over old and new quads (:980-1005), a leaf that balance refines by more than one
    level, or a family whose coarsening balance would undo, is handled (deeper interpolation; the
    coarsening is dropped)."""
    t = mesh.tree
    nb, max_level, lo, hi = t["nb"], t["max_level"], t["lo"], t["hi"]
    lev, crd = np.asarray(t["lev"], dtype=np.int64), np.asarray(t["crd"], dtype=np.int64)
    flags = np.asarray(flags)
    K = nb << max_level

    def key(l, c):   # one integer per (level, x, y, z)
        return ((l * K + c[:, 0]) * K + c[:, 1]) * K + c[:, 2]

    def lookup(sorted_keys, order, k):
        """index (in the unsorted list) of each key k, -1 where absent"""
        if len(sorted_keys) == 0:
            return np.full(len(k), -1, dtype=np.int64)
        pos = np.minimum(np.searchsorted(sorted_keys, k), len(sorted_keys) - 1)
        return np.where(sorted_keys[pos] == k, order[pos], -1)

    ko = key(lev, crd)
    o_ord = np.argsort(ko, kind="stable")
    ko_s = ko[o_ord]
    # complete coarsening families (8 leaves of one parent, all flagged, consecutive c = sx + 2sy + 4sz)
    cand = np.nonzero((flags < 0) & (lev > max(int(min_level), 0)))[0]
    pk = key(lev[cand] - 1, crd[cand] >> 1)
    cc = (crd[cand, 0] & 1) | ((crd[cand, 1] & 1) << 1) | ((crd[cand, 2] & 1) << 2)
    srt = np.argsort(pk, kind="stable")
    pk, cand_s, cc = pk[srt], cand[srt], cc[srt]
    starts = np.nonzero(np.r_[True, pk[1:] != pk[:-1]])[0]
    sizes = np.diff(np.r_[starts, len(pk)])
    first = cand_s - cc                          # equal within a family iff indices are first + c
    st8 = starts[sizes == 8]
    same = np.all(first[st8[:, None] + np.arange(8)[None]] == first[st8][:, None], axis=1) if len(st8) else []
    fam_ok = st8[np.asarray(same, dtype=bool)] if len(st8) else np.zeros(0, dtype=np.int64)
    fam_key = pk[fam_ok] if len(fam_ok) else np.zeros(0, dtype=np.int64)
    fam_first = first[fam_ok] if len(fam_ok) else np.zeros(0, dtype=np.int64)
    fam_lev = (lev[cand_s[fam_ok]] - 1) if len(fam_ok) else np.zeros(0, dtype=np.int64)
    fam_crd = (crd[cand_s[fam_ok]] >> 1) if len(fam_ok) else np.zeros((0, 3), dtype=np.int64)
    refine = (flags > 0) & (lev < max_level)
    while True:
        gone = np.zeros(len(lev), dtype=bool)
        for f0 in fam_first:
            gone[f0:f0 + 8] = True
        l_new, c_new = _children(lev[~gone], crd[~gone], refine[~gone])
        l_new = np.concatenate([l_new, fam_lev])
        c_new = np.concatenate([c_new, fam_crd])
        l_bal, c_bal = _balance(nb, max_level, l_new, c_new)
        keep = np.isin(fam_key, key(np.asarray(l_bal, dtype=np.int64), np.asarray(c_bal, dtype=np.int64)))
        if keep.all():
            break
        fam_key, fam_first, fam_lev, fam_crd = fam_key[keep], fam_first[keep], fam_lev[keep], fam_crd[keep]
    new = forest_mesh(nb, max_level, l_bal, c_bal, lo, hi)
    nl, nc = np.asarray(new.tree["lev"], dtype=np.int64), np.asarray(new.tree["crd"], dtype=np.int64)
    kn = key(nl, nc)
    remap = np.zeros((new.E, 4), dtype=np.int64)
    done = np.zeros(new.E, dtype=bool)
    src = lookup(ko_s, o_ord, kn)                # copies
    m0 = src >= 0
    remap[m0, 1] = src[m0]
    done |= m0
    if len(fam_key):                             # coarsened families
        f_ord = np.argsort(fam_key, kind="stable")
        fs = lookup(fam_key[f_ord], f_ord, kn)
        m2 = ~done & (fs >= 0)
        remap[m2, 0] = 2
        remap[m2, 1] = fam_first[fs[m2]]
        remap[m2, 2] = 1
        done |= m2
    for depth in range(1, max_level + 1):       # refinements: the nearest old ancestor
        todo = np.nonzero(~done & (nl >= depth))[0]
        if len(todo) == 0:
            break
        anc = lookup(ko_s, o_ord, key(nl[todo] - depth, nc[todo] >> depth))
        hit = anc >= 0
        e = todo[hit]
        o = nc[e] - ((nc[e] >> depth) << depth)
        remap[e, 0] = 1
        remap[e, 1] = anc[hit]
        remap[e, 2] = depth
        remap[e, 3] = o[:, 0] | (o[:, 1] << 8) | (o[:, 2] << 16)
        done[e] = True
    if not done.all():
        raise RuntimeError(f"new element {int(np.nonzero(~done)[0][0])} has no source in the old forest")
    remap = remap.astype(np.int32)
    return new, remap
