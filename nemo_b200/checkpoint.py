"""FLASH-layout checkpoints of a run, written from an asynchronous device->host snapshot, and the
restart that reads them back.

The reference writes FLASH 4 checkpoint files (source/checkpoint/flash/checkpoint_mod.f90:11-364,
source/checkpoint/flash/checkpoint_utils_mod.f90): the tree of blocks -- every ancestor of a leaf,
level by level, then all leaves (mesh_alloc_tree, source/mesh/p4est/mesh_utils_mod.f90:490-580) --
with "coordinates", "block size", "bounding box", "gid" (6 face neighbours, parent, 8 children;
1-based, -1 for none), "node type" (1 leaf, 2 parent), "refine level" (level + 1), "which child",
"bflags"; one dataset per variable ("dens", "momx", "momy", "momz", "ener", plus "blnd") shaped
[block][z][y][x]; the "unknown names"; integer/real/logical/string scalars and runtime parameters
as (name, value) records of 80-character names; and "sim info".  The leaves' data goes to the last
nleaves blocks (checkpoint_utils_dataset_iterate, :134-203).  Here the parent blocks hold the L2
projection of their children (the reference leaves them unwritten); "blnd" holds the element's
blending coefficient at every node (the reference writes a per-node blend of its FV levels).

Container: an HDF5 file named like the reference's (`<prefix><count:06d>.f5`), written as `.partial`
and renamed, as the reference does.  This image has no HDF5 library (neither libhdf5 nor h5py), so
`h5lite` writes the original-format HDF5 structures these datasets need (one root group of contiguous
datasets, compound records for the scalar lists) from the file-format specification.  A path ending
in `.npz` selects an uncompressed numpy archive of the same datasets instead.  Restart is the part the reference leaves as a TODO
(source/nemo_prog.f90:107-114): `read` rebuilds the forest from the leaves' levels and coordinates,
and `restart` uploads the state and restores the time and step counter.
"""
import ctypes
import os

import numpy as np

from . import abi, h5lite
from .mesh import forest_mesh

FILE_FORMAT_VERSION = 9
EULER_NAMES = ["dens", "momx", "momy", "momz", "ener"]
MHD_NAMES = EULER_NAMES + ["magx", "magy", "magz", "glmp"]


def _records(items, vtype):
    """(name, value) records as FLASH stores its scalar and runtime-parameter lists."""
    dt = np.dtype([("name", "S80"), ("value", vtype)])
    return np.array([(k.encode(), v) for k, v in items], dtype=dt)


def _tree(mesh):
    """(nb, max_level, lev, crd, lo, hi) of a forest mesh, or of a cubic periodic brick."""
    t = getattr(mesh, "tree", None)
    if t is not None:
        return t["nb"], t["max_level"], np.asarray(t["lev"]), np.asarray(t["crd"]), t["lo"], t["hi"]
    d = mesh.delta
    if not np.allclose(d, d[0]) or not np.allclose(d[0], d[0, 0]):
        raise ValueError("checkpoints need a forest mesh (mesh.forest / mesh.adapt) or a cubic brick")
    lo = mesh.center.min(axis=0) - 0.5 * d[0]
    hi = mesh.center.max(axis=0) + 0.5 * d[0]
    nb = int(round((hi[0] - lo[0]) / d[0, 0]))
    crd = np.rint((mesh.center - lo) / d[0] - 0.5).astype(np.int64)
    return nb, 0, np.zeros(mesh.E, dtype=np.int64), crd, lo, hi


def block_tree(mesh):
    """The FLASH block list of a mesh: dict of levels, integer coordinates, parent/children (0-based,
    -1 for none), the index of each leaf's block, and the domain."""
    nb, max_level, lev, crd, lo, hi = _tree(mesh)
    leaves = [(int(l), int(c[0]), int(c[1]), int(c[2])) for l, c in zip(lev, crd)]
    inner = set()
    for l, x, y, z in leaves:
        for d in range(1, l + 1):
            inner.add((l - d, x >> d, y >> d, z >> d))

    def morton_key(b):
        l, x, y, z = b
        s = max_level - l   # anchor on the finest grid
        key = 0
        for bit in range(20):
            key |= (((x << s) >> bit) & 1) << (3 * bit) | (((y << s) >> bit) & 1) << (3 * bit + 1) | \
                   (((z << s) >> bit) & 1) << (3 * bit + 2)
        return key

    inner = sorted(inner, key=lambda b: (b[0], morton_key(b)))
    blocks = inner + leaves
    index = {b: i for i, b in enumerate(inner)}
    nblocks, nin = len(blocks), len(inner)
    parent = np.full(nblocks, -1, dtype=np.int64)
    children = np.full((nblocks, 8), -1, dtype=np.int64)
    which = np.full(nblocks, -1, dtype=np.int64)
    for i, (l, x, y, z) in enumerate(blocks):
        if l == 0:
            continue
        p = index[(l - 1, x >> 1, y >> 1, z >> 1)]
        c = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2)
        parent[i] = p
        children[p, c] = i
        which[i] = c
    b = np.asarray(blocks, dtype=np.int64)
    return dict(nb=nb, max_level=max_level, lo=np.asarray(lo, float), hi=np.asarray(hi, float),
                level=b[:, 0], crd=b[:, 1:], parent=parent, children=children, which=which, n_inner=nin,
                nblocks=nblocks)


def _restrict(tree, leaf_data):
    """Block data [nblocks, V, 64]: the leaves' data, and for every parent the sum of its children's
    L2 projections (the 2:1 mortar projection matrices in tensor product), finest level first."""
    V = leaf_data.shape[0]
    nb, nin = tree["nblocks"], tree["n_inner"]
    out = np.zeros((nb, V, 4, 4, 4))
    out[nin:] = leaf_data.transpose(1, 0, 2).reshape(-1, V, 4, 4, 4)
    _, prj = abi.mortar_operators()
    lev_in = tree["level"][:nin]
    for lv in sorted(set(lev_in.tolist()), reverse=True):   # children (one level finer) are done
        par = np.nonzero(lev_in == lv)[0]
        acc = np.zeros((len(par), V, 4, 4, 4))
        for c in range(8):
            px, py, pz = prj[c & 1], prj[(c >> 1) & 1], prj[c >> 2]
            acc += np.einsum("ai,bj,ck,nvkji->nvcba", px, py, pz, out[tree["children"][par, c]], optimize=True)
        out[par] = acc
    return out


def datasets(mesh, u, t, steps, cfg, dt=0.0, alpha=None, number=0, basename="chkpt_"):
    """The FLASH checkpoint datasets of state u [V, E, 64] on mesh at time t after `steps` steps."""
    tree = block_tree(mesh)
    V = u.shape[0]
    names = MHD_NAMES if V == 9 else EULER_NAMES
    nbk, nin = tree["nblocks"], tree["n_inner"]
    lo, hi = tree["lo"], tree["hi"]
    size = (hi - lo)[None, :] / (tree["nb"] << tree["level"])[:, None].astype(float)
    coords = lo[None, :] + (tree["crd"] + 0.5) * size
    bbox = np.stack([coords - 0.5 * size, coords + 0.5 * size], axis=2)          # [block][dim][lo,hi]
    gid = np.full((nbk, 15), -1, dtype=np.int32)
    gid[:, 6] = np.where(tree["parent"] >= 0, tree["parent"] + 1, -1)
    gid[:, 7:] = np.where(tree["children"] >= 0, tree["children"] + 1, -1)
    node_type = np.where(np.arange(nbk) < nin, 2, 1).astype(np.int32)
    which = np.where(tree["which"] >= 0, tree["which"] + 1, -1).astype(np.int32)
    blocks = _restrict(tree, np.asarray(u, dtype=np.float64))
    ds = {
        "coordinates": coords, "block size": size, "bounding box": bbox,
        "gid": gid, "node type": node_type, "refine level": (tree["level"] + 1).astype(np.int32),
        "which child": which, "bflags": np.full(nbk, -1, dtype=np.int32),
        "unknown names": np.array([[n.encode()] for n in names + ["blnd"]], dtype="S4"),
    }
    for v, n in enumerate(names):
        ds[n] = np.ascontiguousarray(blocks[:, v])
    blnd = np.zeros((nbk, 4, 4, 4))
    if alpha is not None:
        blnd[nin:] = np.asarray(alpha, dtype=np.float64)[:, None, None, None]
    ds["blnd"] = blnd
    ds["integer scalars"] = _records([
        ("nstep", int(steps)), ("nxb", 4), ("nyb", 4), ("nzb", 4), ("dimensionality", 3),
        ("globalnumblocks", nbk), ("checkpointfilenumber", int(number))], "<i4")
    ds["real scalars"] = _records([
        ("time", t), ("dt", dt), ("dtold", dt), ("dtnew", dt), ("nextcheckpointtime", 0.0)], "<f8")
    ds["logical scalars"] = _records([("doubleprecision", 1)], "<i4")
    ds["string scalars"] = _records([("geometry", b"cartesian"), ("nemo", b"nemo_b200")], "S80")
    ds["integer runtime parameters"] = _records([
        ("lrefine_min", 1), ("lrefine_max", tree["max_level"] + 1), ("checkpointfilenumber", int(number)),
        ("checkpointfileintervalstep", 0), ("fileformatversion", FILE_FORMAT_VERSION),
        ("forcedplotfilenumber", 0), ("nblockx", tree["nb"]), ("nblocky", tree["nb"]), ("nblockz", tree["nb"])],
        "<i4")
    ds["real runtime parameters"] = _records([
        ("xmin", lo[0]), ("xmax", hi[0]), ("ymin", lo[1]), ("ymax", hi[1]), ("zmin", lo[2]), ("zmax", hi[2]),
        ("cfl", float(cfg.cfl)), ("checkpointfileintervaltime", 0.0), ("tinitial", 0.0), ("tmax", 0.0),
        ("gamma", float(cfg.kappa))], "<f8")
    ds["logical runtime parameters"] = _records([("restart", 0)], "<i4")
    ds["string runtime parameters"] = _records(
        [("unitsystem", b"none"), ("geometry", b"cartesian"), ("basen", basename.encode())] +
        [(f"{a}{s}_boundary_type", b"periodic") for a in "xyz" for s in "lr"], "S80")
    info = np.dtype([("file format version", "<i4"), ("setup call", "S400"), ("file creation time", "S80"),
                     ("flash version", "S80"), ("build date", "S80"), ("build dir", "S80"),
                     ("build machine", "S80"), ("cflags", "S400"), ("fflags", "S400"),
                     ("setup time stamp", "S80"), ("build time stamp", "S80")])
    ds["sim info"] = np.array([(FILE_FORMAT_VERSION, b"none", b"none", b"FLASH 4.3_release", b"none",
                                b"none", b"none", b"none", b"none", b"none", b"none")], dtype=info)
    return ds


def write(path, ds):
    """Write the datasets to path through a '.partial' file and a rename: an HDF5 file, or a numpy
    archive if the path ends in '.npz'."""
    tmp = path + ".partial"
    if path.endswith(".npz"):
        with open(tmp, "wb") as f:
            np.savez(f, **ds)
    else:
        h5lite.write(tmp, ds)
    os.replace(tmp, path)


def load_datasets(path):
    """{name: array} of a checkpoint file, HDF5 (recognised by its signature) or numpy archive."""
    with open(path, "rb") as f:
        magic = f.read(8)
    if magic == h5lite.SIG:
        return h5lite.read(path)
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def to_hdf5(npz_path, h5_path):
    """Copy a checkpoint archive (.npz) into an HDF5 file."""
    write(h5_path, load_datasets(npz_path))


def read(path):
    """(mesh, u [V, E, 64], t, steps) from a checkpoint file; the mesh is the forest of its leaves."""
    z = load_datasets(path)
    ip = {r["name"].decode(): int(r["value"]) for r in z["integer runtime parameters"]}
    rp = {r["name"].decode(): float(r["value"]) for r in z["real runtime parameters"]}
    iscal = {r["name"].decode(): int(r["value"]) for r in z["integer scalars"]}
    rscal = {r["name"].decode(): float(r["value"]) for r in z["real scalars"]}
    names = [n[0].decode() for n in z["unknown names"] if n[0].decode() != "blnd"]
    leaf = z["node type"] == 1
    lev = z["refine level"][leaf].astype(np.int64) - 1
    lo = np.array([rp["xmin"], rp["ymin"], rp["zmin"]])
    hi = np.array([rp["xmax"], rp["ymax"], rp["zmax"]])
    nb, max_level = ip["nblockx"], ip["lrefine_max"] - 1
    size = z["block size"][leaf]
    crd = np.rint((z["coordinates"][leaf] - lo) / size - 0.5).astype(np.int64)
    u = np.stack([z[n][leaf].reshape(-1, 64) for n in names])
    mesh = forest_mesh(nb, max_level, lev, crd, lo, hi)
    # forest_mesh orders the leaves by Morton order; the file holds them in that order already
    order = np.lexsort((crd[:, 2], crd[:, 1], crd[:, 0], lev))
    morder = np.lexsort((mesh.tree["crd"][:, 2], mesh.tree["crd"][:, 1], mesh.tree["crd"][:, 0],
                         mesh.tree["lev"]))
    perm = np.empty(len(lev), dtype=np.int64)
    perm[morder] = order
    return mesh, np.ascontiguousarray(u[:, perm]), rscal["time"], iscal["nstep"]


class Checkpointer:
    """Asynchronous checkpoints of a Solver: `begin()` snapshots the state and the last stage's
    blending coefficients in stream order and starts their copy into page-locked buffers;
    `finish(path)` waits for it and writes the file.  Steps issued in between overlap the copy."""

    def __init__(self, solver, basename="chkpt_", directory="checkpoints"):
        self.s = solver
        self.basename, self.directory = basename, directory
        self.count = 0
        self.buf = self.abuf = None

    def _buffers(self):
        import torch
        s = self.s
        n = s.V * s.E * s.n ** 3
        if self.buf is None or self.buf.numel() != n:      # first call, or the mesh changed (adapt)
            pin = torch.cuda.is_available()
            self.buf = torch.empty(n, dtype=torch.float64, pin_memory=pin)
            self.abuf = torch.empty(s.E, dtype=torch.float64, pin_memory=pin)

    def begin(self):
        self._buffers()
        s = self.s
        abi.call("nemo_gpu_checkpoint_begin", ctypes.c_void_p(self.buf.data_ptr()), s.V * s.n ** 3 * 8,
                 ctypes.c_void_p(self.abuf.data_ptr()))

    def finish(self, path=None):
        t, st = ctypes.c_double(), ctypes.c_int64()
        abi.call("nemo_gpu_checkpoint_wait", ctypes.byref(t), ctypes.byref(st))
        s = self.s
        u = self.buf.numpy().reshape(s.E, s.V, s.n ** 3).transpose(1, 0, 2)
        if path is None:
            os.makedirs(self.directory, exist_ok=True)
            path = os.path.join(self.directory, f"{self.basename}{self.count:06d}.f5")
        write(path, datasets(s.mesh, u, t.value, st.value, s.cfg, alpha=self.abuf.numpy().copy(),
                             number=self.count, basename=self.basename))
        self.count += 1
        return path, t.value, st.value


def restart(cfg, path):
    """A Solver on the checkpoint's forest, its state uploaded and its time and step count restored."""
    from .solver import Solver
    mesh, u, t, steps = read(path)
    s = Solver(cfg, mesh)
    s.upload(u)
    abi.call("nemo_gpu_set_time", float(t), int(steps))
    return s
