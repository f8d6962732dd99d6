"""FLASH-layout checkpoints (CPU): the block tree (ancestors level by level, then the leaves), the
datasets' names, shapes and records, the parents' restriction, and write -> read round trips of a
forest and of a brick (mesh, state, time and step count)."""
import numpy as np

from nemo_b200 import abi, checkpoint, mesh, setups
from oracle import oracle as orc


def band_forest():
    return mesh.forest(4, lambda lvl, c, s: np.abs(c[:, 1] - 0.5) < 0.2 / (1 + lvl), max_level=2)


def test_block_tree():
    m = band_forest()
    t = checkpoint.block_tree(m)
    nin, nb = t["n_inner"], t["nblocks"]
    assert nb == nin + m.E
    assert np.array_equal(t["level"][nin:], m.tree["lev"])            # leaves last, in mesh order
    assert np.all(np.diff(t["level"][:nin]) >= 0)                     # ancestors level by level
    for i in range(nb):
        p = t["parent"][i]
        if t["level"][i] == 0:
            assert p == -1 and t["which"][i] == -1
        else:
            assert t["children"][p, t["which"][i]] == i
            assert np.array_equal(t["crd"][p], t["crd"][i] >> 1)
    assert np.all(t["children"][:nin] >= 0) and np.all(t["children"][nin:] == -1)


def test_datasets_and_restriction():
    m = band_forest()
    x, y, z = m.node_coords(orc.lgl(3)[0])
    u = np.stack([1.0 + x + y * y, 0.5 * x * z, y, z, 3.0 + x * y]).copy()   # degree <= 2
    c = abi.default_cfg()
    ds = checkpoint.datasets(m, u, 0.25, 17, c, alpha=np.linspace(0, 0.5, m.E))
    t = checkpoint.block_tree(m)
    nb, nin = t["nblocks"], t["n_inner"]
    assert ds["dens"].shape == (nb, 4, 4, 4) and ds["gid"].shape == (nb, 15)
    assert ds["bounding box"].shape == (nb, 3, 2) and ds["unknown names"].shape == (6, 1)
    assert [n[0] for n in ds["unknown names"]] == [b"dens", b"momx", b"momy", b"momz", b"ener", b"blnd"]
    assert np.array_equal(ds["node type"], np.r_[np.full(nin, 2), np.ones(m.E)])
    iscal = {r["name"]: r["value"] for r in ds["integer scalars"]}
    assert iscal[b"nstep"] == 17 and iscal[b"globalnumblocks"] == nb
    assert {r["name"]: r["value"] for r in ds["real scalars"]}[b"time"] == 0.25
    np.testing.assert_array_equal(ds["dens"][nin:].reshape(m.E, 64), u[0])
    # parents: the projection reproduces the quadratic at the parent's own nodes
    xn = orc.lgl(3)[0]
    for i in range(nin):
        cen, size = ds["coordinates"][i], ds["block size"][i]
        X = cen[0] + 0.5 * size[0] * xn[None, None, :]
        Y = cen[1] + 0.5 * size[1] * xn[None, :, None]
        np.testing.assert_allclose(ds["dens"][i], np.broadcast_to(1.0 + X + Y * Y, (4, 4, 4)), atol=1e-12)
    np.testing.assert_array_equal(ds["blnd"][nin:, 0, 0, 0], np.linspace(0, 0.5, m.E))


def _round_trip(m, tmp_path, name="chkpt_000000.f5"):
    u = setups.smooth_random(m, seed=9)
    path = str(tmp_path / name)
    checkpoint.write(path, checkpoint.datasets(m, u, 0.125, 40, abi.default_cfg()))
    m2, u2, t, steps = checkpoint.read(path)
    assert t == 0.125 and steps == 40 and m2.E == m.E
    np.testing.assert_array_equal(m2.delta, m.delta)
    np.testing.assert_array_equal(m2.center, m.center)
    np.testing.assert_array_equal(m2.neighbors(), m.neighbors())
    np.testing.assert_array_equal(u2, u)


def test_round_trip_forest(tmp_path):
    _round_trip(band_forest(), tmp_path)


def test_round_trip_adapted_forest(tmp_path):
    m = band_forest()
    f = np.where(m.center[:, 0] < 0.3, 1, np.where(m.center[:, 0] > 0.6, -1, 0))
    _round_trip(mesh.adapt(m, f)[0], tmp_path)


def test_round_trip_brick(tmp_path):
    _round_trip(mesh.brick(4), tmp_path)


def test_round_trip_numpy_archive(tmp_path):
    _round_trip(band_forest(), tmp_path, "chkpt_000000.f5.npz")


def test_hdf5_container_holds_every_dataset_unchanged(tmp_path):
    """The HDF5 file (the reference's container) holds every FLASH dataset with its dtype, shape and
    bytes -- the compound scalar and parameter records included -- and its structures are the
    format's: the signature, a version-0 superblock whose end-of-file address is the file size,
    the root group's B-tree, local heap and symbol-table nodes with the names in byte order."""
    import struct
    from nemo_b200 import h5lite
    m = band_forest()
    ds = checkpoint.datasets(m, setups.smooth_random(m, seed=3), 0.25, 12, abi.default_cfg(),
                             alpha=np.linspace(0.0, 0.5, m.E))
    path = str(tmp_path / "chkpt_000001.f5")
    checkpoint.write(path, ds)
    raw = open(path, "rb").read()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n" and raw[8] == 0
    assert struct.unpack_from("<Q", raw, 40)[0] == len(raw)
    btree, heap = struct.unpack_from("<QQ", raw, 80)
    assert raw[btree:btree + 4] == b"TREE" and raw[heap:heap + 4] == b"HEAP"
    back = h5lite.read(path)
    assert sorted(back) == sorted(ds)
    for k, v in ds.items():
        v = np.asarray(v)
        assert back[k].dtype == v.dtype and back[k].shape == v.shape and back[k].tobytes() == v.tobytes(), k
    # the symbol-table nodes list the names in strcmp order
    names, nsnod = [], struct.unpack_from("<H", raw, btree + 6)[0]
    for i in range(nsnod):
        child = struct.unpack_from("<Q", raw, btree + 32 + 16 * i)[0]
        assert raw[child:child + 4] == b"SNOD"
        seg = struct.unpack_from("<Q", raw, heap + 24)[0]
        for j in range(struct.unpack_from("<H", raw, child + 6)[0]):
            off = struct.unpack_from("<Q", raw, child + 8 + 40 * j)[0]
            names.append(raw[seg + off:raw.index(b"\0", seg + off)])
    assert names == sorted(names) and len(names) == len(ds)


def test_numpy_archive_converts_to_hdf5(tmp_path):
    m = mesh.brick(4)
    ds = checkpoint.datasets(m, setups.smooth_random(m, seed=5), 0.5, 3, abi.default_cfg())
    a, b = str(tmp_path / "c.f5.npz"), str(tmp_path / "c.f5")
    checkpoint.write(a, ds)
    checkpoint.to_hdf5(a, b)
    r1, r2 = checkpoint.read(a), checkpoint.read(b)
    assert np.array_equal(r1[1], r2[1]) and r1[2:] == r2[2:]


def test_round_trip_mhd(tmp_path):
    """GLM-MHD state: the 9 FLASH variable names and a lossless round trip."""
    m = band_forest()
    u = setups.orszag_tang(m)
    c = abi.default_cfg(eqn=abi.EQN_MHD, n_vars=9, kappa=5 / 3)
    path = str(tmp_path / "mhd.f5")
    checkpoint.write(path, checkpoint.datasets(m, u, 0.5, 7, c))
    z = checkpoint.load_datasets(path)
    assert [n[0] for n in z["unknown names"]] == [n.encode() for n in checkpoint.MHD_NAMES] + [b"blnd"]
    g = {r["name"]: r["value"] for r in z["real runtime parameters"]}
    assert abs(g[b"gamma"] - 5 / 3) < 1e-15
    m2, u2, t, steps = checkpoint.read(path)
    assert u2.shape == u.shape and np.array_equal(u2, u) and t == 0.5 and steps == 7
