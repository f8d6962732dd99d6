"""A small, dependency-free writer and reader for the subset of the HDF5 file format that the FLASH
checkpoints use: one root group holding contiguous datasets of little-endian integers, IEEE floats,
fixed-length byte strings and compound records of those (numpy structured arrays).

This image has no HDF5 library (neither libhdf5 nor h5py), so the container is written from the
published file-format specification (HDF5 File Format Specification, version 2.0): superblock
version 0 with 8-byte offsets and lengths, version-1 object headers, the root group as a symbol
table (a version-1 B-tree of group nodes over symbol-table nodes, names in a local heap), and per
dataset the dataspace (version 1), datatype (version 1), fill-value (version 2) and data-layout
(version 3, contiguous) messages: structures every HDF5 release reads.  No independent HDF5 reader
is installed here to open the files with; `read` parses exactly this subset back, and the tests
check the round trip byte for byte and the structures' signatures, ordering and addresses.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 4          # symbols per symbol-table node: at most 2 * LEAF_K
NODE_K = 16         # children per group B-tree node: at most 2 * NODE_K
SIG = b"\x89HDF\r\n\x1a\n"


def _pad8(n):
    return (n + 7) & ~7


# ---- datatype messages -------------------------------------------------------------------------

def _datatype(dt):
    """Encoded datatype message (version 1) for a numpy dtype."""
    dt = np.dtype(dt)
    if dt.fields is not None:
        body = b""
        for name in dt.names:
            sub, off = dt.fields[name][0], dt.fields[name][1]
            nm = name.encode() + b"\0"
            body += nm + b"\0" * (_pad8(len(nm)) - len(nm))
            body += struct.pack("<IB3xI4x4I", off, 0, 0, 0, 0, 0, 0)
            body += _datatype(sub)
        return struct.pack("<B3sI", (1 << 4) | 6, len(dt.names).to_bytes(3, "little"), dt.itemsize) + body
    if dt.kind in "iu":
        if dt.byteorder == ">":
            raise ValueError("big-endian integers are not written")
        bits = 0x08 if dt.kind == "i" else 0
        return struct.pack("<B3sIHH", (1 << 4) | 0, bits.to_bytes(3, "little"), dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "f":
        if dt.byteorder == ">":
            raise ValueError("big-endian floats are not written")
        if dt.itemsize == 8:
            sign, eloc, esz, mloc, msz, bias = 63, 52, 11, 0, 52, 1023
        elif dt.itemsize == 4:
            sign, eloc, esz, mloc, msz, bias = 31, 23, 8, 0, 23, 127
        else:
            raise ValueError(f"unsupported float size {dt.itemsize}")
        bits = (2 << 4) | (sign << 8)          # little endian, implied leading mantissa bit, sign bit
        return struct.pack("<B3sIHHBBBBI", (1 << 4) | 1, bits.to_bytes(3, "little"), dt.itemsize, 0,
                           8 * dt.itemsize, eloc, esz, mloc, msz, bias)
    if dt.kind == "S":
        return struct.pack("<B3sI", (1 << 4) | 3, (1).to_bytes(3, "little"), dt.itemsize)   # null padded, ASCII
    raise ValueError(f"unsupported dtype {dt}")


def _parse_datatype(buf, pos):
    """(numpy dtype, position after the message) for an encoded datatype."""
    cv, bits, size = struct.unpack_from("<B3sI", buf, pos)
    cls, bits = cv & 0x0F, int.from_bytes(bits, "little")
    p = pos + 8
    if cls == 0:
        return np.dtype(("<i" if bits & 0x08 else "<u") + str(size)), p + 4
    if cls == 1:
        return np.dtype("<f" + str(size)), p + 12
    if cls == 3:
        return np.dtype("S" + str(size)), p
    if cls == 6:
        names, formats, offsets = [], [], []
        for _ in range(bits & 0xFFFF):
            end = buf.index(b"\0", p)
            names.append(buf[p:end].decode())
            p += _pad8(end - p + 1)
            off = struct.unpack_from("<I", buf, p)[0]
            p += 32                              # offset, rank, permutation, four dimension sizes
            sub, p = _parse_datatype(buf, p)
            formats.append(sub)
            offsets.append(off)
        return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size}), p
    raise ValueError(f"datatype class {cls} is not part of this subset")


# ---- object headers ----------------------------------------------------------------------------

def _message(mtype, body, flags=0):
    body = body + b"\0" * (_pad8(len(body)) - len(body))
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _object_header(messages):
    data = b"".join(messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(data)) + data


def _dataset_header(arr, data_addr):
    shape = arr.shape
    space = struct.pack("<BBBx4x", 1, len(shape), 0) + b"".join(struct.pack("<Q", n) for n in shape)
    fill = struct.pack("<BBBB", 2, 2, 2, 0)     # late allocation, write if set, no fill value defined
    layout = struct.pack("<BBQQ", 3, 1, data_addr, arr.nbytes)
    return _object_header([_message(0x0001, space), _message(0x0003, _datatype(arr.dtype), 1),
                           _message(0x0005, fill, 1), _message(0x0008, layout)])


# ---- file ---------------------------------------------------------------------------------------

def write(path, datasets):
    """Write {name: numpy array} as the root group's datasets of an HDF5 file."""
    names = sorted(datasets)                     # the symbol-table nodes keep their names sorted
    if len(names) > 2 * LEAF_K * 2 * NODE_K:
        raise ValueError("too many datasets for one group B-tree node")
    arrays = {}
    for n in names:
        a = np.ascontiguousarray(datasets[n])
        if a.ndim == 0:
            a = a.reshape(1)
        arrays[n] = a

    # local heap of the names: offset 0 is the empty string
    heap = bytearray(b"\0" * 8)
    name_off = {}
    for n in names:
        name_off[n] = len(heap)
        b = n.encode() + b"\0"
        heap += b + b"\0" * (_pad8(len(b)) - len(b))
    heap_data = bytes(heap)

    # fixed-size structures first, then the object headers and the data
    pos = 96                                     # superblock with the root symbol-table entry
    root_oh = pos
    root_oh_size = len(_object_header([_message(0x0011, b"\0" * 16)]))
    pos += _pad8(root_oh_size)
    heap_hdr = pos
    pos += 32
    heap_seg = pos
    pos += len(heap_data)
    btree = pos
    pos += 24 + (2 * NODE_K + 1) * 8 + 2 * NODE_K * 8
    groups = [names[i:i + 2 * LEAF_K] for i in range(0, len(names), 2 * LEAF_K)]
    snod_addr = []
    for _ in groups:
        snod_addr.append(pos)
        pos += 8 + 2 * LEAF_K * 40
    oh_addr, data_addr = {}, {}
    for n in names:
        oh_addr[n] = pos
        pos += _pad8(len(_dataset_header(arrays[n], 0)))
        data_addr[n] = pos
        pos += _pad8(arrays[n].nbytes)
    eof = pos

    head = bytearray(oh_addr[names[0]] if names else eof)
    root_entry = struct.pack("<QQI4xQQ", 0, root_oh, 1, btree, heap_hdr)
    head[0:96] = SIG + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, LEAF_K, NODE_K, 0) + \
        struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF) + root_entry
    roh = _object_header([_message(0x0011, struct.pack("<QQ", btree, heap_hdr))])
    head[root_oh:root_oh + len(roh)] = roh
    # free-list head: no free block is recorded as offset 1, which no 8-aligned block can have
    head[heap_hdr:heap_hdr + 32] = b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap_data), 1, heap_seg)
    head[heap_seg:heap_seg + len(heap_data)] = heap_data
    node = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(groups), UNDEF, UNDEF)
    node += struct.pack("<Q", 0)
    for g, a in zip(groups, snod_addr):
        node += struct.pack("<QQ", a, name_off[g[-1]])
    head[btree:btree + len(node)] = node
    for g, a in zip(groups, snod_addr):
        sn = b"SNOD" + struct.pack("<BxH", 1, len(g))
        for n in g:
            sn += struct.pack("<QQI4x16x", name_off[n], oh_addr[n], 0)
        head[a:a + len(sn)] = sn
    # then, in file order, each dataset's object header and its data (streamed, no whole-file copy)
    with open(path, "wb") as f:
        f.write(head)
        for n in names:
            h = _dataset_header(arrays[n], data_addr[n])
            f.write(h + b"\0" * (data_addr[n] - oh_addr[n] - len(h)))
            f.write(memoryview(arrays[n]).cast("B"))
            f.write(b"\0" * (_pad8(arrays[n].nbytes) - arrays[n].nbytes))
        if f.tell() != eof:
            raise RuntimeError("HDF5 layout mismatch")


def read(path):
    """{name: numpy array} of the root group's datasets of a file in this subset."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != SIG or buf[8] != 0:
        raise ValueError(f"{path}: not an HDF5 file with a version-0 superblock")
    leaf_k, node_k = struct.unpack_from("<HH", buf, 16)
    eof = struct.unpack_from("<Q", buf, 40)[0]
    if eof != len(buf):
        raise ValueError(f"{path}: end-of-file address {eof} differs from the file size {len(buf)}")
    btree, heap_hdr = struct.unpack_from("<QQ", buf, 56 + 24)
    if buf[heap_hdr:heap_hdr + 4] != b"HEAP":
        raise ValueError("local heap signature missing")
    heap_size, _, heap_seg = struct.unpack_from("<QQQ", buf, heap_hdr + 8)
    heap = buf[heap_seg:heap_seg + heap_size]
    if buf[btree:btree + 4] != b"TREE":
        raise ValueError("group B-tree signature missing")
    ntype, level, used = struct.unpack_from("<BBH", buf, btree + 4)
    if ntype != 0 or level != 0:
        raise ValueError("only a single-level group B-tree is read")
    out = {}
    for i in range(used):
        child = struct.unpack_from("<Q", buf, btree + 24 + 8 + 16 * i)[0]
        if buf[child:child + 4] != b"SNOD":
            raise ValueError("symbol-table node signature missing")
        nsym = struct.unpack_from("<H", buf, child + 6)[0]
        for j in range(nsym):
            noff, oh = struct.unpack_from("<QQ", buf, child + 8 + 40 * j)
            name = heap[noff:heap.index(b"\0", noff)].decode()
            out[name] = _read_dataset(buf, oh)
    return out


def _read_dataset(buf, oh):
    version, _, nmsg, _, size = struct.unpack_from("<BBHII", buf, oh)
    if version != 1:
        raise ValueError("only version-1 object headers are read")
    p, end = oh + 16, oh + 16 + size
    shape = dtype = addr = nbytes = None
    for _ in range(nmsg):
        mtype, msize = struct.unpack_from("<HH", buf, p)
        body = p + 8
        if mtype == 0x0001:
            rank = buf[body + 1]
            shape = struct.unpack_from("<" + "Q" * rank, buf, body + 8)
        elif mtype == 0x0003:
            dtype, _ = _parse_datatype(buf, body)
        elif mtype == 0x0008:
            ver, cls, addr, nbytes = struct.unpack_from("<BBQQ", buf, body)
            if ver != 3 or cls != 1:
                raise ValueError("only contiguous data layouts are read")
        p = body + msize
        if p > end:
            raise ValueError("object header messages overrun the header")
    arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape)), offset=addr).reshape(shape)
    if arr.nbytes != nbytes:
        raise ValueError("data size differs from the layout message")
    return arr.copy()
