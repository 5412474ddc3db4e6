"""The HDF5 reader on the file forms that libhdf5 and h5py write besides the
earliest one: superblock versions 2 and 3 with version-2 object headers
and compact links, version-2 and -3 attribute messages, and chunked
datasets indexed by a version-1 B-tree (layout version 3) or by the
single-chunk, implicit and fixed-array indexes of layout version 4.

The files are assembled here byte by byte from the HDF5 file format
specification (version 3.0): no libhdf5 or h5py is involved.  Checksums
are Bob Jenkins' lookup3 hashlittle, as the specification prescribes
(the reader does not verify them).  The expected arrays are numpy's; chunk
shapes that do not divide the dataset test the clipping at its edges, and
chunks placed out of order in the file test that the index is followed.
"""
import struct

import numpy as np
import pytest

from raptr_b200 import h5

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"
M32 = 0xFFFFFFFF


# ---------------------------------------------------------------- lookup3

def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & M32


def lookup3(data: bytes, initval: int = 0) -> int:
    """hashlittle() of lookup3.c (Bob Jenkins, public domain)."""
    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M32
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & M32
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & M32
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & M32
        a = (a - c) & M32; a ^= _rot(c, 4); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 6); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 8); b = (b + a) & M32
        a = (a - c) & M32; a ^= _rot(c, 16); c = (c + b) & M32
        b = (b - a) & M32; b ^= _rot(a, 19); a = (a + c) & M32
        c = (c - b) & M32; c ^= _rot(b, 4); b = (b + a) & M32
        n -= 12
        i += 12
    if n == 0:
        return c
    tail = data[i:] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M32
    b = (b + int.from_bytes(tail[4:8], "little")) & M32
    c = (c + int.from_bytes(tail[8:12], "little")) & M32
    c ^= b; c = (c - _rot(b, 14)) & M32
    a ^= c; a = (a - _rot(c, 11)) & M32
    b ^= a; b = (b - _rot(a, 25)) & M32
    c ^= b; c = (c - _rot(b, 16)) & M32
    a ^= c; a = (a - _rot(c, 4)) & M32
    b ^= a; b = (b - _rot(a, 14)) & M32
    c ^= b; c = (c - _rot(b, 24)) & M32
    return c


def test_lookup3_known_values():
    # the self-test values printed by lookup3.c's driver
    assert lookup3(b"") == 0xDEADBEEF
    assert lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert lookup3(b"Four score and seven years ago", 0) == 0x17770551
    assert lookup3(b"Four score and seven years ago", 1) == 0xCD628161


# ---------------------------------------------------------------- builder

class Img:
    """A file image with an append allocator (8-byte aligned objects)."""

    def __init__(self):
        self.b = bytearray()

    def add(self, data: bytes) -> int:
        while len(self.b) % 8:
            self.b.append(0)
        at = len(self.b)
        self.b += data
        return at

    def reserve(self, n: int) -> int:
        return self.add(bytes(n))

    def put(self, at: int, data: bytes):
        self.b[at:at + len(data)] = data


def u8(v): return struct.pack("<B", v)
def u16(v): return struct.pack("<H", v)
def u32(v): return struct.pack("<I", v)
def u64(v): return struct.pack("<Q", v)


def dtype_msg(np_dtype) -> bytes:
    dt = np.dtype(np_dtype)
    if dt == np.float32 or dt == np.float64:
        bits = 32 if dt == np.float32 else 64
        epos, esize, msize, bias = (23, 8, 23, 127) if bits == 32 else (52, 11, 52, 1023)
        return (u8(0x11) + bytes([0x20, bits - 1, 0]) + u32(dt.itemsize) + u16(0) + u16(bits) + u8(epos)
                + u8(esize) + u8(0) + u8(msize) + u32(bias))
    assert dt == np.int32
    return u8(0x10) + bytes([0x08, 0, 0]) + u32(4) + u16(0) + u16(32)


def dataspace_v2(dims) -> bytes:
    return u8(2) + u8(len(dims)) + u8(0) + u8(1 if dims else 0) + b"".join(u64(d) for d in dims)


def ohdr_v2(msgs) -> bytes:
    """Version-2 object header with a 4-byte chunk-size field (flags 2):
    messages as (type, body)."""
    body = b"".join(u8(t) + u16(len(d)) + u8(0) + d for t, d in msgs)
    head = b"OHDR" + u8(2) + u8(2) + u32(len(body))
    h = head + body
    return h + u32(lookup3(h))


def ohdr_v1(msgs) -> bytes:
    """Version-1 object header: messages as (type, body), bodies padded to 8."""
    body = b""
    for t, d in msgs:
        d = d + bytes((-len(d)) % 8)
        body += u16(t) + u16(len(d)) + u8(0) + bytes(3) + d
    return u8(1) + u8(0) + u16(len(msgs)) + u32(1) + u32(len(body)) + bytes(4) + body


def link_msg(name: str, addr: int) -> bytes:
    nm = name.encode()
    return u8(1) + u8(0) + u8(len(nm)) + nm + u64(addr)  # hard link, 1-byte name length


def attr_msg(version: int, name: str, value, np_dtype) -> bytes:
    nm = name.encode() + b"\0"
    dt = dtype_msg(np_dtype)
    sp = u8(1) + u8(0) + u8(0) + u8(0) + bytes(4) if version == 1 else u8(2) + u8(0) + u8(0) + u8(0)
    val = np.array([value], np_dtype).tobytes()
    pad = (lambda x: x + bytes((-len(x)) % 8)) if version == 1 else (lambda x: x)
    head = u8(version) + u8(0) + u16(len(nm)) + u16(len(dt)) + u16(len(sp))
    if version == 3:
        head += u8(0)  # name character set: ASCII
    return head + pad(nm) + pad(dt) + pad(sp) + val


def chunk_origins(dims, chunk):
    grid = [(d + c - 1) // c for d, c in zip(dims, chunk)]
    return [tuple(int(i) * c for i, c in zip(idx, chunk)) for idx in np.ndindex(*grid)]


def chunk_bytes(arr, org, chunk) -> bytes:
    """The chunk at `org`, full chunk shape, zero past the dataset's edge."""
    out = np.zeros(chunk, arr.dtype)
    sl = tuple(slice(o, min(o + c, d)) for o, c, d in zip(org, chunk, arr.shape))
    out[tuple(slice(0, s.stop - s.start) for s in sl)] = arr[sl]
    return out.tobytes()


def layout_v4(chunk, itemsize, index_type, addr, extra=b"") -> bytes:
    dims = list(chunk) + [itemsize]
    return (u8(4) + u8(2) + u8(0) + u8(len(dims)) + u8(8) + b"".join(u64(d) for d in dims) + u8(index_type)
            + extra + u64(addr))


def finish_v2_superblock(img: Img, root_oh: int, version: int = 2):
    sb = SIG + u8(version) + u8(8) + u8(8) + u8(0) + u64(0) + u64(UNDEF) + u64(len(img.b)) + u64(root_oh)
    img.put(0, sb + u32(lookup3(sb)))


def file_v2(dset_name: str, dset_msgs_fn, version: int = 2, extra_links=()) -> bytes:
    """Superblock v2/3, root group with compact links; dset_msgs_fn(img)
    writes the data and returns the dataset's messages."""
    img = Img()
    img.reserve(48)
    msgs = dset_msgs_fn(img)
    ds_oh = img.add(ohdr_v2(msgs))
    links = [(0x0006, link_msg(dset_name, ds_oh))] + [(0x0006, link_msg(n, ds_oh)) for n in extra_links]
    root = img.add(ohdr_v2(links))
    finish_v2_superblock(img, root, version)
    return bytes(img.b)


def fixed_array_msgs(arr, chunk, skip=(), order=None):
    """Dataset messages of a chunked dataset with a fixed-array index;
    chunks listed in `skip` are never written (fill value 0)."""
    def fn(img):
        origins = chunk_origins(arr.shape, chunk)
        addrs = [UNDEF] * len(origins)
        for k in (order if order is not None else range(len(origins))):
            if k in skip:
                continue
            addrs[k] = img.add(chunk_bytes(arr, origins[k], chunk))
        hdr_at = img.reserve(28)
        blk = b"FADB" + u8(0) + u8(0) + u64(hdr_at) + b"".join(u64(a) for a in addrs)
        blk_at = img.add(blk + u32(lookup3(blk)))
        hdr = b"FAHD" + u8(0) + u8(0) + u8(8) + u8(10) + u64(len(origins)) + u64(blk_at)
        img.put(hdr_at, hdr + u32(lookup3(hdr)))
        return [(1, dataspace_v2(arr.shape)), (3, dtype_msg(arr.dtype)),
                (8, layout_v4(chunk, arr.dtype.itemsize, 3, hdr_at, extra=u8(10)))]
    return fn


# ---------------------------------------------------------------- tests

def write(tmp_path, name, data):
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


def test_superblock2_fixed_array_measurement(tmp_path):
    rng = np.random.default_rng(0)
    arr = rng.random((3, 5, 4, 5, 4)).astype(np.float32)
    chunk = (2, 3, 4, 2, 3)  # does not divide 3, 5, 5, 4
    n = len(chunk_origins(arr.shape, chunk))
    order = list(rng.permutation(n))
    p = write(tmp_path, "fa.h5", file_v2("messung", fixed_array_msgs(arr, chunk, skip={5}, order=order)))
    want = arr.copy()
    o = chunk_origins(arr.shape, chunk)[5]
    want[tuple(slice(a, a + c) for a, c in zip(o, chunk))] = 0.0  # an unwritten chunk reads as the fill value
    got = h5.read_measurement(p)
    assert got.shape == arr.shape and np.array_equal(got, want)


def test_superblock3_single_chunk_density_with_v3_attributes(tmp_path):
    arr = np.arange(6 * 7 * 5, dtype=np.float32).reshape(6, 7, 5) * 0.25
    attrs = {"xmin": -0.006, "xmax": 0.006, "ymin": -0.007, "ymax": 0.007, "zmin": -0.005, "zmax": 0.005}

    def fn(img):
        at = img.add(arr.tobytes())
        msgs = [(1, dataspace_v2(arr.shape)), (3, dtype_msg(np.float32)),
                (8, layout_v4(arr.shape, 4, 1, at))]
        for k, v in attrs.items():
            msgs.append((0x000C, attr_msg(3, k, v, np.float32)))
        for k, v in zip(("xnbin", "ynbin", "znbin"), arr.shape):
            msgs.append((0x000C, attr_msg(3, k, v, np.int32)))
        return msgs

    p = write(tmp_path, "single.h5", file_v2("density", fn, version=3))
    d, grid = h5.read_density(p)
    assert np.array_equal(d, arr)
    assert grid["n"] == arr.shape
    assert np.allclose(grid["min"], [attrs["xmin"], attrs["ymin"], attrs["zmin"]])
    assert np.allclose(grid["max"], [attrs["xmax"], attrs["ymax"], attrs["zmax"]])


def test_implicit_chunk_index_with_v2_attributes_and_float64(tmp_path):
    arr = np.random.default_rng(1).random((5, 4, 6))  # float64 on disk
    chunk = (2, 4, 4)

    def fn(img):
        at = None
        for org in chunk_origins(arr.shape, chunk):
            a = img.add(chunk_bytes(arr, org, chunk))
            at = a if at is None else at
        msgs = [(1, dataspace_v2(arr.shape)), (3, dtype_msg(np.float64)), (8, layout_v4(chunk, 8, 2, at))]
        for ax, k in zip("xyz", arr.shape):
            msgs += [(0x000C, attr_msg(2, ax + "min", -1.0, np.float32)),
                     (0x000C, attr_msg(2, ax + "max", 1.0, np.float32)),
                     (0x000C, attr_msg(2, ax + "nbin", k, np.int32))]
        return msgs

    p = write(tmp_path, "implicit.h5", file_v2("density", fn))
    d, grid = h5.read_density(p)
    assert np.array_equal(d, arr.astype(np.float32)) and grid["n"] == arr.shape


def btree_v1_chunks(img, arr, chunk, fanout=3):
    """Version-1 B-tree (node type 1) over the chunks, two levels when there
    are more than `fanout` chunks; returns the root's address."""
    r = arr.ndim
    origins = chunk_origins(arr.shape, chunk)
    csize = int(np.prod(chunk)) * arr.dtype.itemsize
    data = [img.add(chunk_bytes(arr, o, chunk)) for o in origins[::-1]][::-1]  # stored last chunk first

    def key(org):
        return u32(csize) + u32(0) + b"".join(u64(v) for v in org) + u64(0)

    end_key = key(tuple(arr.shape))

    def node(level, keys, children, last):
        b = b"TREE" + u8(1) + u8(level) + u16(len(children)) + u64(UNDEF) + u64(UNDEF)
        for k, c in zip(keys, children):
            b += k + u64(c)
        return b + last

    leaves, first_keys = [], []
    for s in range(0, len(origins), fanout):
        ks = [key(o) for o in origins[s:s + fanout]]
        last = key(origins[s + fanout]) if s + fanout < len(origins) else end_key
        leaves.append(img.add(node(0, ks, data[s:s + fanout], last)))
        first_keys.append(ks[0])
    if len(leaves) == 1:
        return leaves[0]
    return img.add(node(1, first_keys, leaves, end_key))


def file_v0_chunked(name, arr, chunk) -> bytes:
    """Superblock 0, root group as a symbol table, a version-1 dataset header
    with a chunked version-3 layout indexed by a version-1 B-tree."""
    img = Img()
    img.reserve(96)
    bt = btree_v1_chunks(img, arr, chunk)
    dims = list(chunk) + [arr.dtype.itemsize]
    layout = u8(3) + u8(2) + u8(len(dims)) + u64(bt) + b"".join(u32(d) for d in dims)
    space = u8(1) + u8(arr.ndim) + u8(0) + u8(0) + bytes(4) + b"".join(u64(d) for d in arr.shape)
    ds_oh = img.add(ohdr_v1([(1, space), (3, dtype_msg(arr.dtype)), (8, layout)]))
    # local heap with "" and the name, symbol table node, group B-tree
    names = b"\0" * 8 + name.encode() + b"\0"
    names += bytes((-len(names)) % 8)
    heap_data = img.add(names)
    heap = img.add(b"HEAP" + u8(0) + bytes(3) + u64(len(names)) + u64(UNDEF) + u64(heap_data))
    snod = img.add(b"SNOD" + u8(1) + u8(0) + u16(1) + u64(8) + u64(ds_oh) + u32(0) + u32(0) + bytes(16))
    gtree = img.add(b"TREE" + u8(0) + u8(0) + u16(1) + u64(UNDEF) + u64(UNDEF) + u64(0) + u64(snod) + u64(8))
    root_oh = img.add(ohdr_v1([(0x11, u64(gtree) + u64(heap))]))
    sb = (SIG + u8(0) + u8(0) + u8(0) + u8(0) + u8(0) + u8(8) + u8(8) + u8(0) + u16(4) + u16(16) + u32(0)
          + u64(0) + u64(UNDEF) + u64(len(img.b)) + u64(UNDEF))
    entry = u64(0) + u64(root_oh) + u32(1) + u32(0) + u64(gtree) + u64(heap)
    img.put(0, sb + entry)
    return bytes(img.b)


def test_superblock0_btree_chunked_measurement(tmp_path):
    arr = np.random.default_rng(2).random((2, 3, 5, 4, 3)).astype(np.float32)
    chunk = (1, 2, 3, 4, 2)
    p = write(tmp_path, "btree.h5", file_v0_chunked("messung", arr, chunk))
    assert len(chunk_origins(arr.shape, chunk)) > 3  # two B-tree levels
    assert np.array_equal(h5.read_measurement(p), arr)


def test_unsupported_forms_are_reported(tmp_path):
    arr = np.ones((4, 4, 4), np.float32)

    def filtered(img):
        msgs = fixed_array_msgs(arr, (4, 4, 4))(img)
        deflate = u8(2) + u8(1) + u16(1) + u16(0) + u16(1) + u32(6)  # version 2, one filter: deflate level 6
        return msgs + [(0x000B, deflate)]

    p = write(tmp_path, "filtered.h5", file_v2("density", filtered))
    with pytest.raises(h5.H5Error, match="filtered"):
        h5.read(p, "density")

    def ext_array(img):
        return [(1, dataspace_v2(arr.shape)), (3, dtype_msg(np.float32)),
                (8, layout_v4((2, 2, 2), 4, 4, img.reserve(8), extra=bytes(5)))]

    p = write(tmp_path, "earray.h5", file_v2("density", ext_array))
    with pytest.raises(h5.H5Error, match="index type 4"):
        h5.read(p, "density")
    # a root group whose links live in a fractal heap
    img = Img()
    img.reserve(48)
    linfo = u8(0) + u8(0) + u64(1234) + u64(UNDEF)
    root = img.add(ohdr_v2([(0x0002, linfo)]))
    finish_v2_superblock(img, root)
    p = write(tmp_path, "dense.h5", bytes(img.b))
    with pytest.raises(h5.H5Error, match="dense storage"):
        h5.read(p, "density")
    # a superblock version the reader does not know
    bad = bytearray(file_v2("density", fixed_array_msgs(arr, (4, 4, 4))))
    bad[8] = 4
    p = write(tmp_path, "sb4.h5", bytes(bad))
    with pytest.raises(h5.H5Error, match="superblock version 4"):
        h5.read(p, "density")


def test_other_names_are_not_found(tmp_path):
    arr = np.ones((2, 2, 2), np.float32)
    p = write(tmp_path, "links.h5", file_v2("density", fixed_array_msgs(arr, (2, 2, 2)), extra_links=("copy",)))
    assert np.array_equal(h5.read(p, "copy"), arr)  # a second hard link to the same dataset
    with pytest.raises(h5.H5Error, match="no dataset"):
        h5.read(p, "messung")
