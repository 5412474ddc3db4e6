"""HDF5 measurement / density files without libhdf5: round trips through
the library's writer and reader, and an independent walk of the written
bytes along the HDF5 file format (superblock 0, symbol-table root group,
version-1 object headers) in plain Python."""
import struct

import numpy as np
import pytest

from raptr_b200 import config as cfg
from raptr_b200 import h5

UNDEF = 0xFFFFFFFFFFFFFFFF


def test_density_round_trip(tmp_path):
    g = cfg.SMALL
    x = np.random.default_rng(1).random(g.n_voxels).astype(np.float32)
    p = str(tmp_path / "d.h5")
    h5.write_density(p, x, g)
    d, grid = h5.read_density(p)
    assert d.shape == tuple(g.grid_n) and np.array_equal(d.ravel(), x)
    assert grid["n"] == tuple(g.grid_n)
    assert np.allclose(grid["min"], g.grid_o) and np.allclose(grid["max"], [-o for o in g.grid_o], atol=1e-7)


def test_measurement_round_trip(tmp_path):
    g = cfg.SMALL
    y = np.random.default_rng(2).poisson(3.0, g.n_channels).astype(np.float32)
    p = str(tmp_path / "m.h5")
    h5.write_measurement(p, y, g)
    m = h5.read_measurement(p)
    assert m.shape == (g.na, g.n0z, g.n0y, g.n1z, g.n1y)
    assert np.array_equal(m.ravel(), y)  # channel id order: id1y fastest


def walk(b: bytes):
    """Independent reader of the written structures; returns {name: (dims,
    dtype class, size, data bytes, attributes)}."""
    u8 = lambda o: b[o]
    u16 = lambda o: struct.unpack_from("<H", b, o)[0]
    u32 = lambda o: struct.unpack_from("<I", b, o)[0]
    u64 = lambda o: struct.unpack_from("<Q", b, o)[0]
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert (u8(8), u8(9), u8(10), u8(12), u8(13), u8(14)) == (0, 0, 0, 0, 8, 8)
    leaf_k, internal_k = u16(16), u16(18)
    assert u64(24) == 0 and u64(32) == UNDEF and u64(40) == len(b) and u64(48) == UNDEF
    root_oh, cache = u64(64), u32(72)
    assert cache == 1
    btree, heap = u64(80), u64(88)
    # root object header: one symbol table message naming the same B-tree/heap
    assert u8(root_oh) == 1 and u16(root_oh + 2) == 1
    assert u16(root_oh + 16) == 0x11 and (u64(root_oh + 24), u64(root_oh + 32)) == (btree, heap)
    assert b[heap:heap + 4] == b"HEAP"
    hsize, hdata = u64(heap + 8), u64(heap + 24)
    assert b[hdata] == 0  # offset 0: the empty name
    assert b[btree:btree + 4] == b"TREE" and u8(btree + 4) == 0 and u8(btree + 5) == 0
    used = u16(btree + 6)
    out = {}
    for i in range(used):
        snod = u64(btree + 32 + 16 * i)
        assert b[snod:snod + 4] == b"SNOD" and u8(snod + 4) == 1
        for s in range(u16(snod + 6)):
            e = snod + 8 + 40 * s
            off = u64(e)
            assert off < hsize
            name = b[hdata + off:b.index(b"\0", hdata + off)].decode()
            oh = u64(e + 8)
            assert oh % 8 == 0 and u8(oh) == 1
            nmsg, size = u16(oh + 2), u32(oh + 8)
            p, end = oh + 16, oh + 16 + size
            dims, cls, esize, addr, nbytes, attrs, types = None, None, None, None, None, {}, []
            for _ in range(nmsg):
                t, ln = u16(p), u16(p + 2)
                assert ln % 8 == 0 and p + 8 + ln <= end
                body = p + 8
                types.append(t)
                if t == 1:
                    assert u8(body) == 1
                    dims = tuple(u64(body + 8 + 8 * k) for k in range(u8(body + 1)))
                elif t == 3:
                    cls, esize = u8(body) & 15, u32(body + 4)
                    assert u8(body) >> 4 == 1
                elif t == 8:
                    assert u8(body) == 3 and u8(body + 1) == 1
                    addr, nbytes = u64(body + 2), u64(body + 10)
                elif t == 12:
                    nl, tl, sl = u16(body + 2), u16(body + 4), u16(body + 6)
                    an = b[body + 8:body + 8 + nl - 1].decode()
                    q = body + 8 + (nl + 7) // 8 * 8
                    acls = u8(q) & 15
                    q2 = q + (tl + 7) // 8 * 8
                    assert u8(q2) == 1 and u8(q2 + 1) == 0  # scalar dataspace
                    q3 = q2 + (sl + 7) // 8 * 8
                    attrs[an] = struct.unpack_from("<f" if acls == 1 else "<i", b, q3)[0]
                p = body + ln
            assert {1, 3, 5, 8} <= set(types)
            count = int(np.prod(dims))
            assert nbytes == count * esize and addr + nbytes <= len(b)
            out[name] = (dims, cls, esize, b[addr:addr + nbytes], attrs)
    assert leaf_k == 4 and internal_k == 16
    return out


def test_written_structures_follow_the_format(tmp_path):
    g = cfg.epet_geometry(12, 0.003, 2, 90.0)
    x = np.arange(g.n_voxels, dtype=np.float32) * 0.5
    p = tmp_path / "d.h5"
    h5.write_density(str(p), x, g)
    ds = walk(p.read_bytes())
    assert list(ds) == ["density"]
    dims, cls, size, raw, attrs = ds["density"]
    assert dims == tuple(g.grid_n) and (cls, size) == (1, 4)
    assert np.array_equal(np.frombuffer(raw, "<f4"), x)
    assert attrs["xnbin"] == 12 and attrs["ynbin"] == 12 and attrs["znbin"] == 12
    assert attrs["xmin"] == np.float32(g.grid_o[0])
    assert attrs["xmax"] == np.float32(np.float32(g.grid_o[0]) + np.float32(12) * np.float32(g.grid_d[0]))
    y = np.arange(g.n_channels, dtype=np.float32)
    q = tmp_path / "m.h5"
    h5.write_measurement(str(q), y, g)
    ms = walk(q.read_bytes())
    assert ms["messung"][0] == (g.na, g.n0z, g.n0y, g.n1z, g.n1y) and ms["messung"][4] == {}


def test_errors(tmp_path):
    with pytest.raises(h5.H5Error):
        h5.read_measurement(str(tmp_path / "missing.h5"))
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(h5.H5Error):
        h5.read_measurement(str(bad))
    g = cfg.epet_geometry(8, 0.003, 1, 90.0)
    p = tmp_path / "d.h5"
    h5.write_density(str(p), np.ones(g.n_voxels, np.float32), g)
    with pytest.raises(h5.H5Error):
        h5.read_measurement(str(p))  # no "messung" in a density file
    data = p.read_bytes()
    (tmp_path / "cut.h5").write_bytes(data[:len(data) - 100])
    with pytest.raises(h5.H5Error):
        h5.read_density(str(tmp_path / "cut.h5"))
