"""HDF5-subset field files (bastr_h5_*, host code; no libhdf5 exists here to check against).

The reference keeps its fields in HDF5 files written by libhdf5 (hdf5io.F90): datasets u1, u2[, u3]
of H5T_NATIVE_DOUBLE with Fortran dimensions (ia+1, ja+1, ka+1) holding the grid values in
[0:ia, 0:ja, 0:max(ka,1)) (hdf5io.F90:752-802), and nstep / time datasets of one element
(hdf5io.F90:1009-1184).  These tests check the library's writer and reader by:

- round trips of 2D and 3D fields with and without counters, and of many datasets (several
  symbol-table nodes);
- the bytes of a written file against the HDF5 File Format Specification, read by a small
  independent parser in this file (superblock version 0 fields, the root group's B-tree, symbol
  table node and local heap, each dataset's dataspace, datatype and layout messages, the zero
  padding row and column);
- files patched by hand into forms libhdf5 writes but this writer does not (compact storage, an
  object-header continuation block), which the reader must follow;
- error cases (missing dataset, wrong datatype, not an HDF5 file, unsupported superblock).
"""
import os
import struct

import numpy as np
import pytest

from bastr_b200 import BASTR_E_INVALID, BASTR_E_UNSUPPORTED, BastrError, h5_read, h5_write, read_field, write_field

U64 = struct.Struct("<Q")


def u(buf, at, n):
    return int.from_bytes(buf[at:at + n], "little")


# ----------------------------------------------------------------------------------------------
# an independent parser of the specification's structures, for the checks below
# ----------------------------------------------------------------------------------------------
def superblock(buf):
    assert buf[:8] == b"\x89HDF\r\n\x1a\n"
    return dict(version=buf[8], freespace_version=buf[9], root_version=buf[10], shared_version=buf[12],
                size_offsets=buf[13], size_lengths=buf[14], leaf_k=u(buf, 16, 2), internal_k=u(buf, 18, 2),
                flags=u(buf, 20, 4), base=u(buf, 24, 8), freespace=u(buf, 32, 8), eof=u(buf, 40, 8),
                driver=u(buf, 48, 8), root_name=u(buf, 56, 8), root_oh=u(buf, 64, 8), root_cache=u(buf, 72, 4),
                root_btree=u(buf, 80, 8), root_heap=u(buf, 88, 8))


def messages(buf, oh):
    """(type, data offset, size) of a version 1 object header without continuation blocks."""
    assert buf[oh] == 1
    n, size = u(buf, oh + 2, 2), u(buf, oh + 8, 4)
    at, end, out = oh + 16, oh + 16 + size, []
    for _ in range(n):
        t, sz = u(buf, at, 2), u(buf, at + 2, 2)
        assert sz % 8 == 0 and at + 8 + sz <= end
        out.append((t, at + 8, sz))
        at += 8 + sz
    return out


def root_entries(buf):
    sb = superblock(buf)
    heap = sb["root_heap"]
    assert buf[heap:heap + 4] == b"HEAP"
    heap_data = u(buf, heap + 24, 8)
    tree = sb["root_btree"]
    assert buf[tree:tree + 4] == b"TREE" and buf[tree + 4] == 0 and buf[tree + 5] == 0
    out = {}
    for c in range(u(buf, tree + 6, 2)):
        snod = u(buf, tree + 24 + 8 + 16 * c, 8)
        assert buf[snod:snod + 4] == b"SNOD" and buf[snod + 4] == 1
        for i in range(u(buf, snod + 6, 2)):
            e = snod + 8 + 40 * i
            off = u(buf, e, 8)
            name = buf[heap_data + off:buf.index(b"\0", heap_data + off)].decode()
            out[name] = u(buf, e + 8, 8)
    return out


def dataset(buf, oh):
    d = {}
    for t, at, sz in messages(buf, oh):
        if t == 1:
            assert buf[at] == 1
            d["dims"] = [u(buf, at + 8 + 8 * i, 8) for i in range(buf[at + 1])]
        elif t == 3:
            d["class"], d["size"], d["bits0"] = buf[at] & 15, u(buf, at + 4, 4), buf[at + 1]
            d["version"] = buf[at] >> 4
        elif t == 8:
            assert buf[at] == 3 and buf[at + 1] == 1
            d["addr"], d["nbytes"] = u(buf, at + 2, 8), u(buf, at + 10, 8)
    return d


def field(shape, seed):
    return [np.random.default_rng(seed + c).standard_normal(shape) for c in range(2 if len(shape) == 2 else 3)]


# ----------------------------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(24, 40), (6, 10, 12)], ids=["2d", "3d"])
def test_field_round_trip(tmp_path, shape):
    uu = field(shape, 3)
    p = str(tmp_path / "flowfield0001.h5")
    write_field(p, uu, nstep=1234, time=0.1234)
    ka, ja, ia = (0, *shape) if len(shape) == 2 else shape
    got, n, t = read_field(p, ia, ja, ka, counters=True)
    assert n == 1234 and t == 0.1234
    for a, b in zip(got, uu):
        assert np.array_equal(a, b)
    # an initial-field file has no counters
    write_field(p, uu)
    assert all(np.array_equal(a, b) for a, b in zip(read_field(p, ia, ja, ka), uu))
    with pytest.raises(BastrError) as e:
        read_field(p, ia, ja, ka, counters=True)
    assert e.value.code == BASTR_E_INVALID and "nstep" in str(e.value)


@pytest.mark.parametrize("shape", [(24, 40), (6, 10, 12)], ids=["2d", "3d"])
def test_written_bytes_follow_the_specification(tmp_path, shape):
    uu = field(shape, 5)
    p = str(tmp_path / "f.h5")
    write_field(p, uu, nstep=7, time=0.5)
    buf = open(p, "rb").read()
    sb = superblock(buf)
    assert (sb["version"], sb["freespace_version"], sb["root_version"], sb["shared_version"]) == (0, 0, 0, 0)
    assert (sb["size_offsets"], sb["size_lengths"], sb["leaf_k"], sb["internal_k"]) == (8, 8, 4, 16)
    assert sb["base"] == 0 and sb["eof"] == len(buf) and sb["freespace"] == sb["driver"] == 2 ** 64 - 1
    assert sb["root_cache"] == 1 and sb["root_oh"] == 96
    # the root object header holds a symbol table message naming the same B-tree and heap
    (t, at, sz), = messages(buf, sb["root_oh"])
    assert t == 0x11 and (u(buf, at, 8), u(buf, at + 8, 8)) == (sb["root_btree"], sb["root_heap"])
    ents = root_entries(buf)
    names = ["time", "nstep", "u1", "u2"] + (["u3"] if len(shape) == 3 else [])
    assert sorted(ents) == sorted(names)
    assert list(ents) == sorted(ents)            # symbol table entries in name order
    ka, ja, ia = (0, *shape) if len(shape) == 2 else shape
    for c, name in enumerate(names[2:]):
        d = dataset(buf, ents[name])
        # Fortran (ia+1, ja+1, ka+1) is C order [ka+1][ja+1][ia+1]
        assert d["dims"] == [ka + 1, ja + 1, ia + 1]
        assert (d["class"], d["size"], d["bits0"] & 1) == (1, 8, 0)      # IEEE float, 8 bytes, little-endian
        assert d["nbytes"] == 8 * (ka + 1) * (ja + 1) * (ia + 1)
        a = np.frombuffer(buf, np.float64, d["nbytes"] // 8, d["addr"]).reshape(d["dims"])
        nz = max(ka, 1)
        assert np.array_equal(a[:nz, :ja, :ia].reshape(uu[c].shape), uu[c])
        assert not a[:, ja, :].any() and not a[:, :, ia].any()
        if ka:
            assert not a[ka].any()
        assert np.array_equal(h5_read(p, name), a)
    dn = dataset(buf, ents["nstep"])
    assert dn["dims"] == [1] and (dn["class"], dn["size"], dn["bits0"] & 8) == (0, 4, 8)   # signed int32
    assert u(buf, dn["addr"], 4) == 7
    dt = dataset(buf, ents["time"])
    assert dt["dims"] == [1] and struct.unpack_from("<d", buf, dt["addr"])[0] == 0.5


def test_many_datasets_span_several_symbol_table_nodes(tmp_path):
    sets = {f"v{i:02d}": np.arange(i + 1, dtype=np.float64) * 0.5 for i in range(20)}
    sets["random_angle"] = np.linspace(0, 1, 12).reshape(3, 4)
    sets["count"] = np.array([3, -4], dtype=np.int32)
    p = str(tmp_path / "many.h5")
    h5_write(p, sets)
    buf = open(p, "rb").read()
    assert u(buf, superblock(buf)["root_btree"] + 6, 2) == 3   # 22 entries, 8 per symbol table node
    assert sorted(root_entries(buf)) == sorted(sets)
    for k, v in sets.items():
        assert np.array_equal(h5_read(p, k, v.dtype), v)


def test_reader_follows_compact_storage_and_continuation_blocks(tmp_path):
    uu = field((8, 16), 9)
    p = str(tmp_path / "f.h5")
    write_field(p, uu, nstep=42, time=2.5)
    buf = bytearray(open(p, "rb").read())
    ents = root_entries(bytes(buf))
    # nstep: turn its contiguous layout into compact storage holding another value
    for t, at, sz in messages(bytes(buf), ents["nstep"]):
        if t == 8:
            buf[at:at + 24] = bytes([3, 0]) + (4).to_bytes(2, "little") + (-17).to_bytes(4, "little", signed=True) \
                + bytes(16)
    # time: move its layout message into a continuation block at the end of the file
    oh = ents["time"]
    for t, at, sz in messages(bytes(buf), oh):
        if t == 8:
            layout_msg = bytes(buf[at - 8:at + sz])
            block = len(buf)
            buf[at - 8:at - 6] = (0x10).to_bytes(2, "little")   # same 24-byte slot, padded
            buf[at:at + sz] = U64.pack(block) + U64.pack(len(layout_msg)) + bytes(sz - 16)
            buf += layout_msg
            buf[oh + 2:oh + 4] = (u(buf, oh + 2, 2) + 1).to_bytes(2, "little")
    buf[40:48] = U64.pack(len(buf))
    open(p, "wb").write(bytes(buf))
    got, n, t = read_field(p, 16, 8, 0, counters=True)
    assert n == -17 and t == 2.5
    assert all(np.array_equal(a, b) for a, b in zip(got, uu))


def test_reader_errors(tmp_path):
    p = str(tmp_path / "f.h5")
    write_field(p, field((8, 16), 1), nstep=1, time=0.0)
    with pytest.raises(BastrError) as e:
        h5_read(p, "u3")
    assert e.value.code == BASTR_E_INVALID and "u3" in str(e.value)
    with pytest.raises(BastrError) as e:
        h5_read(p, "nstep", np.float64)
    assert e.value.code == BASTR_E_INVALID
    with pytest.raises(BastrError):
        read_field(p, 16, 16, 0)          # the file's grid is 16 x 8
    q = str(tmp_path / "not.h5")
    open(q, "wb").write(b"plain text, not HDF5" * 10)
    with pytest.raises(BastrError) as e:
        h5_read(q, "u1")
    assert e.value.code == BASTR_E_INVALID
    buf = bytearray(open(p, "rb").read())
    buf[8] = 2                             # superblock version 2 (libhdf5's newest format)
    open(q, "wb").write(bytes(buf))
    with pytest.raises(BastrError) as e:
        h5_read(q, "u1")
    assert e.value.code == BASTR_E_UNSUPPORTED
    with pytest.raises(BastrError):
        read_field(str(tmp_path / "missing.h5"), 16, 8, 0)
    assert not os.path.exists(str(tmp_path / "missing.h5"))
