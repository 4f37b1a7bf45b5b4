"""Reader for the subset of the HDF5 file format that the library writes
(test infrastructure; no HDF5 package is available to the tests): a
version-0 superblock with 8-byte offsets and lengths, a root group held in
a symbol table (v1 B-tree of group nodes, symbol table nodes, local heap),
datasets with version-1 object headers, version-1 dataspaces,
floating-point / fixed-point datatypes and contiguous layouts.  Written from
the published file-format specification; every structure is checked as it
is read."""
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


def _u(b, at, n):
    return int.from_bytes(b[at:at + n], "little")


def _messages(b, oh):
    """(type, data) of a version-1 object header's messages."""
    assert b[oh] == 1, "object header version"
    nmsg, size = _u(b, oh + 2, 2), _u(b, oh + 8, 4)
    at, end, out = oh + 16, oh + 16 + size, []
    for _ in range(nmsg):
        mtype, msize = _u(b, at, 2), _u(b, at + 2, 2)
        assert msize % 8 == 0, "message data not aligned"
        out.append((mtype, b[at + 8:at + 8 + msize]))
        at += 8 + msize
    assert at == end, "header size does not match its messages"
    return out


def _name(heap, off):
    end = heap.index(b"\0", off)
    return heap[off:end].decode()


def _dataset(b, oh):
    dims, dtype, addr, size = None, None, None, None
    for mtype, d in _messages(b, oh):
        if mtype == 0x0001:  # dataspace, version 1
            assert d[0] == 1 and d[2] == 0
            dims = tuple(_u(d, 8 + 8 * k, 8) for k in range(d[1]))
        elif mtype == 0x0003:  # datatype
            cls, ver, nbytes = d[0] & 0x0F, d[0] >> 4, _u(d, 4, 4)
            assert ver == 1 and nbytes == 8
            if cls == 1:  # floating point
                assert d[1] & 1 == 0 and (d[1] >> 4) & 3 == 2 and d[2] == 63
                off, prec, eloc, esz, mloc, msz, bias = struct.unpack("<HHBBBBI", d[8:20])
                assert (off, prec, eloc, esz, mloc, msz, bias) == (0, 64, 52, 11, 0, 52, 1023)
                dtype = "<f8"
            elif cls == 0:  # fixed point
                assert d[1] & 1 == 0
                assert struct.unpack("<HH", d[8:12]) == (0, 64)
                dtype = "<i8" if d[1] & 8 else "<u8"
            else:
                raise AssertionError("datatype class %d" % cls)
        elif mtype == 0x0008:  # data layout
            assert d[0] == 3 and d[1] == 1, "contiguous layout, version 3"
            addr, size = _u(d, 2, 8), _u(d, 10, 8)
    n = int(np.prod(dims)) if dims else 1
    assert size == 8 * n and addr + size <= len(b)
    a = np.frombuffer(b[addr:addr + size], dtype=dtype)
    return a.reshape(dims) if dims else a[0]


def read(path):
    """{name: array or scalar} of the root group."""
    b = open(path, "rb").read()
    assert b[:8] == SIGNATURE and b[8] == 0, "superblock version 0"
    assert b[13] == 8 and b[14] == 8, "8-byte offsets and lengths"
    leaf_k, internal_k = _u(b, 16, 2), _u(b, 18, 2)
    assert _u(b, 24, 8) == 0 and _u(b, 32, 8) == UNDEF and _u(b, 48, 8) == UNDEF
    assert _u(b, 40, 8) == len(b), "end-of-file address"
    root_oh, cache = _u(b, 56 + 8, 8), _u(b, 56 + 16, 4)
    cached_bt, cached_heap = _u(b, 56 + 24, 8), _u(b, 56 + 32, 8)
    stab = [d for t, d in _messages(b, root_oh) if t == 0x0011]
    assert len(stab) == 1
    bt, hp = _u(stab[0], 0, 8), _u(stab[0], 8, 8)
    assert cache == 1 and (bt, hp) == (cached_bt, cached_heap)
    # local heap
    assert b[hp:hp + 4] == b"HEAP" and b[hp + 4] == 0
    dsize, free, daddr = _u(b, hp + 8, 8), _u(b, hp + 16, 8), _u(b, hp + 24, 8)
    assert free == 1 or free < dsize
    heap = b[daddr:daddr + dsize]
    assert heap[0] == 0, "the empty name at offset 0"
    # B-tree (group nodes, leaf level)
    assert b[bt:bt + 4] == b"TREE" and b[bt + 4] == 0 and b[bt + 5] == 0
    used = _u(b, bt + 6, 2)
    assert 1 <= used <= 2 * internal_k
    keys = [_u(b, bt + 24 + 16 * k, 8) for k in range(used + 1)]
    children = [_u(b, bt + 32 + 16 * k, 8) for k in range(used)]
    out = {}
    for c, (lo, hi) in zip(children, zip(keys, keys[1:])):
        assert b[c:c + 4] == b"SNOD" and b[c + 4] == 1
        nsym = _u(b, c + 6, 2)
        assert nsym <= 2 * leaf_k
        names = []
        for k in range(nsym):
            e = c + 8 + 40 * k
            name = _name(heap, _u(b, e, 8))
            assert _u(b, e + 16, 4) == 0, "no cached data for a dataset"
            names.append(name)
            out[name] = _dataset(b, _u(b, e + 8, 8))
        assert names == sorted(names), "symbol table node in name order"
        assert _name(heap, lo) < names[0] and names[-1] == _name(heap, hi), "B-tree keys"
    return out
