"""A second, independent reading of a field file against the HDF5 file
format specification (test helper): every structure the checkpoint writer
emits is decoded here field by field and its invariants are checked, so that
the writer is not only read back by its own reader."""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIG = b"\x89HDF\r\n\x1a\n"


def _u(fmt, b, off):
    return struct.unpack_from("<" + fmt, b, off)


def _pad8(n):
    return (n + 7) & ~7


def _messages(b, addr):
    """Version-1 object header at addr -> [(type, flags, data)], with the
    header-size invariant checked and continuation blocks followed."""
    ver, _, nmsg, refc, size = _u("BBHII", b, addr)
    assert ver == 1 and refc >= 1
    blocks, out = [(addr + 16, size)], []
    while blocks:
        start, length = blocks.pop(0)
        p = start
        while p < start + length and len(out) < nmsg:
            typ, msz, flags = _u("HHB", b, p)
            assert msz % 8 == 0, "v1 messages are padded to 8 bytes"
            data = b[p + 8:p + 8 + msz]
            if typ == 0x10:
                blocks.append(_u("QQ", data, 0))
            out.append((typ, flags, data))
            p += 8 + msz
        assert p == start + length, "messages fill the header block exactly"
    assert len(out) == nmsg
    return out


def _dtype(d):
    cls_ver = d[0]
    assert cls_ver >> 4 == 1, "datatype version 1"
    cls = cls_ver & 15
    size = _u("I", d, 4)[0]
    if cls == 1:
        assert size == 8 and d[1] & 1 == 0 and d[2] == 63
        off, prec, eloc, esz, mloc, msz, bias = _u("HHBBBBI", d, 8)
        assert (off, prec, eloc, esz, mloc, msz, bias) == (0, 64, 52, 11, 0, 52, 1023)
        return "<f8", 20
    assert cls == 0 and size == 4 and d[1] & 1 == 0 and d[1] & 8
    assert _u("HH", d, 8) == (0, 32)
    return "<i4", 12


def _dspace(d):
    ver, rank, flags = d[0], d[1], d[2]
    assert ver == 1 and flags == 0
    return tuple(_u("Q" * rank, d, 8)) if rank else ()


def parse(path):
    b = open(path, "rb").read()
    assert b[:8] == SIG
    (sb_ver, fs_ver, root_ver, _, sh_ver, so, sl, _, leaf_k, node_k, flags) = _u("BBBBBBBBHHI", b, 8)
    assert (sb_ver, fs_ver, root_ver, sh_ver, so, sl) == (0, 0, 0, 0, 8, 8)
    base, freesp, eof, driver = _u("QQQQ", b, 24)
    assert base == 0 and freesp == UNDEF and driver == UNDEF and eof == len(b)
    name_off, root_oh, cache, _ = _u("QQII", b, 56)
    btree_a, heap_a = _u("QQ", b, 80)
    assert cache == 1
    attrs, st = {}, None
    for typ, _, d in _messages(b, root_oh):
        if typ == 0x11:
            st = _u("QQ", d, 0)
        elif typ == 0x0C:
            ver, _, nl, tl, sl_ = _u("BBHHH", d, 0)
            assert ver == 1
            name = d[8:8 + nl - 1].decode()
            assert d[8 + nl - 1] == 0
            p = 8 + _pad8(nl)
            dt, tsize = _dtype(d[p:p + tl])
            assert tsize == tl
            p += _pad8(tl)
            assert _dspace(d[p:p + sl_]) == ()
            p += _pad8(sl_)
            attrs[name] = np.frombuffer(d, dtype=dt, count=1, offset=p)[0].item()
    assert st == (btree_a, heap_a)
    assert b[heap_a:heap_a + 4] == b"HEAP" and b[heap_a + 4] == 0
    hsize, free_head, hdata = _u("QQQ", b, heap_a + 8)
    assert free_head == 1 or free_head < hsize
    heap = b[hdata:hdata + hsize]
    assert heap[0] == 0, "offset 0 of a group heap is the empty name"

    def name_at(off):
        return heap[off:heap.index(b"\0", off)].decode()

    assert b[btree_a:btree_a + 4] == b"TREE"
    ntype, level, used = _u("BBH", b, btree_a + 4)
    assert ntype == 0 and level == 0 and used >= 1
    left, right = _u("QQ", b, btree_a + 8)
    assert left == UNDEF and right == UNDEF
    links = {}
    p = btree_a + 24
    keys = [name_at(_u("Q", b, p)[0])]
    for c in range(used):
        child = _u("Q", b, p + 8 + 16 * c)[0]
        keys.append(name_at(_u("Q", b, p + 16 + 16 * c)[0]))
        assert b[child:child + 4] == b"SNOD" and b[child + 4] == 1
        ns = _u("H", b, child + 6)[0]
        assert 1 <= ns <= 2 * leaf_k
        names = []
        for e in range(ns):
            lo, oh, ct, _ = _u("QQII", b, child + 8 + 40 * e)
            names.append(name_at(lo))
            links[names[-1]] = oh
            assert ct == 0
        assert names == sorted(names) and keys[-1] == names[-1]
    assert keys[0] == ""
    dsets = {}
    for name, oh in links.items():
        dims = dt = lay = None
        for typ, fl, d in _messages(b, oh):
            if typ == 0x01:
                dims = _dspace(d)
            elif typ == 0x03:
                dt = _dtype(d)[0]
            elif typ == 0x05:
                assert d[0] == 2
            elif typ == 0x08:
                assert d[0] == 3 and d[1] == 1
                lay = _u("QQ", d, 2)
        assert dt == "<f8" and lay is not None and dims is not None
        addr, size = lay
        assert size == 8 * int(np.prod(dims)) and addr + size <= len(b)
        dsets[name] = np.frombuffer(b, dtype="<f8", count=int(np.prod(dims)), offset=addr).reshape(dims)
    return {"attrs": attrs, "datasets": dsets, "leaf_k": leaf_k, "node_k": node_k}
