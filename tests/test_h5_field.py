"""Field files in HDF5 (field_hdf5.c's content and C entry points) written
and read without libhdf5: round trips, the file decoded independently
against the format specification, and the reference's error returns."""
import math
import os

import numpy as np
import pytest

import mobydiff_b200 as M
from tests import h5_spec


def _grid(nx, ny, nz):
    g = M.make_grid(nx, ny, nz, 2 * math.pi, 2.0, math.pi, 2500.0, 3e-4, (1.0, 0.0, 0.0))
    g.t_current = 0.0123
    return g


def _fields(g, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((g.nz + 2, g.ny + 2, g.nx + 2)) for _ in range(4)]


@pytest.mark.parametrize("shape", [(1, 1, 1), (8, 6, 4), (33, 17, 9)])
def test_round_trip_and_spec_decoding(tmp_path, shape):
    g = _grid(*shape)
    un, vn, wn, pn = _fields(g, sum(shape))
    path = str(tmp_path / "field_7.h5")
    M.h5_write_field(path, g, un, vn, wn, pn)
    back = M.h5_read_field(path, g.nx, g.ny, g.nz)
    for a, b in zip((un, vn, wn, pn), back):
        assert np.array_equal(a, b)
    f = h5_spec.parse(path)
    assert f["leaf_k"] == 4 and f["node_k"] == 16
    assert sorted(f["datasets"]) == ["pn", "un", "vn", "wn"]
    for name, a in zip(("un", "vn", "wn", "pn"), (un, vn, wn, pn)):
        d = f["datasets"][name]
        # dims (nx+2, ny+2, nz+2), element (i, j, k) at ((i nj + j) nk + k): field_hdf5.c:9-12
        assert d.shape == (g.nx + 2, g.ny + 2, g.nz + 2)
        assert np.array_equal(d, a.transpose(2, 1, 0))
    at = f["attrs"]
    assert (at["nx"], at["ny"], at["nz"]) == (g.nx, g.ny, g.nz)
    for k in M.H5_ATTRS:
        assert at[k] == getattr(g, k), k
    h = M.h5_read_header(path)
    assert h == at


def test_reference_error_returns(tmp_path):
    g = _grid(8, 6, 4)
    un, vn, wn, pn = _fields(g, 1)
    path = str(tmp_path / "f.h5")
    M.h5_write_field(path, g, un, vn, wn, pn)
    lib = M.lib()
    out = [np.empty(un.size) for _ in range(4)]
    ptrs = [a.ctypes.data for a in out]
    # dimensions that differ from the file's: field_hdf5.c:119-130
    assert lib.fdm_h5_read_field(path.encode(), 8, 6, 5, *ptrs) == 1
    assert lib.fdm_h5_read_field(path.encode(), 0, 6, 4, *ptrs) == 1      # :193
    assert lib.fdm_h5_read_field(b"/nonexistent/x.h5", 8, 6, 4, *ptrs) == 1
    assert lib.fdm_h5_write_field(path.encode(), 0, 6, 4, *[1.0] * 9, *ptrs) == 1   # :161
    with open(str(tmp_path / "text.h5"), "w") as fh:
        fh.write("not an hdf5 file" * 10)
    assert lib.fdm_h5_read_field(str(tmp_path / "text.h5").encode(), 8, 6, 4, *ptrs) == 1
    assert b"signature" in lib.mdx_h5_last_error()
    data = open(path, "rb").read()
    with open(str(tmp_path / "cut.h5"), "wb") as fh:   # truncated
        fh.write(data[:len(data) // 2])
    assert lib.fdm_h5_read_field(str(tmp_path / "cut.h5").encode(), 8, 6, 4, *ptrs) == 1
    with pytest.raises(M.MdxError):
        M.h5_read_header(str(tmp_path / "cut.h5"))


def test_reader_follows_continuation_blocks(tmp_path):
    """libhdf5 moves messages that overflow an object header into
    continuation blocks: a file whose root attributes sit in one is read."""
    g = _grid(4, 4, 4)
    fields = _fields(g, 3)
    path = str(tmp_path / "a.h5")
    M.h5_write_field(path, g, *fields)
    b = bytearray(open(path, "rb").read())
    root = 96
    ver, _, nmsg, refc, size = np.frombuffer(bytes(b[root:root + 12]), dtype="<u1,<u1,<u2,<u4,<u4")[0]
    # keep the first message (symbol table, 24 bytes) in place and move the
    # rest to a block appended at the end of the file
    body = bytes(b[root + 16:root + 16 + size])
    first, rest = body[:24], body[24:]
    cont_addr = len(b)
    cont = np.array([0x10, 16], dtype="<u2").tobytes() + bytes(4) + np.array([cont_addr, len(rest)], "<u8").tobytes()
    # the filler is a NIL message (type 0) covering the rest of the block
    nil_len = size - len(first) - len(cont) - 8
    new_body = first + cont + np.array([0, nil_len], "<u2").tobytes() + bytes(4) + bytes(nil_len)
    assert len(new_body) == size
    b[root + 16:root + 16 + size] = new_body
    b[root + 2:root + 4] = np.array([nmsg + 2], "<u2").tobytes()
    b += rest
    b[40:48] = np.array([len(b)], "<u8").tobytes()   # end-of-file address
    p2 = str(tmp_path / "b.h5")
    open(p2, "wb").write(bytes(b))
    back = M.h5_read_field(p2, 4, 4, 4)
    for a, c in zip(fields, back):
        assert np.array_equal(a, c)
    h = M.h5_read_header(p2)
    assert h["t_current"] == g.t_current and h["nx"] == 4
