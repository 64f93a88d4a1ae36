"""CPU check of the vector FP32 colour sweep k_sor_sweep32v (2 or 4 cells per
thread, tests/sweep32v_model.py) on the colour-split arrays with padded rows:
every access inside its array and aligned, no element written by two
threads, no used value written by another thread, the padding positions
untouched, and the red then black sweeps equal to the two colour sweeps of
tests/rb32_model.py bit for bit, over grids whose rows end inside or at the
edge of a window, with periodic and wall-bounded y and both z directions."""
import numpy as np
import pytest

from tests import rb32_model as R
from tests import sweep32v_model as S
from tests.test_rb32_fused_model import _case

FILL = np.uint32(0x7FC0BEEF).view(np.float32)   # a NaN with a payload: padding


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("V", [2, 4])
@pytest.mark.parametrize("nx,ny,nz,py", [
    (6, 4, 4, 0),     # positions 0..3: one window of 4, two of 2
    (8, 6, 4, 0),     # positions 0..4: the last window holds one position
    (12, 5, 6, 0),
    (14, 4, 2, 1),    # positions 0..7, no padding
    (16, 6, 4, 1),    # hs 12: a window of padding only (V = 2)
    (4, 2, 2, 1),
])
def test_vector_sweeps_equal_colour_sweeps(nx, ny, nz, py, V):
    g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac = _case(nx, ny, nz, py, nx * 100 + ny * 10 + nz + V)
    ru, rv, rw, rdp = R.two_sweeps(g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac)

    L = S.Layout(nx, ny, nz)
    assert L.hs % 4 == 0 and L.hs >= nx // 2 + 1
    f = {n: S.to_split(L, a, FILL) for n, a in (("du", du), ("dv", dv), ("dw", dw), ("dp", dp), ("r", r))}
    mu32 = np.concatenate([S.plane_to_split(L, m, FILL) for m in (mu_u, mu_v, mu_w)])
    fac32 = S.plane_to_split(L, fac, FILL)
    elems = {L.cidx(i, j, k) for k in range(L.nzp) for j in range(L.nyp) for i in range(nx + 2)}
    pad = np.array(sorted(set(range(L.n)) - elems), dtype=np.int64)

    for parity in (0, 1):      # first colour: i + j + k odd, as the kernels sweep it
        f, log = S.vector_sweep(L, P, py, parity, V, parity, f, mu32, fac32)
        assert not log.errors, log.errors[:5]
    for n in ("du", "dv", "dw", "dp"):
        if len(pad):
            assert np.array_equal(_bits(f[n][pad]), _bits(np.full(len(pad), FILL))), n
    inner = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    for name, a, b in (("du", f["du"], ru), ("dv", f["dv"], rv), ("dw", f["dw"], rw), ("dp", f["dp"], rdp)):
        got = S.from_split(L, a)
        assert np.array_equal(_bits(got[inner]), _bits(b[inner])), (name, np.argwhere(got[inner] != b[inner])[:5])
        # ghost layers as well (walls, the faces the sweeps leave alone)
        assert np.array_equal(_bits(got), _bits(b)), name
