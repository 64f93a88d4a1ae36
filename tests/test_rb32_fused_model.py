"""CPU check of the fused FP32 red+black pass's dataflow (tests/rb32_model.py):
tiles, halo rows and columns, the z march with its shared-memory rings and
register history, periodic wrap and walls -- against the two colour sweeps,
bit for bit, on grids with partial tiles, tiles wider than the grid, periodic
and wall-bounded y."""
import numpy as np
import pytest

from tests import rb32_model as R


def _case(nx, ny, nz, py, seed):
    rng = np.random.default_rng(seed)
    g = R.Grid(nx, ny, nz, py)
    shp = (nz + 2, ny + 2, nx + 2)
    P = {"idx": np.float32(nx / 1.3), "idy": np.float32(ny / 0.9), "idz": np.float32(nz / 1.7),
         "idt": np.float32(123.0)}
    du, dv, dw, dp, r = (rng.uniform(-1, 1, shp).astype(np.float32) for _ in range(5))
    if not py:
        dv[:, 0, :] = 0.0
        dv[:, ny + 1, :] = 0.0
    mu_u, mu_v, mu_w = (rng.uniform(0.2, 1.0, shp[1:]).astype(np.float32) for _ in range(3))
    fac = (-rng.uniform(0.5, 1.5, shp[1:]) / (2 * (P["idx"] ** 2 + P["idy"] ** 2 + P["idz"] ** 2))).astype(
        np.float32)
    return g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac


@pytest.mark.parametrize("nx,ny,nz,py,TI,TJ,TK", [
    (8, 6, 4, 0, 4, 2, 2),
    (12, 5, 6, 0, 8, 2, 4),
    (8, 6, 6, 1, 4, 4, 4),
    (4, 4, 4, 1, 8, 4, 8),
    (6, 3, 2, 0, 4, 4, 4),
])
def test_fused_pass_equals_two_sweeps(nx, ny, nz, py, TI, TJ, TK):
    g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac = _case(nx, ny, nz, py, nx * 100 + ny * 10 + nz)
    ru, rv, rw, rdp = R.two_sweeps(g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac)
    fu, fv, fw, fdp = R.fused(g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac, TI, TJ, TK)
    inner = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    for name, a, b in (("u", fu, ru), ("v", fv, rv), ("w", fw, rw), ("dp", fdp, rdp)):
        assert np.array_equal(a[inner], b[inner]), (name, np.argwhere(a[inner] != b[inner])[:5])
    if not py:   # the wall faces stay 0
        assert not fv[:, 0, :].any() and not fv[:, ny + 1, :].any()
