"""CPU check of the potential form of the FP32 correction sweeps
(tests/pot32_model.py, k_pot_sweep): on grids with partial blocks, rows of
one or several vectors, periodic and wall-bounded y and periodic wraps in x
and z, every access is inside the arrays and aligned, no element is written
twice in a sweep, no value a thread uses is written by another thread, and
after several red+black iterations the faces and dp that Phi stands for equal
the face-form sweeps (the update of pressure_redblack.f90:117-241 with
homogeneous boundary values) to FP64 rounding."""
import numpy as np
import pytest

from tests import pot32_model as PM

FILL = np.nan


def _case(nx, ny, nz, py, seed):
    rng = np.random.default_rng(seed)
    shp = (nz + 2, ny + 2, nx + 2)
    idx, idy, idz, idt = nx / 1.3, ny / 0.9, nz / 1.7, 123.0
    r = rng.uniform(-1, 1, shp)
    mu_u, mu_v, mu_w = (rng.uniform(0.2, 1.0, shp[1:]) for _ in range(3))
    fac = np.zeros(shp[1:])
    for j in range(1, ny + 1):
        jp = 1 if (py and j == ny) else j + 1
        for i in range(1, nx + 1):
            ip = 1 if i == nx else i + 1
            denom = ((mu_u[j, i] + mu_u[j, ip]) * idx * idx + (mu_w[j, i] + mu_w[j, i]) * idz * idz
                     + (mu_v[j, i] + mu_v[j, jp]) * idy * idy)
            fac[j, i] = -1.7 / denom
    return (idx, idy, idz, idt), r, mu_u, mu_v, mu_w, fac


@pytest.mark.parametrize("V", [2, 4])
@pytest.mark.parametrize("nx,ny,nz,py,TX,TY,KZ", [
    (8, 6, 4, 0, 1, 2, 2),
    (16, 6, 6, 1, 1, 4, 4),
    (8, 5, 4, 0, 2, 2, 3),     # partial blocks in x, y and z
    (8, 4, 2, 1, 1, 3, 2),
    (16, 8, 8, 0, 2, 4, 16),   # one z block longer than the grid
    (24, 4, 6, 1, 3, 1, 4),
])
def test_potential_sweeps_equal_face_sweeps(nx, ny, nz, py, TX, TY, KZ, V):
    if (nx // 2) % V:
        pytest.skip("rows must hold whole vectors")
    (idx, idy, idz, idt), r, mu_u, mu_v, mu_w, fac = _case(nx, ny, nz, py, nx * 100 + ny * 10 + nz + V)
    iters = 3
    shp = (nz + 2, ny + 2, nx + 2)
    z = np.zeros(shp)
    fu, fv, fw, fdp = PM.face_sweeps(nx, ny, nz, py, idx, idy, idz, idt, z, z, z, z, r, mu_u, mu_v, mu_w, fac,
                                     iters)

    L = PM.PotLayout(nx, ny, nz)
    assert L.hq % 4 == 0 and L.hq >= nx // 2 + 5 and L.H % 64 == 0
    tab = PM.tables(nx, ny, nz, py, idx * idx, idy * idy, idz * idz, mu_u, mu_v, mu_w, fac)
    phi = np.zeros(L.n)
    rl = PM.to_layout(L, r, FILL)
    interior = {L.idx(i, j, k) for k in range(1, nz + 1) for j in range(1, ny + 1) for i in range(1, nx + 1)}
    for _ in range(iters):
        for cs in (1, 0):
            log = PM.Log()
            phi = PM.sweep(L, py, cs, phi, rl, tab, V, TX, TY, KZ, log)
            # each element written by one thread, once
            for e, ts in log.writes.items():
                assert len(ts) == 1, ("written twice", e)
            # no thread uses a value another thread writes
            for e, ts in log.reads.items():
                if e in log.writes:
                    assert ts <= set(log.writes[e]), ("read of another thread's write", e)
            # the swept cells of the interior are all written
            swept = {L.idx(i, j, k) for k in range(1, nz + 1) for j in range(1, ny + 1)
                     for i in range(1, nx + 1) if (i + j + k) & 1 == cs}
            assert swept <= set(log.writes)
            # besides them only the copies of swept cells, in the swept half
            for e in set(log.writes) - swept:
                assert e not in interior
                assert (e >= L.H) == (cs == 1)
            assert np.all(np.isfinite(phi))
    pu, pv, pw, pdp = PM.faces_of_phi(L, py, idx, idy, idz, idt, phi, mu_u, mu_v, mu_w)
    inner = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    for name, a, b in (("u", pu, fu), ("v", pv, fv), ("w", pw, fw), ("dp", pdp, fdp)):
        err = np.max(np.abs(a[inner] - b[inner])) / np.max(np.abs(b[inner]))
        assert err < 1e-12, (name, err)
    # the copies hold the cells they stand for
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            assert phi[L.idx(0, j, k)] == phi[L.idx(nx, j, k)]
            assert phi[L.idx(nx + 1, j, k)] == phi[L.idx(1, j, k)]
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            assert phi[L.idx(i, j, 0)] == phi[L.idx(i, j, nz)]
            assert phi[L.idx(i, j, nz + 1)] == phi[L.idx(i, j, 1)]
    if py:
        for k in range(1, nz + 1):
            for i in range(1, nx + 1):
                assert phi[L.idx(i, 0, k)] == phi[L.idx(i, ny, k)]
                assert phi[L.idx(i, ny + 1, k)] == phi[L.idx(i, 1, k)]


@pytest.mark.parametrize("nx,ny,nz,py,KZ", [(128, 8, 4, 0, 8), (128, 16, 6, 1, 4), (256, 8, 4, 0, 16)])
def test_row_warp_sweeps_equal_thread_sweeps(nx, ny, nz, py, KZ):
    """k_pot_sweep_w (one warp per row, shuffles and a shared-memory row
    exchange) against the thread-by-thread sweep: the same values, copies
    included, after a red and a black sweep from a random Phi."""
    (idx, idy, idz, idt), r, mu_u, mu_v, mu_w, fac = _case(nx, ny, nz, py, nx + ny + nz)
    L = PM.PotLayout(nx, ny, nz)
    tab = PM.tables(nx, ny, nz, py, idx * idx, idy * idy, idz * idz, mu_u, mu_v, mu_w, fac)
    rl = PM.to_layout(L, r, 0.0)
    rng = np.random.default_rng(7)
    phi = np.zeros(L.n)
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                phi[L.idx(i, j, k)] = rng.uniform(-1, 1)
    # the copies a sweep's predecessor leaves
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            phi[L.idx(0, j, k)] = phi[L.idx(nx, j, k)]
            phi[L.idx(nx + 1, j, k)] = phi[L.idx(1, j, k)]
    for j in range(0 if py else 1, ny + 2 if py else ny + 1):
        jj = (j - 1) % ny + 1
        for i in range(0, nx + 2):
            phi[L.idx(i, j, 0)] = phi[L.idx(i, jj, nz)]
            phi[L.idx(i, j, nz + 1)] = phi[L.idx(i, jj, 1)]
    if py:
        for k in range(0, nz + 2):
            for i in range(0, nx + 2):
                phi[L.idx(i, 0, k)] = phi[L.idx(i, ny, k)]
                phi[L.idx(i, ny + 1, k)] = phi[L.idx(i, 1, k)]
    a = b = phi
    for cs in (1, 0):
        a = PM.sweep(L, py, cs, a, rl, tab, 2, 64, 8, KZ)
        b = PM.sweep_rows(L, py, cs, b, rl, tab, KZ)
        assert np.array_equal(a, b), cs


@pytest.mark.parametrize("nz", [2, 7, 16, 128, 130])
def test_cooperative_run_chunks_cover_every_plane_once(nz):
    """k_pot_run_w cuts z into gridDim.y chunks [1 + b nz / n, (b + 1) nz / n]
    (integer division); for every chunk count up to nz the chunks are
    non-empty and cover planes 1..nz exactly once, in order."""
    for n in range(1, nz + 1):
        planes = []
        for b in range(n):
            k0, k1 = 1 + (b * nz) // n, ((b + 1) * nz) // n
            assert k1 >= k0, (n, b)
            planes.extend(range(k0, k1 + 1))
        assert planes == list(range(1, nz + 1)), n
