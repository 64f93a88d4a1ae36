"""Walls in x or z on the FFT path (pressure Neumann there).

The reference's FFT builds take periodic x and z only (boundary.f90:23-170,
pressure_fft.f90:20-148); its red-black path takes walls in any direction
(boundary.f90:173-368, pressure_redblack.f90:27-254).  With walls the FFT
path solves the pressure equation on the even extension of the grid, which
is the Neumann problem the converged red-black iteration solves.  Checks:
- CPU: the identity behind it -- the periodic spectral solve of the mirrored
  right-hand side restricted to the grid satisfies the Neumann-operator
  equation -- on a 2-D example with numpy's FFT;
- GPU: the projection leaves a divergence-free field with the wall faces at
  their boundary values; one projection and three RK3 steps agree with the
  oracle's red-black solution converged to round-off (the red-black method
  with the same boundary conditions); a pressure-Dirichlet wall is refused.
"""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import random_fields, rel_l2, to_device


def _neumann_lap_1d(n, h):
    L = np.zeros((n, n))
    for i in range(n):
        if i > 0:
            L[i, i - 1] += 1.0
            L[i, i] -= 1.0
        if i < n - 1:
            L[i, i + 1] += 1.0
            L[i, i] -= 1.0
    return L / (h * h)


def test_even_extension_solves_the_neumann_problem():
    nx, nz, hx, hz = 12, 10, 0.3, 0.7
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((nz, nx))
    rhs -= rhs.mean()                                  # compatible with Neumann in both directions
    ext = np.concatenate([rhs, rhs[:, ::-1]], axis=1)
    ext = np.concatenate([ext, ext[::-1, :]], axis=0)  # (2nz, 2nx), mirrored about the walls
    kx = np.arange(2 * nx)
    kz = np.arange(2 * nz)
    lam = -(4 / hx ** 2) * np.sin(np.pi * kx / (2 * nx)) ** 2 - (4 / hz ** 2) * np.sin(np.pi * kz[:, None] / (2 * nz)) ** 2
    hat = np.fft.fft2(ext)
    lam[0, 0] = 1.0
    hat = hat / lam
    hat[0, 0] = 0.0
    phi = np.real(np.fft.ifft2(hat))[:nz, :nx]
    L = np.kron(np.eye(nz), _neumann_lap_1d(nx, hx)) + np.kron(_neumann_lap_1d(nz, hz), np.eye(nx))
    assert np.allclose(L @ phi.ravel(), rhs.ravel(), atol=1e-10 * np.abs(rhs).max())


def _walls_bc(x_wall, z_wall):
    """No-slip walls (velocity Dirichlet 0) in y and where asked in x and z,
    Neumann pressure on every wall."""
    bc = O.BC((not x_wall, False, not z_wall))
    for d, wall in ((1, x_wall), (2, True), (3, z_wall)):
        if wall:
            bc.set(d, 0, 0, typ=1, value=0.0).set(d, 1, 0, typ=1, value=0.0)
    return bc


CASES = [(True, False), (False, True), (True, True)]


@pytest.mark.gpu
@pytest.mark.parametrize("x_wall,z_wall", CASES)
def test_projection_divergence_free_with_walls(x_wall, z_wall):
    g = O.Grid(32, 12, 16, lx=1.3, ly=0.8, lz=1.1, re=400.0)
    bc = _walls_bc(x_wall, z_wall)
    f = random_fields(g, 17, scale=0.5)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.apply_bc()
        s.pressure_projection(0.3e-3)
        s.apply_bc()
        l2, linf = s.divergence_norms()
        un, wn = s.get("un"), s.get("wn")
    assert linf <= 1e-12, linf
    if x_wall:   # wall faces u(1), u(nx+1) at their value 0
        assert not un[1:-1, 1:-1, 1].any() and not un[1:-1, 1:-1, g.nx + 1].any()
    if z_wall:
        assert not wn[1, 1:-1, 1:-1].any() and not wn[g.nz + 1, 1:-1, 1:-1].any()


def _zero_mean(a):
    a = a[1:-1, 1:-1, 1:-1]
    return a - a.mean()


@pytest.mark.gpu
@pytest.mark.parametrize("x_wall,z_wall", CASES)
def test_projection_with_walls_matches_converged_redblack(x_wall, z_wall):
    g = O.Grid(24, 12, 20, lx=1.3, ly=0.8, lz=1.1, re=400.0)
    bc = _walls_bc(x_wall, z_wall)
    f = random_fields(g, 23, scale=0.5)
    dg = 0.3e-3
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.apply_bc()
        s.pressure_projection(dg)
        s.apply_bc()
        got = {n: s.get(n) for n in ("un", "vn", "wn", "pn")}
    # tol 1e-14 of ||div u*|| or the round-off floor, whichever is larger
    st, it, res = O.pressure_projection_redblack(g, bc, f, dg, sor=1.8, tol=1e-14, max_iter=400000, check_every=20)
    O.apply_bc_redblack(g, bc, f)
    for n in ("un", "vn", "wn"):
        assert rel_l2(got[n], getattr(f, n)) <= 1e-10, (n, rel_l2(got[n], getattr(f, n)), it)
    assert rel_l2(_zero_mean(got["pn"]), _zero_mean(f.pn)) <= 1e-9


@pytest.mark.gpu
def test_duct_steps_match_converged_redblack():
    """Three RK3 steps of a duct (walls in y and z, periodic x) on the FFT
    path against the oracle's red-black steps converged to round-off."""
    g = O.Grid(32, 16, 12, lx=2.0, ly=1.0, lz=0.8, re=300.0, dt=2e-3, forcing=(1.0, 0.0, 0.0))
    bc = _walls_bc(False, True)
    f = random_fields(g, 29, scale=0.2)
    for n in O.RHS_NAMES:
        getattr(f, n)[...] = 0.0
    O.apply_bc_redblack(g, bc, f)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.step(3)
        got = {n: s.get(n) for n in ("un", "vn", "wn", "pn")}
    st, it = O.run(g, bc, f, g.dt, 3, solver=1, sor=1.8, tol=1e-14, max_iter=400000, check_every=20)
    for n in ("un", "vn", "wn"):
        assert rel_l2(got[n], getattr(f, n)) <= 1e-9, (n, rel_l2(got[n], getattr(f, n)))
    assert rel_l2(_zero_mean(got["pn"]), _zero_mean(f.pn)) <= 1e-8


@pytest.mark.gpu
def test_pressure_dirichlet_wall_is_refused():
    g = O.Grid(16, 8, 8)
    bc = _walls_bc(True, False)
    bc.set(1, 0, 0, typ=0, value=0.0)
    with to_device(M, g, bc, O.Fields(g)) as s:
        with pytest.raises(M.MdxError, match="Neumann pressure"):
            s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
