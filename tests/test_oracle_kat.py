"""Known-answer tests of the CPU oracle, derived from the discrete equations
(the reference has no tests or fixtures of its own)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import channel_case, oracle_channel_ic, random_fields


def _laplacian_rhs_layout(g, phi):
    """7-point Laplacian of phi(ny,nz,nx) with periodic x/z and the Neumann
    rows of pressure_fft.f90:70-82 in y."""
    lap = (np.roll(phi, 1, 2) - 2 * phi + np.roll(phi, -1, 2)) / g.dx ** 2
    lap += (np.roll(phi, 1, 1) - 2 * phi + np.roll(phi, -1, 1)) / g.dz ** 2
    up = np.concatenate([phi[1:], phi[-1:]], 0)
    dn = np.concatenate([phi[:1], phi[:-1]], 0)
    lap += (up - 2 * phi + dn) / g.dy ** 2
    return lap


def test_rk3_identities():
    a, b, c = O.rk_coeffs()
    for s in range(3):
        assert abs(a[s] + b[s] - c[s]) < 1e-16
    assert abs(sum(c) - 1.0) < 1e-15
    assert b[0] == 0.0


@pytest.mark.parametrize("m,n,l", [(3, 2, 5), (1, 0, 1), (0, 3, 2), (7, 5, 0)])
def test_poisson_eigenmode(m, n, l):
    g = O.Grid(32, 24, 16, lx=2 * np.pi, ly=2.0, lz=np.pi)
    i = np.arange(g.nx)
    j = np.arange(1, g.ny + 1)
    k = np.arange(g.nz)
    phi = (np.cos(2 * np.pi * m * i / g.nx)[None, None, :] * np.cos(np.pi * n * (j - 0.5) / g.ny)[:, None, None]
           * np.cos(2 * np.pi * l * k / g.nz)[None, :, None])
    lam = -(4 / g.dx ** 2 * np.sin(np.pi * m / g.nx) ** 2 + 4 / g.dz ** 2 * np.sin(np.pi * l / g.nz) ** 2
            + 4 / g.dy ** 2 * np.sin(np.pi * n / (2 * g.ny)) ** 2)
    sol = O.solve_pressure_fft(g, lam * phi)
    if m == 0 and l == 0:
        phi = phi - phi[0:1]          # zero mode pinned at the j = 1 plane
    assert np.abs(sol - phi).max() < 1e-12


def test_operator_residual_and_zero_mode_pin():
    g = O.Grid(24, 20, 12, lx=2.0, ly=1.5, lz=1.0)
    rhs = np.random.default_rng(1).standard_normal((g.ny, g.nz, g.nx))
    rhs -= rhs.mean()                 # compatible right-hand side
    phi = O.solve_pressure_fft(g, rhs)
    res = _laplacian_rhs_layout(g, phi) - rhs
    assert np.abs(res).max() <= 1e-12 * np.abs(rhs).max() * (2 / g.dy ** 2 + 4 / g.dx ** 2) * g.dy ** 2
    assert abs(phi[0].mean()) < 1e-13 * np.abs(phi).max()


def test_projection_is_divergence_free():
    g, bc = channel_case(32, 24, 16)
    f = random_fields(g, 2, scale=0.5)
    O.apply_bc(g, f)
    O.pressure_projection_fft(g, f, 0.5e-3)
    O.apply_bc(g, f)
    l2, linf = O.divergence_norms(g, bc, f)
    assert linf <= 1e-12


def test_uniform_flow_is_exact():
    g = O.Grid(16, 8, 8, re=500.0, forcing=(0.7, 0.0, 0.0))
    bc = O.BC((True, True, True))
    f = O.Fields(g)
    f.un[...] = 1.25
    dt = 3e-3
    a, b, c = O.rk_coeffs()
    O.momentum(g, bc, f, dt * a[0], dt * b[0], dt * c[0])
    assert np.all(f.us[1:-1, 1:-1, 1:-1] == 1.25 + dt * a[0] * 0.7)
    assert np.all(f.vs[1:-1, 1:-1, 1:-1] == 0.0) and np.all(f.ws[1:-1, 1:-1, 1:-1] == 0.0)
    assert np.all(f.oldrhsu == 0.7)


def test_redblack_sweep_order_independent():
    """Same-colour cells share no face: the OpenMP-parallel sweep equals the
    sequential loop of pressure_redblack.f90:103-245 bit for bit."""
    g = O.Grid(16, 10, 12, re=300.0)
    for bc in (O.channel_bc(), O.BC((False, False, False)).set(2, 0, 0, typ=1).set(1, 1, 2, typ=1, value=0.2)):
        f1 = random_fields(g, 5, "random")
        f2 = f1.copy()
        O.pressure_projection_redblack(g, bc, f1, 1e-3, niter=4, sor=1.6, parallel=True)
        O.pressure_projection_redblack(g, bc, f2, 1e-3, niter=4, sor=1.6, parallel=False)
        for n in ("un", "vn", "wn", "pn"):
            assert np.array_equal(getattr(f1, n), getattr(f2, n))


def test_redblack_converges_to_tolerance():
    g, bc = channel_case(32, 16, 16)
    f = random_fields(g, 6, scale=0.2)
    st, it, res = O.pressure_projection_redblack(g, bc, f, 1e-3, sor=1.7, tol=1e-10, check_every=10)
    assert st == 0 and res <= 1e-10 and it % 10 == 0
    l2, _ = O.divergence_norms(g, bc, f)
    assert l2 >= 0.0


def test_restart_at_step_boundary_is_exact():
    """beta_1 = 0 (step.f90:22): oldrhs is not needed across a step boundary,
    so dropping it (as the HDF5 restart does) changes nothing."""
    g, bc = channel_case(24, 16, 12)
    f = O.Fields(g)
    oracle_channel_ic(g, bc, f, 5)
    ref = f.copy()
    O.run(g, bc, ref, g.dt, 4, solver=0)
    O.run(g, bc, f, g.dt, 2, solver=0)
    for n in O.RHS_NAMES:
        getattr(f, n)[...] = 0.0
    f.us[...] = 0.0
    f.vs[...] = 0.0
    f.ws[...] = 0.0
    O.run(g, bc, f, g.dt, 2, solver=0)
    for n in ("un", "vn", "wn", "pn"):
        assert np.array_equal(getattr(f, n), getattr(ref, n)), n


def test_ibm_reference_geometry():
    """ibm.f90:84-99,156-187: solid below amp/2(1+sin(2 pi x/lx)) + 2dy with amp = 5dy."""
    g = O.Grid(32, 32, 4, re=100.0)
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_reference(g), f)
    solid = f.coef_u == 1e30 / g.re
    ix = np.arange(g.nx + 2)
    iy = np.arange(g.ny + 2)
    x = (ix - 1.0) * g.dx
    y = (iy - 0.5) * g.dy
    yb = 5 * g.dy * 0.5 * (1 + np.sin(2 * np.pi * x / g.lx)) + 2 * g.dy
    expect = y[:, None] < yb[None, :]
    assert np.array_equal(solid[2], expect)
    assert np.all(f.coef_u[:, ~expect] < 1e30 / g.re)
    near = (f.coef_u > 0) & ~solid
    assert near.any()
