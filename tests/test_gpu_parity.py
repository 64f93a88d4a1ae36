"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Bit-exact where the reference arithmetic is followed operation by operation
(predictor, boundary conditions, red-black sweeps); within the FP64
tolerance of the north star (relative L2 <= 1e-11 on u, v, w, p after N
steps, max|div u| <= 1e-12) on the FFT path, whose FFT is a different
algorithm from the oracle's.
"""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, compare_all, oracle_channel_ic, random_fields, rel_l2, to_device

pytestmark = pytest.mark.gpu

BC_CASES = {
    "periodic": lambda: O.BC((True, True, True)),
    "channel": O.channel_bc,
    "walls_mixed": lambda: (O.BC((False, False, False))
                            .set(1, 0, 1, typ=0, value=0.3).set(1, 1, 1, typ=1, value=-0.2)
                            .set(2, 0, 2, typ=1, value=0.1).set(2, 1, 2, typ=0, value=0.05)
                            .set(3, 0, 3, typ=0, value=-0.1).set(3, 1, 3, typ=1, value=0.2)
                            .set(2, 0, 1, typ=1, value=0.4).set(2, 1, 3, typ=1, value=-0.3)
                            .set(1, 0, 0, typ=1, value=0.01).set(1, 1, 0, typ=0, value=0.02)
                            .set(2, 0, 0, typ=0, value=0.03).set(2, 1, 0, typ=1, value=0.04)
                            .set(3, 0, 0, typ=1, value=0.05).set(3, 1, 0, typ=0, value=0.06)),
}


@pytest.mark.parametrize("bcname", list(BC_CASES))
@pytest.mark.parametrize("ibm", ["none", "random"])
def test_momentum_bitwise(bcname, ibm):
    g = O.Grid(20, 12, 10, lx=2.0, ly=1.5, lz=1.0, re=350.0, forcing=(0.3, -0.2, 0.1))
    bc = BC_CASES[bcname]()
    f = random_fields(g, 11, ibm)
    with to_device(M, g, bc, f) as s:
        a, b, c = O.rk_coeffs()
        dt = 2e-3
        for st in range(3):
            O.momentum(g, bc, f, dt * a[st], dt * b[st], dt * c[st])
            s.momentum(dt * a[st], dt * b[st], dt * c[st])
        diff = compare_all(s, f)
    assert all(v == 0.0 for v in diff.values()), diff


def test_apply_bc_bitwise():
    g = O.Grid(18, 10, 12)
    f = random_fields(g, 3)
    with to_device(M, g, O.channel_bc(), f) as s:
        O.apply_bc(g, f)
        s.apply_bc()
        diff = compare_all(s, f)
    assert all(v == 0.0 for v in diff.values()), diff


@pytest.mark.parametrize("bcname", list(BC_CASES))
def test_apply_bc_redblack_bitwise(bcname):
    g = O.Grid(16, 10, 12, lx=1.3, ly=0.7, lz=2.0)
    bc = BC_CASES[bcname]()
    f = random_fields(g, 5)
    with to_device(M, g, bc, f) as s:
        O.apply_bc_redblack(g, bc, f)
        s.apply_bc_redblack()
        diff = compare_all(s, f)
    assert all(v == 0.0 for v in diff.values()), diff


@pytest.mark.parametrize("bcname", list(BC_CASES))
@pytest.mark.parametrize("ibm", ["none", "random", "zinv"])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
def test_redblack_fixed_iterations_bitwise(bcname, ibm, variant):
    """pressure_projection_redblack with the reference's fixed nIter: bit-exact with
    every kernel variant -- one launch per colour sweep (1), the fused red+black passes
    (2, 3), the sweeps on colour-split copies (4) and with two cells per thread (5), the
    autotuner's choice (0); 2-5 run when x and z are periodic and the IBM factors are 1
    or z-invariant."""
    g = O.Grid(16, 10, 12, lx=1.3, ly=0.7, lz=2.0, re=500.0)
    bc = BC_CASES[bcname]()
    f = random_fields(g, 7, ibm)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, n_iter=3, sor=1.5, sor_variant=variant))
        O.pressure_projection_redblack(g, bc, f, 0.37e-3, niter=3, sor=1.5, tol=0.0)
        s.pressure_projection(0.37e-3)
        diff = compare_all(s, f)
    assert all(v == 0.0 for v in diff.values()), diff


@pytest.mark.parametrize("shape,kz", [((36, 10, 6), 4), ((64, 24, 20), 16), ((40, 12, 10), 3), ((96, 48, 34), 8)])
@pytest.mark.parametrize("bcname", ["periodic", "channel"])
@pytest.mark.parametrize("variant", [2, 3, 4, 5])
def test_redblack_fused_partial_tiles_bitwise(shape, kz, bcname, variant):
    """Fused passes on grids that are not multiples of their 32x8 / 32x16 tiles or z
    chunk, and the colour-split sweeps on the same odd sizes."""
    g = O.Grid(*shape, lx=1.1, ly=0.8, lz=1.7, re=800.0)
    bc = BC_CASES[bcname]()
    f = random_fields(g, 13, "zinv")
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, n_iter=5, sor=1.7, sor_kz=kz,
                                                  sor_variant=variant))
        O.pressure_projection_redblack(g, bc, f, 0.5e-3, niter=5, sor=1.7, tol=0.0)
        s.pressure_projection(0.5e-3)
        diff = compare_all(s, f, ["un", "vn", "wn", "pn"])
    assert all(v == 0.0 for v in diff.values()), diff


@pytest.mark.parametrize("variant", [0, 1, 4, 5])
def test_redblack_residual_driven_matches_oracle(variant):
    g, bc = channel_case(32, 16, 16, re=3000.0)
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_wavy(0.05, g.lx / 2, 0.0), f)
    oracle_channel_ic(g, bc, f, 99, solver=1, wave_amp=0.05, wave_lambda=g.lx / 2)
    f.us[...] = f.un + 0.01 * np.sin(np.arange(f.un.size).reshape(f.un.shape))
    f.vs[...] = f.vn
    f.ws[...] = f.wn
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-10, check_every=10,
                                                  adaptive_checks=False, sor_variant=variant))
        st_o, it_o, res_o = O.pressure_projection_redblack(g, bc, f, 1e-3 * 64 / 120, sor=1.7, tol=1e-10,
                                                           check_every=10)
        st = s.pressure_projection(1e-3 * 64 / 120)
        assert st_o == 0 and st.status == 0
        assert st.iterations == it_o
        diff = compare_all(s, f, ["un", "vn", "wn", "pn"])
    assert all(v == 0.0 for v in diff.values()), diff


@pytest.mark.parametrize("shape", [(32, 16, 24), (64, 64, 64), (48, 32, 80), (200, 20, 24)])
def test_fft_projection(shape):
    nx, ny, nz = shape
    g, bc = channel_case(nx, ny, nz)
    f = random_fields(g, 21, scale=0.5)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        O.apply_bc(g, f)
        s.apply_bc()
        phi_o = O.pressure_projection_fft(g, f, 0.4e-3)
        s.pressure_projection(0.4e-3)
        assert rel_l2(s.get("phi"), phi_o) < 1e-12
        for n in ("un", "vn", "wn", "pn"):
            assert rel_l2(s.get(n), getattr(f, n)) < 1e-12, n


def test_fft_projection_ibm_reference_geometry():
    g = O.Grid(32, 24, 16, lx=1.0, ly=1.0, lz=1.0, re=100.0)
    bc = O.channel_bc()
    f = random_fields(g, 4, "reference", scale=0.3)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver()
        O.apply_bc(g, f)
        s.apply_bc()
        O.pressure_projection_fft(g, f, 1e-4)
        s.pressure_projection(1e-4)
        for n in ("un", "vn", "wn", "pn"):
            assert rel_l2(s.get(n), getattr(f, n)) < 1e-12, n


def _c0_pair(nsteps, shape=(64, 64, 64), ibm=False):
    g, bc = channel_case(*shape, re=2000.0, dt=1e-3)
    f = O.Fields(g)
    if ibm:
        O.set_ibm_coeff(g, O.ibm_reference(g), f)
    oracle_channel_ic(g, bc, f, 20261203)
    s = to_device(M, g, bc, O.Fields(g))
    s.enter_ibm_data(f.coef_u, f.coef_v, f.coef_w)
    s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
    s.channel_ic(20261203)
    for n in ("un", "vn", "wn"):
        assert rel_l2(s.get(n), getattr(f, n)) < 1e-13, n
    O.run(g, bc, f, g.dt, nsteps, solver=0)
    s.step(nsteps)
    return g, bc, f, s


def test_c0_channel_100_steps():
    """Config 0: 64^3 channel, Re 2000, dt 1e-3, 100 RK3 steps, FFT+Thomas FP64."""
    g, bc, f, s = _c0_pair(100)
    with s:
        errs = {n: rel_l2(s.get(n), getattr(f, n)) for n in ("un", "vn", "wn", "pn")}
        l2, linf = s.divergence_norms()
    assert all(e <= 1e-11 for e in errs.values()), errs
    assert linf <= 1e-12, linf


def test_c0_reference_ibm_variant():
    g, bc, f, s = _c0_pair(10, shape=(32, 32, 16), ibm=True)
    with s:
        errs = {n: rel_l2(s.get(n), getattr(f, n)) for n in ("un", "vn", "wn", "pn")}
    assert all(e <= 1e-11 for e in errs.values()), errs


def test_c1_wavy_redblack_truncated():
    """Config-1 geometry (wavy IBM walls, RB-SOR omega 1.7 to 1e-10) on a reduced grid, 2 steps."""
    ly = 2.25
    y0 = (ly - 2.0) / 2.0
    g = O.Grid(64, 32, 32, lx=2 * np.pi, ly=ly, lz=np.pi, re=3000.0, dt=1e-3, forcing=(2.0 / 3000.0, 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_wavy(0.05, g.lx / 2, y0), f)
    oracle_channel_ic(g, bc, f, 20261203, solver=1, sor=1.7, tol=1e-10, check_every=50, y0=y0,
                      wave_amp=0.05, wave_lambda=g.lx / 2)
    s = to_device(M, g, bc, O.Fields(g))
    with s:
        s.enter_ibm_data(f.coef_u, f.coef_v, f.coef_w)
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-10, check_every=50,
                                                  adaptive_checks=False))
        s.channel_ic(20261203, y0=y0, wave_amp=0.05, wave_lambda=g.lx / 2)
        for n in ("un", "vn", "wn"):
            assert np.array_equal(s.get(n), getattr(f, n)), n
        st, it_o = O.run(g, bc, f, g.dt, 2, solver=1, sor=1.7, tol=1e-10, check_every=50)
        it_g = s.step(2)
        assert st == 0 and it_g == it_o
        for n in ("un", "vn", "wn", "pn"):
            assert rel_l2(s.get(n), getattr(f, n)) <= 1e-11, n


def test_step_graph_equals_eager():
    g, bc = channel_case(32, 16, 16)
    f = random_fields(g, 8, scale=0.3)
    O.apply_bc(g, f)
    s1 = to_device(M, g, bc, f)
    s2 = to_device(M, g, bc, f)
    with s1, s2:
        for s in (s1, s2):
            s.init_pressure_solver()
        s1.step(3)                              # CUDA graph replay
        a, b, c = M.rk_coeffs()
        for _ in range(3):
            for st in range(3):
                s2.momentum(g.dt * a[st], g.dt * b[st], g.dt * c[st])
                s2.apply_bc()
                s2.pressure_projection(g.dt * c[st])
                s2.apply_bc()
        for n in ("un", "vn", "wn", "pn", "us", "oldrhsu"):
            assert np.array_equal(s1.get(n), s2.get(n)), n


def test_cfl_and_center_vel():
    g, bc = channel_case(24, 12, 16)
    f = random_fields(g, 9)
    with to_device(M, g, bc, f) as s:
        assert s.get_cfl() == O.get_cfl(g, f)
        uc, vc, wc = s.center_vel()
        un, vn, wn = f.un, f.vn, f.wn
        assert np.array_equal(uc, 0.5 * (un[1:-1, 1:-1, 1:-1] + un[1:-1, 1:-1, 2:]))
        assert np.array_equal(vc, 0.5 * (vn[1:-1, 1:-1, 1:-1] + vn[1:-1, 2:, 1:-1]))
        assert np.array_equal(wc, 0.5 * (wn[1:-1, 1:-1, 1:-1] + wn[2:, 1:-1, 1:-1]))


def test_update_host_device_roundtrip():
    g, bc = channel_case(16, 8, 8)
    f = random_fields(g, 10)
    with to_device(M, g, bc, f) as s:
        z = [np.zeros(g.padded) for _ in range(4)]
        s.update_host(*z)
        for a, n in zip(z, ("un", "vn", "wn", "pn")):
            assert np.array_equal(a, getattr(f, n))
        z[0][...] = 7.0
        s.update_device(un=z[0])
        assert np.array_equal(s.get("un"), z[0])
