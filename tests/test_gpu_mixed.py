"""Mixed precision red-black projection (FP32 sweeps inside FP64 defect
correction) against the FP64 path and the FP64 oracle."""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import oracle_channel_ic, random_fields, rel_l2, to_device

pytestmark = pytest.mark.gpu


def _wavy_case(nx=64, ny=32, nz=32, re=3000.0):
    ly = 2.25
    y0 = (ly - 2.0) / 2.0
    g = O.Grid(nx, ny, nz, lx=2 * np.pi, ly=ly, lz=np.pi, re=re, dt=1e-3, forcing=(2.0 / re, 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_wavy(0.05, g.lx / 2, y0), f)
    oracle_channel_ic(g, bc, f, 20261203, solver=1, sor=1.7, tol=1e-10, check_every=50, y0=y0,
                      wave_amp=0.05, wave_lambda=g.lx / 2)
    return g, bc, f


def _pair(g, bc, f, tol):
    sp = to_device(M, g, bc, f)
    sm = to_device(M, g, bc, f)
    sp.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=tol, check_every=50))
    sm.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=tol, check_every=50,
                                               precision=M.PREC_MIXED))
    return sp, sm


@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_mixed_projection_matches_fp64(tol):
    g, bc, f = _wavy_case()
    a, b, c = O.rk_coeffs()
    O.momentum(g, bc, f, g.dt * a[0], g.dt * b[0], g.dt * c[0])
    sp, sm = _pair(g, bc, f, tol)
    with sp, sm:
        stp = sp.pressure_projection(g.dt * c[0])
        stm = sm.pressure_projection(g.dt * c[0])
        assert stp.status == 0 and stm.status == 0
        assert stm.variant // 100 == 7                # the mixed path ran, in the potential form
        assert stm.residual <= tol * 1.0000001 or stm.residual * stm.residual0 <= stm.atol
        # FP32 sweeps: about as many iterations as FP64
        assert stm.iterations <= 1.5 * stp.iterations + 200
        l2, _ = sm.divergence_norms()
        assert l2 <= max(tol * stm.residual0, stm.atol) * 1.0000001
        # both solves stop within the tolerance of the same projection; the
        # north-star bound for the mixed path is a velocity error <= 1e-6
        errs = {n: rel_l2(sm.get(n), sp.get(n)) for n in ("un", "vn", "wn", "pn")}
        print("mixed vs fp64 rel-L2", tol, errs, stp.iterations, stm.iterations)
        for n in ("un", "vn", "wn"):
            assert errs[n] <= 1e-6, (n, errs)
        assert errs["pn"] <= 1e-4, errs


def test_mixed_two_steps_velocity_error():
    """Two RK3 steps: velocity error of the mixed path vs the FP64 oracle <= 1e-6."""
    g, bc, f = _wavy_case()
    sp, sm = _pair(g, bc, f, 1e-8)
    with sp, sm:
        st, _ = O.run(g, bc, f, g.dt, 2, solver=1, sor=1.7, tol=1e-8, check_every=50)
        assert st == 0
        sm.step(2)
        for n in ("un", "vn", "wn"):
            assert rel_l2(sm.get(n), getattr(f, n)) <= 1e-6, n


def test_mixed_periodic_y():
    g = O.Grid(32, 16, 16, lx=1.3, ly=0.9, lz=1.1, re=700.0, dt=1e-3)
    bc = O.BC((True, True, True))
    f = random_fields(g, 17, "zinv", scale=0.2)
    sp, sm = _pair(g, bc, f, 1e-10)
    with sp, sm:
        stp = sp.pressure_projection(0.5e-3)
        stm = sm.pressure_projection(0.5e-3)
        assert stp.status == 0 and stm.status == 0 and stm.variant > 100
        for n in ("un", "vn", "wn"):
            assert rel_l2(sm.get(n), sp.get(n)) <= 1e-6, n


def test_mixed_falls_back_to_fp64_for_other_boundaries():
    """Walls with Dirichlet pressure (the mixed path needs Neumann): the FP64 path runs, bit for bit."""
    g = O.Grid(32, 16, 16, lx=1.3, ly=0.9, lz=1.1, re=700.0, dt=1e-3)
    bc = O.channel_bc().set(2, 0, 0, typ=0).set(2, 1, 0, typ=0)
    f = random_fields(g, 18, scale=0.2)
    sp, sm = _pair(g, bc, f, 1e-8)
    with sp, sm:
        stp = sp.pressure_projection(0.5e-3)
        stm = sm.pressure_projection(0.5e-3)
        assert stm.variant < 100 and stm.iterations == stp.iterations
        for n in ("un", "vn", "wn", "pn"):
            assert np.array_equal(sm.get(n), sp.get(n)), n



@pytest.mark.parametrize("shape,periodic_y", [((64, 32, 32), False), ((40, 12, 10), False), ((32, 16, 16), True),
                                              ((96, 20, 18), False)])
@pytest.mark.parametrize("tol", [1e-8, 0.0])
def test_fused_and_vector_fp32_sweeps_equal_colour_sweeps(shape, periodic_y, tol):
    """Face form of the FP32 correction sweeps: the fused red+black FP32
    pass (one launch per iteration, every tile shape the autotuner tries) and the vector colour sweeps (2 and 4 cells
    per thread, then the faster) against one launch per colour with one cell
    per thread: the same FP32 corrections bit for bit, so the same
    iterations and the same FP64 state after the projection; tol 0 runs 25
    fixed iterations per inner pass."""
    nx, ny, nz = shape
    if periodic_y:
        g = O.Grid(nx, ny, nz, lx=2.0, ly=1.0, lz=1.0, re=800.0, dt=1e-3, forcing=(0.1, 0.0, 0.0))
        bc = O.BC((True, True, True))
        f = random_fields(g, 31, "zinv", scale=0.3)
    else:
        g, bc, f = _wavy_case(nx, ny, nz)
        a, b, c = O.rk_coeffs()
        O.momentum(g, bc, f, g.dt * a[0], g.dt * b[0], g.dt * c[0])
    out = {}
    # 1: colour sweeps; 2: fused pass only (4 tile shapes, then the tuned
    # one); 4: vector colour sweeps only (2 and 4 cells, then the tuned one)
    for variant in (1, 2, 4):
        with to_device(M, g, bc, f) as s:
            s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=tol or 1e-30, check_every=5,
                                                      max_iter=25 if tol == 0.0 else 100000,
                                                      precision=M.PREC_MIXED, sor_variant=variant,
                                                      adaptive_checks=False, inner_form=1))
            sts = [s.pressure_projection(0.4e-3, check=False) for _ in range(5)]
            out[variant] = ([st.iterations for st in sts], [st.variant for st in sts],
                            {n: s.get(n) for n in ("un", "vn", "wn", "pn")})
    it1, v1, f1 = out[1]
    assert all(v // 100 == 1 for v in v1), v1
    for variant, kind in ((2, 3), (4, 5)):
        it0, v0, f0 = out[variant]
        assert all(v // 100 == kind for v in v0), (variant, v0)
        assert it1 == it0, variant
        for n in f1:
            assert np.array_equal(f1[n], f0[n]), (variant, n, float(np.max(np.abs(f1[n] - f0[n]))))


def _sweep_case(shape, periodic_y):
    nx, ny, nz = shape
    if periodic_y:
        g = O.Grid(nx, ny, nz, lx=2.0, ly=1.0, lz=1.0, re=800.0, dt=1e-3, forcing=(0.1, 0.0, 0.0))
        bc = O.BC((True, True, True))
        f = random_fields(g, 31, "zinv", scale=0.3)
    else:
        g, bc, f = _wavy_case(nx, ny, nz)
        a, b, c = O.rk_coeffs()
        O.momentum(g, bc, f, g.dt * a[0], g.dt * b[0], g.dt * c[0])
    return g, bc, f


# positions per thread of the potential form's sweep shapes (sor_variant 1-15; 0: one warp per row, -1: one
# warp per row with the planes staged in shared memory, -2: one warp per row, a whole block of iterations in
# one cooperative launch)
POT_V = [2, 2, 4, 4, 2, 4, 2, 4, 0, 0, -1, -1, -1, -2, -2]


def _pot_shape_ok(shape, variant):
    nx, ny, _ = shape
    v = POT_V[variant - 1]
    return (nx in (128, 256) and ny % 8 == 0) if v <= 0 else (nx // 2) % v == 0


@pytest.mark.parametrize("shape,periodic_y", [((64, 32, 32), False), ((40, 12, 10), False), ((32, 16, 16), True),
                                              ((96, 20, 18), False), ((128, 24, 20), False), ((128, 16, 12), True)])
def test_potential_form_shapes_agree_and_match_face_form(shape, periodic_y):
    """The potential form of the FP32 correction sweeps (the accumulated phi
    of each cell swept with the 7-point stencil the face updates amount to):
    each shape of its sweep kernel (2 or 4 cells per thread, marches of 4, 8
    or 16 planes, with or without the next plane's prefetch, one warp per
    row, planes staged in shared memory, whole blocks of iterations in one
    cooperative launch; sor_variant 1-15) gives the same bits; against the face form
    the projections meet the same FP64 tolerance with velocity within 1e-6
    and about as many red-black iterations."""
    g, bc, f = _sweep_case(shape, periodic_y)
    nx = shape[0]
    out = {}
    for form, variant in [(1, 1)] + [(0, v) for v in range(1, 16)]:
        if form == 0 and not _pot_shape_ok(shape, variant):
            continue
        with to_device(M, g, bc, f) as s:
            s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=5,
                                                      max_iter=100000, precision=M.PREC_MIXED, sor_variant=variant,
                                                      adaptive_checks=False, inner_form=form))
            sts = [s.pressure_projection(0.4e-3, check=False) for _ in range(3)]
            assert all(st.status == 0 for st in sts)
            l2, _ = s.divergence_norms()
            assert l2 <= max(1e-8 * sts[-1].residual0, sts[-1].atol) * 1.0000001
            out[(form, variant)] = ([st.iterations for st in sts], [st.variant for st in sts],
                                    {n: s.get(n) for n in ("un", "vn", "wn", "pn")})
    it_f, v_f, f_f = out[(1, 1)]
    it_p, v_p, f_p = out[(0, 1)]
    assert all(v // 100 == 1 for v in v_f), v_f
    assert all(v // 100 == 7 for v in v_p), v_p
    for key, (it, v, fl) in out.items():
        if key[0] == 0 and key != (0, 1):
            assert it == it_p, key
            for n in fl:
                assert np.array_equal(fl[n], f_p[n]), (key, n)
    print("iterations face", it_f, "potential", it_p)
    assert sum(it_p) <= 1.3 * sum(it_f) + 50
    num = sum(float(np.sum((f_p[n] - f_f[n]) ** 2)) for n in ("un", "vn", "wn"))
    den = sum(float(np.sum(f_f[n] ** 2)) for n in ("un", "vn", "wn"))
    assert (num / den) ** 0.5 <= 1e-6


def test_potential_form_needs_nx_multiple_of_4():
    """nx = 42 (nx/2 odd): the mixed path runs the face form."""
    g, bc, f = _sweep_case((42, 12, 10), False)
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-8, check_every=5,
                                                  precision=M.PREC_MIXED))
        st = s.pressure_projection(0.4e-3, check=False)
        assert st.status == 0 and st.variant > 100 and st.variant // 100 != 7
