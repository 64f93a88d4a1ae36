"""Residual-check schedule of the red-black solves: checks spaced by the
convergence rate of the last two reach the same tolerance as checks every
check_every iterations, with fewer checks, FP64 and mixed precision."""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import oracle_channel_ic, rel_l2, to_device

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


@pytest.mark.parametrize("precision", [M.PREC_FP64, M.PREC_MIXED])
def test_adaptive_checks_reach_tolerance_with_fewer_checks(precision):
    g, bc, f = _wavy_case()
    tol, every = 1e-8, 10
    solvers = []
    for adaptive in (True, False):
        s = to_device(M, g, bc, f)
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=tol, check_every=every,
                                                  max_iter=200000, precision=precision,
                                                  adaptive_checks=adaptive))
        s.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
        solvers.append(s)
    sa, sf = solvers
    with sa, sf:
        for s in solvers:
            s.step(2)
            s.set_timing(True)
        ia, i_f = sa.step(3), sf.step(3)
        ca, cf = sa.get_timing()["residual"][1], sf.get_timing()["residual"][1]
        print("iterations adaptive", ia, "fixed", i_f, "residual launches", ca, cf)
        st = sa.last_solve_stats()
        assert st.status == 0 and st.iterations % every == 0
        l2, _ = sa.divergence_norms()
        assert l2 <= max(tol * st.residual0, st.atol) * 1.0000001
        assert abs(ia - i_f) <= 0.05 * i_f + 9 * every
        assert ca < (0.6 if precision == M.PREC_FP64 else 0.9) * cf
        for n in ("un", "vn", "wn"):
            assert rel_l2(sa.get(n), sf.get(n)) <= 1e-6, n
