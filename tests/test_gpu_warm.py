"""Warm starts of the red-black projection: the increment history, the
previous-step guess (FP64 and mixed precision) and its agreement with the
unguessed solve."""
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


def _solver(g, bc, f, tol, precision=M.PREC_FP64):
    s = to_device(M, g, bc, f)
    s.init_pressure_solver(M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=tol, check_every=25,
                                              precision=precision))
    return s


def test_increments_sum_to_step_change():
    """The three recorded increments of a step add up to its pressure change."""
    g, bc, f = _wavy_case(32, 16, 16)
    s = _solver(g, bc, f, 1e-10)
    with s:
        s.set_pressure_guess(M.GUESS_ZERO, record=True)
        p0 = s.get("pn")[1:-1, 1:-1, 1:-1].copy()
        s.step(1)
        assert s.last_solve_stats().guessed == 0
        p1 = s.get("pn")[1:-1, 1:-1, 1:-1]
        dsum = s.get_increment(0) + s.get_increment(1) + s.get_increment(2)
        assert rel_l2(dsum, p1 - p0) <= 1e-12
        assert np.abs(s.get_increment(2)).max() > 0.0


def test_no_increment_without_record():
    g, bc, f = _wavy_case(32, 16, 16)
    s = _solver(g, bc, f, 1e-8)
    with s:
        s.step(1)
        with pytest.raises(M.MdxError):
            s.get_increment(0)


@pytest.mark.parametrize("precision", [M.PREC_FP64, M.PREC_MIXED])
def test_guesses_save_iterations(precision):
    """Starting each projection from the same substage's increment of the
    previous step, or its linear extrapolation from the two previous steps,
    converges to the same tolerance in fewer sweeps."""
    g, bc, f = _wavy_case()
    tol = 1e-8
    sz = _solver(g, bc, f, tol, precision)
    sp = _solver(g, bc, f, tol, precision)
    se = _solver(g, bc, f, tol, precision)
    with sz, sp, se:
        sp.set_pressure_guess(M.GUESS_PREVIOUS, record=True)
        se.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
        # step 1 has no history; step 2's guess is step 1's pressure build-up
        # from p = 0, which raises the divergence and is undone
        iz0 = sz.step(2)
        assert sp.step(2) == iz0 and se.step(2) == iz0
        assert sp.last_solve_stats().guessed == 0
        iz, ip, ie = sz.step(4), sp.step(4), se.step(4)
        print("iterations, 4 steps: zero", iz, "previous", ip, "extrapolated", ie)
        for s in (sp, se):
            st = s.last_solve_stats()
            assert st.guessed == 1 and st.status == 0
            l2, _ = s.divergence_norms()
            assert l2 <= max(tol * st.residual0, st.atol) * 1.0000001
            # both solves stop within the tolerance of the same projections
            for n in ("un", "vn", "wn"):
                assert rel_l2(s.get(n), sz.get(n)) <= 1e-6, n
            assert rel_l2(s.get("pn"), sz.get("pn")) <= 1e-4
        assert ip < 0.6 * iz
        assert ie < 0.45 * iz and ie < ip


def test_guess_matches_oracle_trajectory():
    """Five extrapolated-guess FP64 steps stay within 1e-6 of the oracle's unguessed ones."""
    g, bc, f = _wavy_case()
    sp = _solver(g, bc, f, 1e-8)
    with sp:
        sp.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
        st, _ = O.run(g, bc, f, g.dt, 5, solver=1, sor=1.7, tol=1e-8, check_every=25)
        assert st == 0
        sp.step(5)
        for n in ("un", "vn", "wn"):
            assert rel_l2(sp.get(n), getattr(f, n)) <= 1e-6, n


def test_checkpoint_replays_the_same_steps():
    """u, v, w, p from the host plus the device checkpoint of the increment
    history replay the same guessed steps bit for bit."""
    g, bc, f = _wavy_case()
    s = _solver(g, bc, f, 1e-8)
    with s:
        s.set_pressure_guess(M.GUESS_EXTRAPOLATED, record=True)
        s.step(4)
        state = [s.get(n).copy() for n in ("un", "vn", "wn", "pn")]
        s.warm_checkpoint()
        ia = s.step(2)
        a = [s.get(n).copy() for n in ("un", "vn", "wn", "pn")]
        s.warm_checkpoint(restore=True)
        s.update_device(*state)
        ib = s.step(2)
        assert ia == ib
        for x, n in zip(a, ("un", "vn", "wn", "pn")):
            assert np.array_equal(x, s.get(n)), n
