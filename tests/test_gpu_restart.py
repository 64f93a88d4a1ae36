"""Restart: N steps, the state u, v, w, p copied to the host, a fresh
context from it, M more steps -- bit for bit the N+M-step run (the first
substage has beta_1 = 0, so oldrhs is not read before it is rewritten,
src/modules/step.f90:21-23)."""
import math

import numpy as np
import pytest

import mobydiff_b200 as M

pytestmark = pytest.mark.gpu


def _case(solver, amp):
    nx, ny, nz, re = 32, 32, 32, 2000.0
    ly = 2.25 if amp > 0 else 2.0
    g = M.make_grid(nx, ny, nz, 2 * math.pi, ly, math.pi, re, 1e-3, (2.0 / re, 0.0, 0.0))
    if solver == M.SOLVER_FFT:
        opts = M.make_solver_opts(M.SOLVER_FFT)
    else:
        opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-9, check_every=10)
    y0 = (ly - 2.0) / 2.0
    coef = M.set_ibm_coeff(g, M.ibm_wavy(amp, math.pi, y0)) if amp > 0 else None
    return g, opts, y0, coef


def _solver(g, opts, coef):
    s = M.Solver(g, M.channel_bc(), 0)
    s.enter_field_data()
    if coef is not None:
        s.enter_ibm_data(*coef)
    s.init_pressure_solver(opts)
    return s


@pytest.mark.parametrize("solver,amp", [(M.SOLVER_FFT, 0.0), (M.SOLVER_REDBLACK, 0.05)])
def test_restart_from_host_state_is_bitwise(solver, amp):
    g, opts, y0, coef = _case(solver, amp)
    with _solver(g, opts, coef) as a:
        a.channel_ic(20261203, 0.1, 0.01, y0, amp, math.pi)
        a.step(3)
        saved = [a.get(n).copy() for n in ("un", "vn", "wn", "pn")]
        a.step(2)
        full = [a.get(n) for n in ("un", "vn", "wn", "pn")]
    with _solver(g, opts, coef) as b:
        b.update_device(*saved)
        b.step(2)
        for x, n in zip(full, ("un", "vn", "wn", "pn")):
            assert np.array_equal(x, b.get(n)), n


@pytest.mark.parametrize("solver,amp", [(M.SOLVER_FFT, 0.0), (M.SOLVER_REDBLACK, 0.05)])
def test_restart_through_hdf5_field_file_is_bitwise(tmp_path, solver, amp):
    """write_field / read_field (io.f90:105-166) through a field file: the
    restarted run equals the uninterrupted one, and the file holds the
    context's time and grid."""
    g, opts, y0, coef = _case(solver, amp)
    path = str(tmp_path / "field_3.h5")
    with _solver(g, opts, coef) as a:
        a.channel_ic(20261203, 0.1, 0.01, y0, amp, math.pi)
        a.step(3)
        a.write_field_h5(path)
        on_file = M.h5_read_field(path, g.nx, g.ny, g.nz)
        for x, n in zip(on_file, ("un", "vn", "wn", "pn")):
            assert np.array_equal(x, a.get(n)), n
        a.step(2)
        full = [a.get(n) for n in ("un", "vn", "wn", "pn")]
    h = M.h5_read_header(path)
    assert (h["nx"], h["ny"], h["nz"]) == (g.nx, g.ny, g.nz) and h["dt"] == g.dt and h["re"] == g.re
    assert abs(h["t_current"] - 3 * g.dt) <= 1e-15
    with _solver(g, opts, coef) as b:
        b.read_field_h5(path)
        b.step(2)
        for x, n in zip(full, ("un", "vn", "wn", "pn")):
            assert np.array_equal(x, b.get(n)), n


def test_set_flow_steps_like_a_context_created_at_that_re():
    """Re and body force changed on an existing context (with its IBM
    coefficients re-entered) give the steps of a context created with them."""
    g_a, opts, y0, _ = _case(M.SOLVER_REDBLACK, 0.05)
    g_b = M.make_grid(g_a.nx, g_a.ny, g_a.nz, g_a.lx, g_a.ly, g_a.lz, 3500.0, g_a.dt, (2.0 / 3500.0, 0.0, 0.0))
    geom = M.ibm_wavy(0.05, math.pi, y0)
    a = M.Solver(g_a, M.channel_bc(), 0)
    b = M.Solver(g_b, M.channel_bc(), 0)
    with a, b:
        for s in (a, b):
            s.enter_field_data()
        a.set_flow(3500.0)
        with pytest.raises(M.MdxError):
            a.set_flow(-1.0)
        for s in (a, b):
            s.enter_ibm_geometry(geom)
            s.init_pressure_solver(opts)
            s.channel_ic(20261203, 0.1, 0.01, y0, 0.05, math.pi)
            s.step(2)
        for n in ("un", "vn", "wn", "pn"):
            assert np.array_equal(a.get(n), b.get(n)), n
