"""Adaptive dt, src/main.f90:66-97: after every step cfl = get_cfl and, when
cflmax > 0 and cfl > 0, dt = min(cflmax/cfl, dtmax).  mdx_step_adaptive
runs the FP64 FFT path as one CUDA graph per step whose kernels read dt
from device memory, with the CFL reduction and the dt update on the device
(no host read until the last step).  Checks:
- it equals, bit for bit, the driver's host loop through the single-call
  entry points (momentum, apply_bc, pressure_projection, get_cfl) with the
  host's dt, in fields, dt, t_current and cfl; also with IBM forcing and
  with walls in z (the extended-grid FFT path);
- it agrees with the oracle's adaptive loop (oracle steps with the CFL read
  after each) to rounding;
- the red-black path (CFL read on the host every step) follows the same
  rule; cflmax <= 0 is mdx_step with fixed dt.
"""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import random_fields, rel_l2, to_device

CFLMAX, DTMAX, NSTEPS = 0.02, 5e-3, 6


def _case(ibm=False, z_wall=False):
    g = O.Grid(32, 16, 16, lx=2 * np.pi, ly=2.0, lz=np.pi, re=2000.0, dt=1e-3, forcing=(1e-3, 0.0, 0.0))
    bc = O.channel_bc()
    if z_wall:
        bc = O.BC((True, False, False))
        for d in (2, 3):
            bc.set(d, 0, 0, typ=1, value=0.0).set(d, 1, 0, typ=1, value=0.0)
    f = O.Fields(g)
    O.channel_ic(g, f, 11)
    f.us[...] = f.un
    f.vs[...] = f.vn
    f.ws[...] = f.wn
    if ibm:
        O.set_ibm_coeff(g, O.ibm_reference(g), f)
    return g, bc, f


def _host_loop(s, nsteps, cflmax, dtmax, start=None):
    """The driver's loop through the single-call entry points; start =
    (dt, t, cfl) to continue from (default: the context's)."""
    a, b, c = O.rk_coeffs()
    dt, t, cfl = start if start else s.time()
    for _ in range(nsteps):
        t = t + dt
        for q in range(3):
            s.momentum(dt * a[q], dt * b[q], dt * c[q])
            s.apply_bc()
            s.pressure_projection(dt * c[q])
            s.apply_bc()
        cfl = s.get_cfl()
        if cflmax > 0.0 and cfl > 0.0:
            dt = min(cflmax / cfl, dtmax)
    return dt, t, cfl


@pytest.mark.gpu
@pytest.mark.parametrize("ibm,z_wall", [(False, False), (True, False), (False, True)])
def test_device_dt_graph_equals_host_loop(ibm, z_wall):
    g, bc, f = _case(ibm, z_wall)
    with to_device(M, g, bc, f) as sa, to_device(M, g, bc, f) as sb:
        for s in (sa, sb):
            s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        l0 = sa.launch_count()
        sa.step_adaptive(NSTEPS, CFLMAX, DTMAX)
        assert sa.launch_count() > l0
        dta, ta, cfla = sa.time()
        dtb, tb, cflb = _host_loop(sb, NSTEPS, CFLMAX, DTMAX)
        assert (dta, ta, cfla) == (dtb, tb, cflb)
        assert dta < DTMAX and dta != g.dt          # dt followed the CFL
        for n in ("un", "vn", "wn", "pn"):
            assert np.array_equal(sa.get(n), sb.get(n)), n
        # a second call continues from the device's dt and t
        sa.step_adaptive(2, CFLMAX, DTMAX)
        dtb, tb, cflb = _host_loop(sb, 2, CFLMAX, DTMAX, start=(dtb, tb, cflb))
        assert sa.time() == (dtb, tb, cflb)
        assert np.array_equal(sa.get("un"), sb.get("un"))


@pytest.mark.gpu
def test_device_dt_matches_oracle_adaptive_loop():
    g, bc, f = _case()
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.step_adaptive(NSTEPS, CFLMAX, DTMAX)
        dt, t, cfl = s.time()
        got = {n: s.get(n) for n in ("un", "vn", "wn", "pn")}
    odt, ot = g.dt, 0.0
    for _ in range(NSTEPS):
        ot += odt
        O.run(g, bc, f, odt, 1, solver=0)
        ocfl = O.get_cfl(g, f)
        odt = min(CFLMAX / ocfl, DTMAX)
    assert abs(t - ot) <= 1e-12 * ot
    assert abs(dt - odt) <= 1e-10 * odt and abs(cfl - ocfl) <= 1e-10 * ocfl
    for n in got:
        assert rel_l2(got[n], getattr(f, n)) <= 1e-10, (n, rel_l2(got[n], getattr(f, n)))


@pytest.mark.gpu
def test_redblack_adaptive_and_fixed_dt():
    g, bc, f = _case()
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-9, check_every=10, max_iter=100000)
    with to_device(M, g, bc, f) as sa, to_device(M, g, bc, f) as sb, to_device(M, g, bc, f) as sc:
        for s in (sa, sb, sc):
            s.init_pressure_solver(opts)
        sa.step_adaptive(3, CFLMAX, DTMAX)
        dt, t, cfl = sa.time()
        # the same rule, one step at a time through mdx_step with the host's dt
        t2, dt2 = 0.0, g.dt
        for _ in range(3):
            sb.set_dt(dt2)
            sb.step(1)
            t2 += dt2
            c2 = sb.get_cfl()
            dt2 = min(CFLMAX / c2, DTMAX)
        assert (dt, t, cfl) == (dt2, t2, c2)
        assert np.array_equal(sa.get("un"), sb.get("un"))
        # cflmax <= 0: fixed dt
        sc.step_adaptive(2, 0.0, 0.0)
        assert sc.time()[0] == g.dt and sc.time()[1] == 2 * g.dt
