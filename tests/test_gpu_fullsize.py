"""Parity of the plain FP64 step against the oracle at the configurations'
full sizes (slow: the oracle runs a whole step on the host cores).

- Wavy-wall IBM channel, 256x128x128, Re 3000, dt 1e-3, red-black SOR
  omega 1.7 to residual 1e-10 (src/modules/step.f90:27-207,
  src/modules/pressure/pressure_redblack.f90:27-254, src/main.f90:66-90).
  The sweeps follow the reference's arithmetic operation by operation on
  both sides, so the residual checks stop at the same iteration and u, v,
  w, p agree bit for bit; the test asserts equal iteration counts and the
  north star's rel-L2 <= 1e-11.
- Channel 512x256x256 (Lx 4 pi, Lz 2 pi), Re 5000, dt 1e-3, FFT + Thomas
  FP64 (src/modules/pressure/pressure_fft.f90:102-148,
  src/modules/pressure_solver.f90:77-173): the transforms are different
  algorithms, so the bar is rel-L2 <= 1e-11 on u, v, w, p and
  max|div u| <= 1e-12 after two steps from the same projected start.
"""
import math
import time

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import oracle_channel_ic, rel_l2, to_device

pytestmark = pytest.mark.gpu

SEED = 20261203


def _report(name, d):
    print(f"\n[{name}] " + ", ".join(f"{k}={v}" for k, v in d.items()), flush=True)


def test_c1_full_size_redblack_step():
    """One RK3 step of the 256x128x128 wavy channel at residual 1e-10: equal
    iteration counts in all three projections, identical fields."""
    ly = 2.25
    y0 = (ly - 2.0) / 2.0
    g = O.Grid(256, 128, 128, lx=2 * math.pi, ly=ly, lz=math.pi, re=3000.0, dt=1e-3,
               forcing=(2.0 / 3000.0, 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_wavy(0.05, g.lx / 2, y0), f)
    opts = M.make_solver_opts(M.SOLVER_REDBLACK, sor=1.7, tol=1e-10, check_every=50, max_iter=400000,
                              adaptive_checks=False)
    s = to_device(M, g, bc, O.Fields(g))
    with s:
        s.enter_ibm_data(f.coef_u, f.coef_v, f.coef_w)
        s.init_pressure_solver(opts)
        # the seeded start projected at t = 0 on the device; the oracle starts
        # from the same arrays
        s.channel_ic(SEED, y0=y0, wave_amp=0.05, wave_lambda=g.lx / 2)
        for n in O.FIELD_NAMES + O.RHS_NAMES:
            getattr(f, n)[...] = s.get(n)
        t0 = time.perf_counter()
        st, it_o = O.run(g, bc, f, g.dt, 1, solver=1, sor=1.7, tol=1e-10, check_every=50)
        t_cpu = time.perf_counter() - t0
        it_g = s.step(1)
        errs = {n: rel_l2(s.get(n), getattr(f, n)) for n in ("un", "vn", "wn", "pn")}
        maxabs = {n: float(np.max(np.abs(s.get(n) - getattr(f, n)))) for n in ("un", "vn", "wn", "pn")}
        l2, linf = s.divergence_norms()
    _report("c1 256x128x128 1 step tol 1e-10",
            dict(iters_gpu=it_g, iters_oracle=it_o, oracle_s=round(t_cpu, 1), threads=O.get_threads(),
                 rel_l2=errs, max_abs=maxabs, div_l2=l2, div_linf=linf))
    assert st == 0
    assert it_g == it_o
    assert all(e <= 1e-11 for e in errs.values()), errs


def test_c2_full_size_fft_steps():
    """Two RK3 steps of the 512x256x256 channel on the FP64 FFT path."""
    g = O.Grid(512, 256, 256, lx=4 * math.pi, ly=2.0, lz=2 * math.pi, re=5000.0, dt=1e-3,
               forcing=(2.0 / 5000.0, 0.0, 0.0))
    bc = O.channel_bc()
    f = O.Fields(g)
    t0 = time.perf_counter()
    oracle_channel_ic(g, bc, f, SEED)
    s = to_device(M, g, bc, O.Fields(g))
    with s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.channel_ic(SEED)
        ic = {n: rel_l2(s.get(n), getattr(f, n)) for n in ("un", "vn", "wn")}
        O.run(g, bc, f, g.dt, 2, solver=0)
        t_cpu = time.perf_counter() - t0
        s.step(2)
        errs = {n: rel_l2(s.get(n), getattr(f, n)) for n in ("un", "vn", "wn", "pn")}
        l2, linf = s.divergence_norms()
        l2_o, linf_o = O.divergence_norms(g, bc, f)
    _report("c2 512x256x256 2 steps FFT",
            dict(ic_rel_l2=ic, rel_l2=errs, div_linf=linf, div_linf_oracle=linf_o, div_l2=l2,
                 oracle_s=round(t_cpu, 1), threads=O.get_threads()))
    assert all(e <= 1e-13 for e in ic.values()), ic
    assert all(e <= 1e-11 for e in errs.values()), errs
    assert linf <= 1e-12, linf
