"""Mixed precision on the FFT path: FP32 x-z FFTs and Thomas solves inside
FP64 defect correction, the zero-wavenumber mode in FP64, against the FP64
FFT path and the oracle."""
import math

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, oracle_channel_ic, rel_l2, to_device

pytestmark = pytest.mark.gpu


def _pair(nx=64, ny=32, nz=32, tol=1e-10):
    g, bc = channel_case(nx, ny, nz)
    f = O.Fields(g)
    oracle_channel_ic(g, bc, f, 20261203, solver=0)
    a, b, c = O.rk_coeffs()
    O.momentum(g, bc, f, g.dt * a[0], g.dt * b[0], g.dt * c[0])
    O.apply_bc(g, f)
    s64 = to_device(M, g, bc, f)
    s32 = to_device(M, g, bc, f)
    s64.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
    s32.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT, tol=tol, precision=M.PREC_MIXED))
    return g, f, s64, s32, g.dt * c[0]


@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_fft_mixed_projection_matches_fp64(tol):
    g, f, s64, s32, dg = _pair(tol=tol)
    with s64, s32:
        s64.pressure_projection(dg)
        st = s32.pressure_projection(dg)
        assert st.status == 0 and 200 < st.variant <= 203 and st.iterations == st.variant - 200
        assert st.residual <= tol * 1.0000001 or st.residual * st.residual0 <= st.atol * 1.0000001
        # interiors: from its second pass on the mixed path refreshes ghost
        # cells (apply_bc) that the FP64 projection leaves to the caller
        errs = {n: rel_l2(s32.get(n)[1:-1, 1:-1, 1:-1], s64.get(n)[1:-1, 1:-1, 1:-1]) for n in ("un", "vn", "wn", "pn")}
        print("fft mixed vs fp64", tol, st.iterations, "passes", errs)
        for n in ("un", "vn", "wn"):
            assert errs[n] <= 1e-6, (n, errs)
        assert errs["pn"] <= 1e-5


def test_fft_mixed_channel_steps_vs_oracle():
    """20 RK3 steps of the 64x32x32 channel: velocity within 1e-6 of the FP64 oracle."""
    g, bc = channel_case(64, 32, 32)
    f = O.Fields(g)
    oracle_channel_ic(g, bc, f, 20261203, solver=0)
    s = to_device(M, g, bc, f)
    with s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT, tol=1e-10, precision=M.PREC_MIXED))
        passes = s.step(20)
        st, _ = O.run(g, bc, f, g.dt, 20, solver=0)
        assert st == 0
        assert passes <= 20 * 3 * 3
        for n in ("un", "vn", "wn"):
            assert rel_l2(s.get(n), getattr(f, n)) <= 1e-6, n
        _, linf = s.divergence_norms()
        assert linf <= 1e-9
