"""Warp-shuffle x and z transforms of the FFT path (lengths 32 P, P = 1..16)
against the oracle's projection (pressure_solver.f90:58-61 with the FFTW
transforms) and against the shared-memory Stockham transforms on the same
inputs, FP64 and the FP32 inner solve of the mixed path."""
import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, random_fields, rel_l2, to_device

pytestmark = pytest.mark.gpu

# (nx, ny, nz): nx/2 and nz in 32 * {1, 2, 4, 8, 16}, one side Stockham in the last two
SHAPES = [(64, 5, 32), (128, 8, 128), (256, 6, 64), (512, 8, 256), (1024, 4, 512), (96, 4, 128), (256, 4, 40)]


def _project(g, bc, f, fft_kernel, precision=M.PREC_FP64, dg=0.4e-3):
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT, precision=precision, fft_kernel=fft_kernel,
                                                  tol=1e-10 if precision == M.PREC_MIXED else 0.0))
        s.apply_bc()
        s.pressure_projection(dg)
        return {n: s.get(n) for n in ("phi", "un", "vn", "wn", "pn")}


@pytest.mark.parametrize("shape", SHAPES)
def test_warp_transforms_match_oracle_and_stockham(shape):
    g, bc = channel_case(*shape)
    f = random_fields(g, 31, scale=0.5)
    warp = _project(g, bc, f, 0)
    stock = _project(g, bc, f, 1)
    O.apply_bc(g, f)
    phi_o = O.pressure_projection_fft(g, f, 0.4e-3)
    assert rel_l2(warp["phi"], phi_o) < 1e-12
    assert rel_l2(warp["phi"], stock["phi"]) < 1e-13
    for n in ("un", "vn", "wn", "pn"):
        assert rel_l2(warp[n], getattr(f, n)) < 1e-12, n
        assert rel_l2(warp[n], stock[n]) < 1e-13, n


@pytest.mark.parametrize("shape", [(128, 8, 128), (512, 8, 256), (1024, 4, 512)])
def test_warp_transforms_mixed_precision(shape):
    """FP32 warp transforms inside FP64 defect correction reach the FP64
    projection like the FP32 Stockham transforms do."""
    g, bc = channel_case(*shape)
    f = random_fields(g, 32, scale=0.5)
    ref = _project(g, bc, f, 0)
    errs = {}
    for k in (0, 1):
        out = _project(g, bc, f, k, precision=M.PREC_MIXED)
        errs[k] = {n: rel_l2(out[n][1:-1, 1:-1, 1:-1], ref[n][1:-1, 1:-1, 1:-1]) for n in ("un", "vn", "wn")}
    print("mixed vs fp64 (warp, stockham)", errs)
    for n in ("un", "vn", "wn"):
        assert errs[0][n] <= 1e-6, (n, errs)
        assert errs[0][n] <= 10 * errs[1][n] + 1e-9, (n, errs)

