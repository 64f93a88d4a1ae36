"""The allocation-free pressure solve (mdx_solve_pressure_fft_noalloc).

Some callers cannot allocate device memory through the CUDA runtime: an
OpenMP-offload Fortran program, for instance, owns its device arrays through
the OpenMP runtime and hands their addresses to libraries (the reference
passes them to cuFFT with use_device_addr).  For them the library offers one
entry point that takes the caller's device arrays and keeps its own
intermediates in a fixed static array instead of cudaMalloc'd memory.

This test calls it through the C ABI twice in a row, on two different grids
and right-hand sides, and checks each result against the pressure correction
of the regular entry point (mdx_pressure_projection on a context) for the
same right-hand side, within the 1e-12 relative tolerance of the FFT-path
tests.  A second test solves in place (phi and rhs the same array) and then a
grid of another size on a fresh non-default stream, so each call must rebuild
every part of the shared scratch it reads.  It lives in a file of its own that
pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, random_fields, rel_l2, to_device


def _regular_phi(shape, seed, dg):
    """Right-hand side div(u*)/dt_gamma and phi from the context entry point."""
    g, bc = channel_case(*shape)
    f = random_fields(g, seed, scale=0.5)
    O.apply_bc(g, f)
    rhs = O.build_fft_rhs(g, f, dg)            # rhs(nx,nz,ny) as (ny,nz,nx), same divergence arithmetic
    with to_device(M, g, bc, f) as s:
        s.init_pressure_solver(M.make_solver_opts(M.SOLVER_FFT))
        s.apply_bc()
        s.pressure_projection(dg)
        phi = s.get("phi")
    return g, rhs, phi


@pytest.mark.gpu
def test_noalloc_solve_matches_regular_entry_point():
    import torch

    L = M.lib()
    fn = L.mdx_solve_pressure_fft_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_void_p]
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    for shape, seed, dg in (((32, 16, 24), 41, 0.4e-3), ((48, 20, 16), 42, 0.7e-3)):
        g, rhs, phi_ref = _regular_phi(shape, seed, dg)
        # the caller's device arrays (allocated by the caller, not by the library)
        d_rhs = torch.from_numpy(rhs).to("cuda")
        d_phi = torch.full_like(d_rhs, float("nan"))
        rc = fn(d_rhs.data_ptr(), d_phi.data_ptr(), g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, stream.cuda_stream)
        assert rc == M.MDX_OK, L.mdx_last_error(None).decode()
        torch.cuda.synchronize()
        phi = d_phi.cpu().numpy()
        assert np.all(np.isfinite(phi))
        assert rel_l2(phi, phi_ref) <= 1e-12


def _fn():
    fn = M.lib().mdx_solve_pressure_fft_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_void_p]
    return fn


@pytest.mark.gpu
def test_noalloc_in_place_then_other_grid_on_new_stream():
    import torch

    fn = _fn()
    torch.cuda.set_device(0)
    cases = (((40, 12, 30), 43, 0.5e-3, None), ((24, 18, 40), 44, 0.3e-3, torch.cuda.Stream()))
    for shape, seed, dg, stream in cases:
        g, rhs, phi_ref = _regular_phi(shape, seed, dg)
        d = torch.from_numpy(rhs).to("cuda")
        sp = (stream or torch.cuda.current_stream()).cuda_stream
        if stream is not None:
            stream.wait_stream(torch.cuda.current_stream())
        rc = fn(d.data_ptr(), d.data_ptr(), g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, sp)   # phi = rhs, in place
        assert rc == M.MDX_OK, M.lib().mdx_last_error(None).decode()
        torch.cuda.synchronize()
        assert rel_l2(d.cpu().numpy(), phi_ref) <= 1e-12, shape


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Runs without a GPU: the size check comes before any device call."""
    L = M.lib()
    fn = L.mdx_solve_pressure_fft_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_void_p]
    # 256^3 needs ~0.2 GB of intermediates; the static array is 8 MiB.  The
    # size check comes before any device work, so the pointers are never used.
    rc = fn(C.c_void_p(16), C.c_void_p(16), 256, 256, 256, 0.1, 0.1, 0.1, None)
    assert rc == M.MDX_ERR_ARG
    assert "scratch" in L.mdx_last_error(None).decode()
