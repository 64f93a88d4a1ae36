"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by ``bench.py``'s cpu_baseline / reference arm, as the checker.  The
product (``mobydiff_b200``) never imports it.

Parity status: unpinned (see the header of mdx_oracle.cpp).

Arrays use the reference layout: padded fields ``(0:nx+1,0:ny+1,0:nz+1)`` in
Fortran order are numpy arrays of shape ``(nz+2, ny+2, nx+2)`` in C order;
``oldrhs*`` are ``(nz, ny, nx)``; the FFT workspace ``rhs(nx,nz,ny)`` is
``(ny, nz, nx)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "mdx_oracle.cpp")
    if force or not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


class GridC(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("re", C.c_double),
                ("forcing_x", C.c_double), ("forcing_y", C.c_double), ("forcing_z", C.c_double)]


class BCC(C.Structure):
    _fields_ = [("periodic", C.c_int * 3), ("bc_type", C.c_int * 24), ("bc_value", C.c_double * 24)]


class FieldsC(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("un", "us", "vn", "vs", "wn", "ws", "pn", "oldrhsu", "oldrhsv", "oldrhsw",
                 "coef_u", "coef_v", "coef_w")]


class IbmC(C.Structure):
    _fields_ = [("geometry", C.c_int), ("n_wave_x", C.c_int), ("amp", C.c_double), ("phase", C.c_double),
                ("lambda_", C.c_double), ("y0", C.c_double), ("height", C.c_double)]


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        d = C.c_double
        P = C.POINTER
        L = _LIB
        L.or_momentum.argtypes = [P(GridC), P(BCC), P(FieldsC), d, d, d]
        L.or_apply_bc.argtypes = [P(GridC), P(FieldsC)]
        L.or_apply_bc_redblack.argtypes = [P(GridC), P(BCC), P(FieldsC)]
        L.or_build_fft_rhs.argtypes = [P(GridC), P(FieldsC), d, C.c_void_p]
        L.or_solve_pressure_fft.argtypes = [P(GridC), C.c_void_p]
        L.or_fft2_r2c.argtypes = [P(GridC), C.c_void_p, C.c_void_p]
        L.or_fft2_c2r.argtypes = [P(GridC), C.c_void_p, C.c_void_p]
        L.or_solve_tridiagonal_y.argtypes = [P(GridC), C.c_void_p]
        L.or_fft_correction.argtypes = [P(GridC), P(FieldsC), d, C.c_void_p]
        L.or_pressure_projection_fft.argtypes = [P(GridC), P(FieldsC), d, C.c_void_p]
        L.or_pressure_projection_redblack.argtypes = [P(GridC), P(BCC), P(FieldsC), d, C.c_int, d, d, d,
                                                      C.c_int, C.c_int, C.c_int, P(C.c_int), P(C.c_double)]
        L.or_pressure_projection_redblack.restype = C.c_int
        L.or_sor_sweep.argtypes = [P(GridC), P(BCC), P(FieldsC), d, d, C.c_int]
        L.or_divergence_norms.argtypes = [P(GridC), P(BCC), P(FieldsC), P(d), P(d)]
        L.or_set_ibm_coeff.argtypes = [P(GridC), P(IbmC), C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.or_channel_ic.argtypes = [P(GridC), C.c_uint64, d, d, d, d, d, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_run.argtypes = [P(GridC), P(BCC), P(FieldsC), d, C.c_int, C.c_int, C.c_int, d, d, d, C.c_int,
                             C.c_int, C.c_int, P(C.c_int)]
        L.or_divergence_norms3.argtypes = [P(GridC), P(BCC), P(FieldsC), P(d), P(d), P(d)]
        L.or_run.restype = C.c_int
        L.or_get_cfl.argtypes = [P(GridC), P(FieldsC)]
        L.or_get_cfl.restype = d
        L.or_rk_coeffs.argtypes = [P(d), P(d), P(d)]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
    return _LIB


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Grid:
    """grid_type (src/modules/init.f90:5-12, finalize_grid :38-44)."""

    def __init__(self, nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, re=100.0, dt=1e-4,
                 forcing=(1.0, 0.0, 0.0)):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.lx, self.ly, self.lz = float(lx), float(ly), float(lz)
        self.re, self.dt = float(re), float(dt)
        self.forcing = tuple(float(v) for v in forcing)
        self.dx = self.lx / float(self.nx)
        self.dy = self.ly / float(self.ny)
        self.dz = self.lz / float(self.nz)

    def c(self) -> GridC:
        return GridC(self.nx, self.ny, self.nz, self.lx, self.ly, self.lz, self.dx, self.dy, self.dz,
                     self.re, *self.forcing)

    @property
    def padded(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)

    @property
    def interior(self):
        return (self.nz, self.ny, self.nx)


def bc_index(d: int, side: int, var: int) -> int:
    """Index of bcType(d, side, var) in Fortran memory order (d = 1..3)."""
    return (d - 1) + 3 * (side + 2 * var)


class BC:
    """boundary_type (src/modules/boundary.f90:6-20); defaults of init_bc."""

    def __init__(self, periodic=(True, True, True)):
        self.periodic = [bool(p) for p in periodic]
        self.bc_type = [0] * 24
        self.bc_value = [0.0] * 24

    def set(self, d, side, var, typ=None, value=None):
        if typ is not None:
            self.bc_type[bc_index(d, side, var)] = int(typ)
        if value is not None:
            self.bc_value[bc_index(d, side, var)] = float(value)
        return self

    def c(self) -> BCC:
        b = BCC()
        for t in range(3):
            b.periodic[t] = 1 if self.periodic[t] else 0
        for t in range(24):
            b.bc_type[t] = self.bc_type[t]
            b.bc_value[t] = self.bc_value[t]
        return b


def channel_bc() -> BC:
    """Periodic x/z, walls in y with Neumann pressure (tutorials/wavychannel/input.ini:24-30)."""
    b = BC((True, False, True))
    b.set(2, 0, 0, typ=1)
    b.set(2, 1, 0, typ=1)
    return b


FIELD_NAMES = ("un", "us", "vn", "vs", "wn", "ws", "pn")
RHS_NAMES = ("oldrhsu", "oldrhsv", "oldrhsw")
COEF_NAMES = ("coef_u", "coef_v", "coef_w")


class Fields:
    """field_type (src/modules/init.f90:14-19, zero-initialised :57-70) plus IBM coefficients."""

    def __init__(self, g: Grid):
        self.g = g
        for n in FIELD_NAMES + COEF_NAMES:
            setattr(self, n, np.zeros(g.padded))
        for n in RHS_NAMES:
            setattr(self, n, np.zeros(g.interior))

    def c(self) -> FieldsC:
        return FieldsC(*[_ptr(getattr(self, n)) for n in FIELD_NAMES + RHS_NAMES + COEF_NAMES])

    def copy(self) -> "Fields":
        f = Fields(self.g)
        for n in FIELD_NAMES + RHS_NAMES + COEF_NAMES:
            getattr(f, n)[...] = getattr(self, n)
        return f


def rk_coeffs():
    a = (C.c_double * 3)()
    b = (C.c_double * 3)()
    c = (C.c_double * 3)()
    lib().or_rk_coeffs(a, b, c)
    return list(a), list(b), list(c)


def momentum(g, bc, f, dt_alpha, dt_beta, dt_gamma):
    fc = f.c()
    lib().or_momentum(C.byref(g.c()), C.byref(bc.c()), C.byref(fc), dt_alpha, dt_beta, dt_gamma)


def apply_bc(g, f):
    lib().or_apply_bc(C.byref(g.c()), C.byref(f.c()))


def apply_bc_redblack(g, bc, f):
    lib().or_apply_bc_redblack(C.byref(g.c()), C.byref(bc.c()), C.byref(f.c()))


def build_fft_rhs(g, f, dt_gamma):
    rhs = np.zeros((g.ny, g.nz, g.nx))
    lib().or_build_fft_rhs(C.byref(g.c()), C.byref(f.c()), dt_gamma, rhs.ctypes.data)
    return rhs


def fft2_r2c(g, rhs):
    """rhs (ny,nz,nx) real -> plane_hat (ny,nz,nxh) complex; FFTW forward sign, unnormalised."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    hat = np.zeros((g.ny, g.nz, g.nx // 2 + 1), dtype=np.complex128)
    lib().or_fft2_r2c(C.byref(g.c()), rhs.ctypes.data, hat.ctypes.data)
    return hat


def fft2_c2r(g, hat):
    hat = np.array(hat, dtype=np.complex128, order="C", copy=True)
    out = np.zeros((g.ny, g.nz, g.nx))
    lib().or_fft2_c2r(C.byref(g.c()), hat.ctypes.data, out.ctypes.data)
    return out


def solve_pressure_fft(g, rhs):
    phi = np.array(rhs, dtype=np.float64, order="C", copy=True)
    lib().or_solve_pressure_fft(C.byref(g.c()), phi.ctypes.data)
    return phi


def pressure_projection_fft(g, f, dt_gamma):
    phi = np.zeros((g.ny, g.nz, g.nx))
    lib().or_pressure_projection_fft(C.byref(g.c()), C.byref(f.c()), dt_gamma, phi.ctypes.data)
    return phi


def pressure_projection_redblack(g, bc, f, dt_gamma, niter=3, sor=1.5, tol=0.0, max_iter=100000,
                                 check_every=10, parallel=True, atol=-1.0):
    it = C.c_int(0)
    res = C.c_double(0.0)
    st = lib().or_pressure_projection_redblack(C.byref(g.c()), C.byref(bc.c()), C.byref(f.c()), dt_gamma,
                                               niter, sor, tol, atol, max_iter, check_every, 1 if parallel else 0,
                                               C.byref(it), C.byref(res))
    return st, it.value, res.value


def sor_sweep(g, bc, f, dt_gamma, sor, parity):
    lib().or_sor_sweep(C.byref(g.c()), C.byref(bc.c()), C.byref(f.c()), dt_gamma, sor, parity)


def divergence_norms(g, bc, f):
    l2 = C.c_double(0.0)
    li = C.c_double(0.0)
    lib().or_divergence_norms(C.byref(g.c()), C.byref(bc.c()), C.byref(f.c()), C.byref(l2), C.byref(li))
    return l2.value, li.value


def get_cfl(g, f):
    return lib().or_get_cfl(C.byref(g.c()), C.byref(f.c()))


def ibm_reference(g: Grid) -> IbmC:
    """The reference's hard-coded geometry, src/modules/ibm.f90:45-50."""
    return IbmC(0, 1, 5 * g.dy, 0.0, 0.0, 0.0, 0.0)


def ibm_wavy(amp, lam, y0, height=2.0, phase=0.0) -> IbmC:
    return IbmC(1, 1, float(amp), float(phase), float(lam), float(y0), float(height))


def set_ibm_coeff(g, ibm: IbmC, f: Fields):
    """set_ibm_coeff for u, v and w (src/main.f90:57-60)."""
    for name, d in (("coef_u", (1, 0, 0)), ("coef_v", (0, 1, 0)), ("coef_w", (0, 0, 1))):
        arr = getattr(f, name)
        lib().or_set_ibm_coeff(C.byref(g.c()), C.byref(ibm), arr.ctypes.data, *d)


def channel_ic(g, f, seed, amp_u=0.1, amp_vw=0.01, y0=0.0, wave_amp=0.0, wave_lambda=1.0):
    lib().or_channel_ic(C.byref(g.c()), seed, amp_u, amp_vw, y0, wave_amp, wave_lambda,
                        f.un.ctypes.data, f.vn.ctypes.data, f.wn.ctypes.data)


def run(g, bc, f, dt, nsteps, solver=0, niter=3, sor=1.5, tol=0.0, max_iter=100000, check_every=10,
        parallel=True, atol=-1.0):
    tot = C.c_int(0)
    st = lib().or_run(C.byref(g.c()), C.byref(bc.c()), C.byref(f.c()), dt, nsteps, solver, niter, sor, tol, atol,
                      max_iter, check_every, 1 if parallel else 0, C.byref(tot))
    return st, tot.value


def set_threads(n: int):
    lib().or_set_threads(int(n))


def get_threads() -> int:
    return lib().or_get_threads()
