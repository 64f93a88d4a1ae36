"""mobydiff_b200 -- sm_100a implementation of the mobydiff RK3 time step.

The compute lives in ``libmobyb200.so`` (CUDA, built in-tree by
``mobydiff_b200.build``) behind the C ABI of ``include/mobydiff_b200.h``.
This package is the Python-side mirror of the reference's Fortran modules
for that path, calling the C ABI through ctypes:

=======================  ==============================================
reference (Fortran)      here
=======================  ==============================================
init_openmp_offload      device_count()
enter/exit_field_data    Solver.enter_field_data / exit_field_data
enter/exit_ibm_data      Solver.enter_ibm_data / exit_ibm_data
momentum                 Solver.momentum
apply_bc(_redblack)      Solver.apply_bc / apply_bc_redblack
init_pressure_solver     Solver.init_pressure_solver
pressure_projection      Solver.pressure_projection
get_cfl                  Solver.get_cfl
center_vel               Solver.center_vel
read_runtime_config      read_runtime_config
set_ibm_coeff            set_ibm_coeff
=======================  ==============================================

There is no CPU fallback: every compute call goes to the CUDA library and
raises ``MdxError`` when the library or a device is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmobyb200.so")

MDX_OK = 0
MDX_ERR_ARG = 1
MDX_ERR_CUDA = 2
MDX_ERR_NO_DEVICE = 3
MDX_ERR_STATE = 4
MDX_NOT_CONVERGED = 5
MDX_ERR_NONFINITE = 6
MDX_ERR_IO = 7
MDX_ERR_TIMEOUT = 8

SOLVER_FFT = 0
SOLVER_REDBLACK = 1
PREC_FP64 = 0
PREC_MIXED = 1
GUESS_ZERO = 0
GUESS_PREVIOUS = 1
GUESS_LEARNED = 2
UNET_INPUTS = 5            # input channels of the warm-start network (mdx_unet_loss_grad)
GUESS_EXTRAPOLATED = 3

FIELDS = ["un", "us", "vn", "vs", "wn", "ws", "pn", "oldrhsu", "oldrhsv", "oldrhsw",
          "coef_u", "coef_v", "coef_w", "phi"]
FIELD_ID = {n: t for t, n in enumerate(FIELDS)}
TIMER_CLASSES = ["momentum", "bc", "fft_fwd", "thomas", "fft_inv", "correct", "sor_sweep", "residual", "other",
                 "sor_run"]


class MdxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mdx error {code}: {msg}")
        self.code = code


class GridT(C.Structure):
    """grid_type, src/modules/init.f90:5-12."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nsteps", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("re", C.c_double), ("dt", C.c_double), ("t_final", C.c_double), ("t_current", C.c_double),
                ("cfl", C.c_double), ("cflmax", C.c_double), ("dtmax", C.c_double),
                ("forcing_x", C.c_double), ("forcing_y", C.c_double), ("forcing_z", C.c_double)]


class BcT(C.Structure):
    """boundary_type, src/modules/boundary.f90:6-10 (bcType in Fortran memory order)."""
    _fields_ = [("is_periodic", C.c_int * 3), ("bc_type", C.c_int * 24), ("bc_value", C.c_double * 24)]


class SolverOptsT(C.Structure):
    _fields_ = [("solver", C.c_int), ("n_iter", C.c_int), ("sor", C.c_double), ("tol", C.c_double),
                ("max_iter", C.c_int), ("check_every", C.c_int), ("precision", C.c_int),
                ("sor_variant", C.c_int), ("sor_kz", C.c_int), ("check_mode", C.c_int),
                ("fft_kernel", C.c_int), ("inner_form", C.c_int), ("reserved_i", C.c_int * 2),
                ("atol", C.c_double), ("inner_sor", C.c_double), ("reserved_d", C.c_double * 6)]


class SolveStatsT(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("residual", C.c_double), ("residual0", C.c_double),
                ("atol", C.c_double), ("variant", C.c_int), ("guessed", C.c_int)]


class UnetOptsT(C.Structure):
    _fields_ = [("channels0", C.c_int), ("channels", C.c_int), ("extra_bottleneck", C.c_int), ("capacity", C.c_int),
                ("slope", C.c_double), ("seed", C.c_uint64), ("conv_kernel", C.c_int), ("step_rule", C.c_int),
                ("gate_period", C.c_int), ("reserved_i", C.c_int * 5),
                ("reserved_d", C.c_double * 8)]


class UnetStatsT(C.Structure):
    _fields_ = [("corrections", C.c_longlong), ("rejected", C.c_longlong), ("snapshots", C.c_longlong),
                ("stored", C.c_int), ("trained", C.c_int), ("out_scale", C.c_double), ("last_gain", C.c_double),
                ("infer_ms", C.c_double), ("train_ms", C.c_double), ("tc_convs", C.c_longlong),
                ("last_step", C.c_double), ("gated", C.c_longlong),
                ("reserved_d", C.c_double * 3)]


class MemberT(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("lx", C.c_double), ("ly", C.c_double),
                ("lz", C.c_double), ("re", C.c_double), ("dt", C.c_double), ("amp", C.c_double), ("seed", C.c_uint64),
                ("reserved_i", C.c_int * 4), ("reserved_d", C.c_double * 4)]


class TimingT(C.Structure):
    _fields_ = [("ms", C.c_double * 10), ("launches", C.c_longlong * 10)]


class RunConfigT(C.Structure):
    _fields_ = [("output_interval", C.c_int), ("field_interval", C.c_int),
                ("output_prefix", C.c_char * 256), ("field_prefix", C.c_char * 256),
                ("ic", C.c_int), ("seed", C.c_uint64), ("ibm", C.c_int),
                ("ibm_amp", C.c_double), ("ibm_lambda", C.c_double), ("ibm_y0", C.c_double),
                ("ibm_height", C.c_double), ("warnings", C.c_int), ("guess", C.c_int)]


class IbmGeomT(C.Structure):
    _fields_ = [("geometry", C.c_int), ("n_wave_x", C.c_int), ("amp", C.c_double), ("phase", C.c_double),
                ("lambda_", C.c_double), ("y0", C.c_double), ("height", C.c_double)]


_lib = None


def lib():
    """Load libmobyb200.so (built by ``python -m mobydiff_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MdxError(MDX_ERR_STATE, f"{LIB_PATH} is missing: run `python -m mobydiff_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    d = C.c_double
    vp = C.c_void_p
    i = C.c_int
    sig = {
        "mdx_version": (C.c_char_p, []),
        "mdx_device_count": (i, [P(i)]),
        "mdx_last_error": (C.c_char_p, [vp]),
        "mdx_default_grid": (None, [P(GridT)]),
        "mdx_default_bc": (None, [P(BcT)]),
        "mdx_default_solver_opts": (None, [P(SolverOptsT)]),
        "mdx_finalize_grid": (None, [P(GridT)]),
        "mdx_read_runtime_config": (i, [C.c_char_p, P(GridT), P(BcT), P(SolverOptsT), P(RunConfigT)]),
        "mdx_set_ibm_coeff": (i, [P(GridT), P(IbmGeomT), vp, i, i, i]),
        "mdx_create": (i, [i, P(GridT), P(BcT), P(vp)]),
        "mdx_destroy": (i, [vp]),
        "mdx_set_stream": (i, [vp, vp]),
        "mdx_get_stream": (i, [vp, P(vp)]),
        "mdx_enter_field_data": (i, [vp] + [vp] * 10),
        "mdx_exit_field_data": (i, [vp]),
        "mdx_update_host": (i, [vp, vp, vp, vp, vp]),
        "mdx_update_device": (i, [vp, vp, vp, vp, vp]),
        "mdx_copy_field": (i, [vp, i, vp, i]),
        "mdx_enter_ibm_data": (i, [vp, vp, vp, vp]),
        "mdx_set_flow": (i, [vp, d, d, d, d]),
        "mdx_enter_ibm_geometry": (i, [vp, P(IbmGeomT)]),
        "fdm_h5_write_field": (i, [C.c_char_p, i, i, i] + [d] * 9 + [vp] * 4),
        "fdm_h5_read_field": (i, [C.c_char_p, i, i, i] + [vp] * 4),
        "mdx_h5_read_header": (i, [C.c_char_p, P(i), P(d)]),
        "mdx_h5_last_error": (C.c_char_p, []),
        "mdx_write_field_h5": (i, [vp, C.c_char_p]),
        "mdx_read_field_h5": (i, [vp, C.c_char_p]),
        "mdx_set_ibm_coeff_device": (i, [P(GridT), P(IbmGeomT), vp, i, i, i, vp]),
        "mdx_exit_ibm_data": (i, [vp]),
        "mdx_momentum": (i, [vp, d, d, d]),
        "mdx_apply_bc": (i, [vp]),
        "mdx_apply_bc_redblack": (i, [vp]),
        "mdx_init_pressure_solver": (i, [vp, P(SolverOptsT)]),
        "mdx_destroy_pressure_solver": (i, [vp]),
        "mdx_pressure_projection": (i, [vp, d, P(SolveStatsT)]),
        "mdx_get_cfl": (i, [vp, P(d)]),
        "mdx_center_vel": (i, [vp, vp, vp, vp]),
        "mdx_step": (i, [vp, i, P(C.c_longlong)]),
        "mdx_step_adaptive": (i, [vp, i, d, d, P(C.c_longlong)]),
        "mdx_get_time": (i, [vp, P(d), P(d), P(d)]),
        "mdx_set_dt": (i, [vp, d]),
        "mdx_channel_ic": (i, [vp, C.c_uint64, d, d, d, d, d, P(SolveStatsT)]),
        "mdx_divergence_norms": (i, [vp, P(d), P(d)]),
        "mdx_set_timing": (i, [vp, i]),
        "mdx_get_timing": (i, [vp, P(TimingT)]),
        "mdx_launch_count": (C.c_longlong, [vp]),
        "mdx_last_solve_stats": (i, [vp, P(SolveStatsT)]),
        "mdx_set_pressure_guess": (i, [vp, i, i]),
        "mdx_get_increment": (i, [vp, i, vp]),
        "mdx_warm_checkpoint": (i, [vp, i]),
        "mdx_default_member": (None, [P(MemberT)]),
        "mdx_ensemble_create": (i, [i, i, P(MemberT), P(SolverOptsT), P(vp)]),
        "mdx_ensemble_destroy": (i, [vp]),
        "mdx_ensemble_last_error": (C.c_char_p, [vp]),
        "mdx_ensemble_set_guess": (i, [vp, i]),
        "mdx_ensemble_ic": (i, [vp]),
        "mdx_ensemble_step": (i, [vp, i, P(C.c_longlong)]),
        "mdx_ensemble_member_stats": (i, [vp, i, P(SolveStatsT), P(C.c_longlong)]),
        "mdx_ensemble_get": (i, [vp, i, i, vp]),
        "mdx_ensemble_set": (i, [vp, i, i, vp]),
        "mdx_ensemble_config": (i, [vp, i, i, i]),
        "mdx_ensemble_tune": (i, [vp, C.c_char_p, P(i), P(i), P(i), P(d)]),
        "mdx_ensemble_use_graph": (i, [vp, i]),
        "mdx_ensemble_info": (i, [vp, P(i), P(i), P(i), P(i), P(d), P(C.c_longlong)]),
        "mdx_ensemble_unet_load": (i, [vp, P(UnetOptsT), P(C.c_float), C.c_longlong, d]),
        "mdx_ensemble_unet_stats": (i, [vp, P(C.c_longlong), P(C.c_longlong), P(C.c_longlong)]),
        "mdx_default_unet_opts": (None, [P(UnetOptsT)]),
        "mdx_unet_create": (i, [vp, P(UnetOptsT)]),
        "mdx_unet_destroy": (i, [vp]),
        "mdx_unet_record": (i, [vp, i]),
        "mdx_unet_train": (i, [vp, i, d, P(d), P(d)]),
        "mdx_unet_param_count": (C.c_longlong, [vp]),
        "mdx_unet_get_params": (i, [vp, vp, C.c_longlong]),
        "mdx_unet_set_params": (i, [vp, vp, C.c_longlong]),
        "mdx_unet_get_out_scale": (i, [vp, P(d)]),
        "mdx_unet_set_out_scale": (i, [vp, d]),
        "mdx_unet_loss_grad": (i, [vp, vp, vp, P(d), vp, vp]),
        "mdx_unet_stats": (i, [vp, P(UnetStatsT)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def version() -> str:
    return lib().mdx_version().decode()


def device_count() -> int:
    n = C.c_int(0)
    lib().mdx_device_count(C.byref(n))
    return n.value


def _check(rc: int, ctx=None):
    if rc != MDX_OK:
        msg = lib().mdx_last_error(ctx).decode(errors="replace")
        raise MdxError(rc, msg)


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous, "need C-contiguous float64"
    return a.ctypes.data


# ---- reference-default structures -------------------------------------------
def make_grid(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, re=100.0, dt=1e-4, forcing=(1.0, 0.0, 0.0), nsteps=1) -> GridT:
    g = GridT()
    lib().mdx_default_grid(C.byref(g))
    g.nx, g.ny, g.nz, g.nsteps = int(nx), int(ny), int(nz), int(nsteps)
    g.lx, g.ly, g.lz, g.re, g.dt = float(lx), float(ly), float(lz), float(re), float(dt)
    g.forcing_x, g.forcing_y, g.forcing_z = (float(v) for v in forcing)
    lib().mdx_finalize_grid(C.byref(g))
    return g


def make_bc(periodic=(True, True, True), types=None, values=None) -> BcT:
    """types/values: dict {(dir, side, var): int/float}, dir 1..3, side 0/1, var p,u,v,w = 0..3."""
    b = BcT()
    lib().mdx_default_bc(C.byref(b))
    for t in range(3):
        b.is_periodic[t] = 1 if periodic[t] else 0
    for (dd, s, v), val in (types or {}).items():
        b.bc_type[(dd - 1) + 3 * (s + 2 * v)] = int(val)
    for (dd, s, v), val in (values or {}).items():
        b.bc_value[(dd - 1) + 3 * (s + 2 * v)] = float(val)
    return b


def channel_bc() -> BcT:
    """Periodic x/z, walls in y, Neumann pressure (tutorials/wavychannel/input.ini:24-30)."""
    return make_bc((True, False, True), types={(2, 0, 0): 1, (2, 1, 0): 1})


def make_solver_opts(solver=SOLVER_FFT, n_iter=3, sor=1.5, tol=0.0, max_iter=100000, check_every=10,
                     precision=PREC_FP64, atol=-1.0, sor_variant=0, sor_kz=0, inner_sor=0.0,
                     adaptive_checks=True, fft_kernel=0, inner_form=0) -> SolverOptsT:
    o = SolverOptsT()
    lib().mdx_default_solver_opts(C.byref(o))
    o.solver, o.n_iter, o.sor, o.tol = int(solver), int(n_iter), float(sor), float(tol)
    o.max_iter, o.check_every, o.precision = int(max_iter), int(check_every), int(precision)
    o.atol = float(atol)
    o.sor_variant, o.sor_kz = int(sor_variant), int(sor_kz)
    o.inner_sor = float(inner_sor)
    o.check_mode = 0 if adaptive_checks else 1
    o.fft_kernel = int(fft_kernel)
    o.inner_form = int(inner_form)
    return o


def read_runtime_config(path: str):
    """read_runtime_config (src/modules/config.f90:10-75) -> (grid, bc, opts, run)."""
    g = GridT()
    b = BcT()
    o = SolverOptsT()
    r = RunConfigT()
    lib().mdx_default_grid(C.byref(g))
    lib().mdx_default_bc(C.byref(b))
    lib().mdx_default_solver_opts(C.byref(o))
    _check(lib().mdx_read_runtime_config(path.encode(), C.byref(g), C.byref(b), C.byref(o), C.byref(r)))
    return g, b, o, r


def ibm_reference(g: GridT) -> IbmGeomT:
    """The reference's hard-coded lower-wall sinusoid, src/modules/ibm.f90:45-50."""
    return IbmGeomT(0, 1, 5 * g.dy, 0.0, 0.0, 0.0, 0.0)


def ibm_wavy(amp, lam, y0, height=2.0, phase=0.0) -> IbmGeomT:
    return IbmGeomT(1, 1, float(amp), float(phase), float(lam), float(y0), float(height))


def set_ibm_coeff(g: GridT, geom: IbmGeomT):
    """set_ibm_coeff for u, v, w (src/main.f90:57-60) -> (coef_u, coef_v, coef_w)."""
    out = []
    for dd in ((1, 0, 0), (0, 1, 0), (0, 0, 1)):
        a = np.zeros((g.nz + 2, g.ny + 2, g.nx + 2))
        _check(lib().mdx_set_ibm_coeff(C.byref(g), C.byref(geom), a.ctypes.data, *dd))
        out.append(a)
    return tuple(out)


H5_ATTRS = ("lx", "ly", "lz", "dx", "dy", "dz", "re", "dt", "t_current")


def h5_write_field(path: str, g: GridT, un, vn, wn, pn, t_current=None) -> None:
    """fdm_h5_write_field (src/modules/field_hdf5.c:149-184): padded arrays
    (any shape holding (nx+2)(ny+2)(nz+2) values in Fortran order)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (un, vn, wn, pn)]
    n = (g.nx + 2) * (g.ny + 2) * (g.nz + 2)
    if any(a.size != n for a in arrs):
        raise MdxError(MDX_ERR_ARG, "h5_write_field: arrays must hold (nx+2)(ny+2)(nz+2) values")
    t = g.t_current if t_current is None else t_current
    rc = lib().fdm_h5_write_field(os.fsencode(path), g.nx, g.ny, g.nz, g.lx, g.ly, g.lz, g.dx, g.dy, g.dz, g.re,
                                  g.dt, t, *[a.ctypes.data for a in arrs])
    if rc != 0:
        raise MdxError(MDX_ERR_IO, f"could not write HDF5 field file: {path}")


def h5_read_field(path: str, nx: int, ny: int, nz: int):
    """fdm_h5_read_field (src/modules/field_hdf5.c:186-204) -> (un, vn, wn, pn),
    padded arrays indexed [k, j, i]."""
    arrs = [np.empty((nz + 2, ny + 2, nx + 2)) for _ in range(4)]
    if lib().fdm_h5_read_field(os.fsencode(path), nx, ny, nz, *[a.ctypes.data for a in arrs]) != 0:
        raise MdxError(MDX_ERR_IO, lib().mdx_h5_last_error().decode())
    return tuple(arrs)


def h5_read_header(path: str) -> dict:
    """Root attributes of a field file: nx, ny, nz and lx .. t_current."""
    dims = (C.c_int * 3)()
    vals = (C.c_double * 9)()
    rc = lib().mdx_h5_read_header(os.fsencode(path), dims, vals)
    if rc != MDX_OK:
        raise MdxError(rc, lib().mdx_h5_last_error().decode())
    out = {"nx": dims[0], "ny": dims[1], "nz": dims[2]}
    out.update({k: vals[t] for t, k in enumerate(H5_ATTRS)})
    return out


def rk_coeffs():
    """src/modules/step.f90:21-23."""
    return ([64.0 / 120.0, 50.0 / 120.0, 90.0 / 120.0],
            [0.0, -34.0 / 120.0, -50.0 / 120.0],
            [64.0 / 120.0, 16.0 / 120.0, 40.0 / 120.0])


class Solver:
    """One device context: the field mirrors, IBM coefficients and pressure solver."""

    def __init__(self, grid: GridT, bc: BcT, device: int = 0):
        self.grid = grid
        self.bc = bc
        h = C.c_void_p()
        _check(lib().mdx_create(int(device), C.byref(grid), C.byref(bc), C.byref(h)))
        self.h = h

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            lib().mdx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        _check(rc, self.h)

    @property
    def padded(self):
        g = self.grid
        return (g.nz + 2, g.ny + 2, g.nx + 2)

    @property
    def interior(self):
        g = self.grid
        return (g.nz, g.ny, g.nx)

    # -- data residency (gpu_runtime.f90, ibm.f90, io.f90)
    def enter_field_data(self, un=None, us=None, oldrhsu=None, vn=None, vs=None, oldrhsv=None, wn=None, ws=None,
                         oldrhsw=None, pn=None):
        self._c(lib().mdx_enter_field_data(self.h, _p(un), _p(us), _p(oldrhsu), _p(vn), _p(vs), _p(oldrhsv),
                                           _p(wn), _p(ws), _p(oldrhsw), _p(pn)))

    def exit_field_data(self):
        self._c(lib().mdx_exit_field_data(self.h))

    def enter_ibm_data(self, coef_u=None, coef_v=None, coef_w=None):
        self._c(lib().mdx_enter_ibm_data(self.h, _p(coef_u), _p(coef_v), _p(coef_w)))

    def write_field_h5(self, path: str) -> None:
        """write_field (src/modules/io.f90:105-137) from the device mirrors."""
        self._c(lib().mdx_write_field_h5(self.h, os.fsencode(path)))

    def read_field_h5(self, path: str) -> None:
        """read_field (src/modules/io.f90:139-166) into the device mirrors."""
        self._c(lib().mdx_read_field_h5(self.h, os.fsencode(path)))

    def set_flow(self, re: float, forcing=(None, 0.0, 0.0)):
        """Re and body force of this context (default forcing_x = 2/Re, the
        force that keeps the Poiseuille profile steady)."""
        fx = 2.0 / re if forcing[0] is None else forcing[0]
        self._c(lib().mdx_set_flow(self.h, float(re), float(fx), float(forcing[1]), float(forcing[2])))
        self.grid.re = float(re)
        self.grid.forcing_x, self.grid.forcing_y, self.grid.forcing_z = fx, float(forcing[1]), float(forcing[2])

    def enter_ibm_geometry(self, geom: IbmGeomT):
        """set_ibm_coeff for u, v, w generated on the device, then enter_ibm_data."""
        self._c(lib().mdx_enter_ibm_geometry(self.h, C.byref(geom)))

    def exit_ibm_data(self):
        self._c(lib().mdx_exit_ibm_data(self.h))

    def update_host(self, un=None, vn=None, wn=None, pn=None):
        self._c(lib().mdx_update_host(self.h, _p(un), _p(vn), _p(wn), _p(pn)))

    def update_device(self, un=None, vn=None, wn=None, pn=None):
        self._c(lib().mdx_update_device(self.h, _p(un), _p(vn), _p(wn), _p(pn)))

    def get(self, name: str) -> np.ndarray:
        g = self.grid
        if name in ("oldrhsu", "oldrhsv", "oldrhsw"):
            a = np.empty(self.interior)
        elif name == "phi":
            a = np.empty((g.ny, g.nz, g.nx))
        else:
            a = np.empty(self.padded)
        self._c(lib().mdx_copy_field(self.h, FIELD_ID[name], a.ctypes.data, 0))
        return a

    def set(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._c(lib().mdx_copy_field(self.h, FIELD_ID[name], a.ctypes.data, 1))

    # -- time step
    def momentum(self, dt_alpha, dt_beta, dt_gamma):
        self._c(lib().mdx_momentum(self.h, dt_alpha, dt_beta, dt_gamma))

    def apply_bc(self):
        self._c(lib().mdx_apply_bc(self.h))

    def apply_bc_redblack(self):
        self._c(lib().mdx_apply_bc_redblack(self.h))

    def init_pressure_solver(self, opts: SolverOptsT | None = None):
        self.opts = opts if opts is not None else make_solver_opts()
        self._c(lib().mdx_init_pressure_solver(self.h, C.byref(self.opts)))

    def destroy_pressure_solver(self):
        self._c(lib().mdx_destroy_pressure_solver(self.h))

    def pressure_projection(self, dt_gamma, check=True) -> SolveStatsT:
        st = SolveStatsT()
        rc = lib().mdx_pressure_projection(self.h, dt_gamma, C.byref(st))
        if check:
            self._c(rc)
        st.rc = rc
        return st

    def get_cfl(self) -> float:
        c = C.c_double(0.0)
        self._c(lib().mdx_get_cfl(self.h, C.byref(c)))
        return c.value

    def center_vel(self):
        uc = np.empty(self.interior)
        vc = np.empty(self.interior)
        wc = np.empty(self.interior)
        self._c(lib().mdx_center_vel(self.h, uc.ctypes.data, vc.ctypes.data, wc.ctypes.data))
        return uc, vc, wc

    def step(self, nsteps: int) -> int:
        it = C.c_longlong(0)
        self._c(lib().mdx_step(self.h, int(nsteps), C.byref(it)))
        return it.value

    def step_adaptive(self, nsteps: int, cflmax: float, dtmax: float) -> int:
        """nsteps RK3 steps with the adaptive dt of src/main.f90:92-97
        (dt = min(cflmax/cfl, dtmax) after every step); see time()."""
        it = C.c_longlong(0)
        self._c(lib().mdx_step_adaptive(self.h, int(nsteps), float(cflmax), float(dtmax), C.byref(it)))
        return it.value

    def time(self):
        """(dt, t_current, cfl) of the context."""
        a, b, c = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
        self._c(lib().mdx_get_time(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def set_dt(self, dt: float) -> None:
        self._c(lib().mdx_set_dt(self.h, float(dt)))

    def channel_ic(self, seed, amp_u=0.1, amp_vw=0.01, y0=0.0, wave_amp=0.0, wave_lambda=1.0) -> SolveStatsT:
        st = SolveStatsT()
        self._c(lib().mdx_channel_ic(self.h, seed, amp_u, amp_vw, y0, wave_amp, wave_lambda, C.byref(st)))
        return st

    def divergence_norms(self):
        a = C.c_double(0.0)
        b = C.c_double(0.0)
        self._c(lib().mdx_divergence_norms(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_timing(self, on):
        """0/False off; 1/True sampled launches of every class plus whole
        sweep runs; 2 whole sweep runs only (no event between two sweeps)."""
        self._c(lib().mdx_set_timing(self.h, int(on)))

    def get_timing(self) -> dict:
        t = TimingT()
        self._c(lib().mdx_get_timing(self.h, C.byref(t)))
        return {n: (t.ms[k], t.launches[k]) for k, n in enumerate(TIMER_CLASSES)}

    def launch_count(self) -> int:
        return lib().mdx_launch_count(self.h)

    def last_solve_stats(self) -> SolveStatsT:
        st = SolveStatsT()
        self._c(lib().mdx_last_solve_stats(self.h, C.byref(st)))
        return st

    def set_pressure_guess(self, mode: int, record: bool = True) -> None:
        """Warm start of the red-black projection: GUESS_ZERO, GUESS_PREVIOUS
        (the same substage's increment of the previous step) or GUESS_LEARNED
        (U-Net prediction); `record` keeps the increments of every projection."""
        self._c(lib().mdx_set_pressure_guess(self.h, int(mode), 1 if record else 0))

    def warm_checkpoint(self, restore: bool = False) -> None:
        """Save (or restore) the warm-start history on the device."""
        self._c(lib().mdx_warm_checkpoint(self.h, 1 if restore else 0))

    # ---- learned warm start ----------------------------------------------
    def unet_create(self, channels: int = 32, extra_bottleneck: int = 0, capacity: int = 64, slope: float = 0.1,
                    seed: int = 20261203, tcgen05: bool = True, step_rule: int = 0, gate_period: int = 0) -> None:
        o = UnetOptsT()
        lib().mdx_default_unet_opts(C.byref(o))
        o.channels = channels
        o.extra_bottleneck = extra_bottleneck
        o.capacity = capacity
        o.slope = slope
        o.seed = seed
        o.conv_kernel = 0 if tcgen05 else 1
        o.step_rule = step_rule
        o.gate_period = gate_period
        self._c(lib().mdx_unet_create(self.h, C.byref(o)))

    def unet_destroy(self) -> None:
        self._c(lib().mdx_unet_destroy(self.h))

    def unet_record(self, on: bool = True) -> None:
        self._c(lib().mdx_unet_record(self.h, 1 if on else 0))

    def unet_train(self, iters: int, lr: float = 1e-3):
        """Adam steps on the recorded snapshots; (first loss, last loss)."""
        a, b = C.c_double(0.0), C.c_double(0.0)
        self._c(lib().mdx_unet_train(self.h, int(iters), float(lr), C.byref(a), C.byref(b)))
        return a.value, b.value

    def unet_param_count(self) -> int:
        return int(lib().mdx_unet_param_count(self.h))

    def unet_params(self) -> np.ndarray:
        p = np.empty(self.unet_param_count(), dtype=np.float32)
        self._c(lib().mdx_unet_get_params(self.h, p.ctypes.data_as(C.c_void_p), p.size))
        return p

    def unet_set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._c(lib().mdx_unet_set_params(self.h, p.ctypes.data_as(C.c_void_p), p.size))

    def unet_out_scale(self, value: float | None = None) -> float:
        if value is not None:
            self._c(lib().mdx_unet_set_out_scale(self.h, float(value)))
        v = C.c_double(0.0)
        self._c(lib().mdx_unet_get_out_scale(self.h, C.byref(v)))
        return v.value

    def unet_loss_grad(self, in4, target):
        """One forward/backward pass on host inputs [UNET_INPUTS][n] and
        target [n]: (loss, gradient [param_count], output [n])."""
        in4 = np.ascontiguousarray(in4, dtype=np.float32)
        target = np.ascontiguousarray(target, dtype=np.float32)
        n = int(np.prod(self.interior))
        if target.size != n or in4.size != UNET_INPUTS * n:
            raise ValueError(f"unet_loss_grad: inputs must be [{UNET_INPUTS}][{n}] and the target [{n}], "
                             f"got {in4.shape} and {target.shape}")
        grad = np.empty(self.unet_param_count(), dtype=np.float32)
        out = np.empty(target.size, dtype=np.float32)
        loss = C.c_double(0.0)
        self._c(lib().mdx_unet_loss_grad(self.h, in4.ctypes.data_as(C.c_void_p), target.ctypes.data_as(C.c_void_p),
                                         C.byref(loss), grad.ctypes.data_as(C.c_void_p),
                                         out.ctypes.data_as(C.c_void_p)))
        return loss.value, grad, out

    def unet_stats(self) -> UnetStatsT:
        st = UnetStatsT()
        self._c(lib().mdx_unet_stats(self.h, C.byref(st)))
        return st

    def get_increment(self, substage: int) -> np.ndarray:
        """Pressure increment of the last projection of RK substage 0..2 over
        the interior cells, indexed [k, j, i] like the fields."""
        g = self.grid
        out = np.empty(g.nx * g.ny * g.nz, dtype=np.float64)
        self._c(lib().mdx_get_increment(self.h, int(substage), out.ctypes.data_as(C.c_void_p)))
        return out.reshape((g.nz, g.ny, g.nx))

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(lib().mdx_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_stream(self, stream_ptr: int | None):
        self._c(lib().mdx_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))


def make_member(nx, ny, nz, lx=2 * np.pi, ly=2.25, lz=np.pi, re=3000.0, dt=1e-3, amp=0.05, seed=20261203) -> MemberT:
    m = MemberT()
    lib().mdx_default_member(C.byref(m))
    m.nx, m.ny, m.nz = int(nx), int(ny), int(nz)
    m.lx, m.ly, m.lz, m.re, m.dt, m.amp, m.seed = float(lx), float(ly), float(lz), float(re), float(dt), float(amp), int(seed)
    return m


class Ensemble:
    """Independent wavy-wall channels of different sizes advanced together:
    one persistent launch per RK3 substage for all members (C ABI
    mdx_ensemble_*)."""

    def __init__(self, members, opts: SolverOptsT, device: int = 0):
        arr = (MemberT * len(members))(*members)
        h = C.c_void_p()
        rc = lib().mdx_ensemble_create(int(device), len(members), arr, C.byref(opts), C.byref(h))
        if rc != MDX_OK:
            raise MdxError(rc, lib().mdx_last_error(None).decode(errors="replace"))
        self.h = h
        self.members = list(members)

    def _c(self, rc):
        if rc != MDX_OK:
            raise MdxError(rc, lib().mdx_ensemble_last_error(self.h).decode(errors="replace"))

    def close(self):
        if self.h:
            lib().mdx_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_guess(self, mode: int) -> None:
        self._c(lib().mdx_ensemble_set_guess(self.h, int(mode)))

    def ic(self) -> None:
        self._c(lib().mdx_ensemble_ic(self.h))

    def step(self, nsteps: int) -> int:
        it = C.c_longlong(0)
        self._c(lib().mdx_ensemble_step(self.h, int(nsteps), C.byref(it)))
        return it.value

    def unet_load(self, params, out_scale: float, channels: int = 32, extra_bottleneck: int = 0,
                  slope: float = 0.1, tcgen05: bool = True, gate_period: int = 0) -> None:
        """A trained network (mobydiff_b200.learned.TrainedNet's parameters
        and output scale) for the learned warm start of every member;
        gate_period > 0 applies its correction per member and substage only
        while it takes fewer iterations than the extrapolated guess alone."""
        o = UnetOptsT()
        lib().mdx_default_unet_opts(C.byref(o))
        o.channels = channels
        o.extra_bottleneck = extra_bottleneck
        o.capacity = 0
        o.slope = slope
        o.conv_kernel = 0 if tcgen05 else 1
        o.gate_period = gate_period
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._c(lib().mdx_ensemble_unet_load(self.h, C.byref(o), p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                             float(out_scale)))

    def unet_stats(self):
        """(learned corrections kept, undone, left to the extrapolated guess
        by the gate) over all members."""
        a, b, c = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
        self._c(lib().mdx_ensemble_unet_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def member_stats(self, m: int):
        st = SolveStatsT()
        tot = C.c_longlong(0)
        self._c(lib().mdx_ensemble_member_stats(self.h, int(m), C.byref(st), C.byref(tot)))
        return st, tot.value

    def get(self, m: int, name: str) -> np.ndarray:
        q = self.members[m]
        a = np.empty((q.nz + 2, q.ny + 2, q.nx + 2))
        self._c(lib().mdx_ensemble_get(self.h, int(m), FIELD_ID[name], a.ctypes.data_as(C.c_void_p)))
        return a

    def set(self, m: int, name: str, a) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._c(lib().mdx_ensemble_set(self.h, int(m), FIELD_ID[name], a.ctypes.data_as(C.c_void_p)))

    def config(self, threads: int, blocks_per_sm: int = 0, low_regs: bool = False) -> None:
        self._c(lib().mdx_ensemble_config(self.h, int(threads), int(blocks_per_sm), 1 if low_regs else 0))

    def tune(self, cache_path=None):
        """(threads, blocks per SM, low-register variant, ms of the chosen
        shape's step; -1 when it came from the cache)."""
        t, b, r, ms = C.c_int(0), C.c_int(0), C.c_int(0), C.c_double(0.0)
        path = cache_path.encode() if cache_path else None
        self._c(lib().mdx_ensemble_tune(self.h, path, C.byref(t), C.byref(b), C.byref(r), C.byref(ms)))
        return t.value, b.value, bool(r.value), ms.value

    def use_graph(self, on: bool) -> None:
        self._c(lib().mdx_ensemble_use_graph(self.h, 1 if on else 0))

    def info(self) -> dict:
        t, g, lr, gr, ms, ln = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_double(0.0), C.c_longlong(0)
        self._c(lib().mdx_ensemble_info(self.h, C.byref(t), C.byref(g), C.byref(lr), C.byref(gr), C.byref(ms),
                                        C.byref(ln)))
        return {"threads": t.value, "grid": g.value, "low_regs": bool(lr.value), "graph": bool(gr.value),
                "last_step_ms": ms.value, "launches": ln.value}
