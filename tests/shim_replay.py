"""The Fortran drop-in (mobydiff_b200/fortran/mdx_shim.f90) replayed call for
call through the C ABI, for a repository without a Fortran compiler.

`Shim` has one method per shim procedure, with the procedure's name, and each
body makes the C calls the Fortran body makes, in the same order, with the
same state (the last boundary conditions sent, the addresses of the IBM
arrays last uploaded).  `SHIM_CALLS` lists those calls per procedure; a CPU
test reads them out of the Fortran source and compares, so the replay cannot
drift from the shim.  `run_main` follows the call order of src/main.f90:41-106
with the reference's unchanged host modules stood in for by the library's
host restatements (input.ini reader, set_ibm_coeff).
"""
from __future__ import annotations

import ctypes as C
import re

import numpy as np

import mobydiff_b200 as M

# procedure -> the mdx_* functions and shim helpers its body calls, in order
SHIM_CALLS = {
    "sync_ibm": ["mdx_enter_ibm_data"],
    "init_openmp_offload": ["mdx_device_count"],
    "enter_field_data": ["mdx_create", "mdx_enter_field_data"],
    "exit_field_data": ["mdx_exit_field_data", "mdx_destroy"],
    "sync_bc": ["mdx_set_bc"],
    "apply_bc": ["mdx_apply_bc"],
    "apply_bc_redblack": ["sync_bc", "mdx_apply_bc_redblack"],
    "momentum": ["sync_bc", "sync_ibm", "mdx_momentum"],
    "get_cfl": ["mdx_get_cfl"],
    "init_pressure_solver": ["mdx_default_solver_opts", "mdx_init_pressure_solver"],
    "pressure_projection": ["sync_bc", "sync_ibm", "mdx_pressure_projection"],
    "destroy_pressure_solver": ["mdx_destroy_pressure_solver"],
}


def fortran_calls(source: str) -> dict:
    """procedure name -> ordered mdx_* / sync_* calls in its body (the status
    wrapper mdx_check and the ctypes-free helpers excluded)."""
    out = {}
    pat = re.compile(r"^\s*(?:real\([^)]*\)\s+)?(subroutine|function)\s+(\w+)", re.I | re.M)
    for m in pat.finditer(source):
        kind, name = m.group(1).lower(), m.group(2)
        end = re.search(rf"^\s*end\s+{kind}\s+{name}\b", source[m.end():], re.I | re.M)
        body = source[m.end(): m.end() + end.start()]
        body = re.sub(r"!.*", "", body)
        calls = re.findall(r"\b(mdx_\w+|sync_bc|sync_ibm)\s*\(", body)
        out[name] = [c for c in calls if c != "mdx_check"]
    return out


class FortranError(RuntimeError):
    """What the shim's mdx_check / error stop would print before stopping."""


class Ibm:
    """ibm_type's coefficient arrays (src/modules/ibm.f90:23-32)."""

    def __init__(self, cu, cv, cw):
        self.coef_u, self.coef_v, self.coef_w = (np.ascontiguousarray(a) for a in (cu, cv, cw))


class Shim:
    def __init__(self):
        self.lib = M.lib()
        self.ctx = C.c_void_p()
        self.ibm_sent = [None, None, None]
        self.ibm_stale = True
        self.last_bc = None
        self.calls = []     # (procedure, C function) in the order made

    def _c(self, proc, fn, *args):
        self.calls.append((proc, fn))
        return getattr(self.lib, fn)(*args)

    def _check(self, rc, what):
        if rc != 0:
            raise FortranError(f"mobydiff_b200: {what} failed: {M.lib().mdx_last_error(self.ctx).decode()}")

    # module gpu_runtime
    def init_openmp_offload(self):
        n = C.c_int(0)
        rc = self._c("init_openmp_offload", "mdx_device_count", C.byref(n))
        if rc != 0 or n.value <= 0:
            raise FortranError(f"no CUDA device available (status {rc})")
        return n.value

    def enter_field_data(self, f, g: M.GridT):
        cb = M.make_bc((True, True, True))               # init_bc defaults
        self._check(self._c("enter_field_data", "mdx_create", 0, C.byref(g), C.byref(cb), C.byref(self.ctx)),
                    "mdx_create")
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        self._check(self._c("enter_field_data", "mdx_enter_field_data", self.ctx,
                            ptr(f["un"]), ptr(f["us"]), ptr(f["oldrhsu"]), ptr(f["vn"]), ptr(f["vs"]),
                            ptr(f["oldrhsv"]), ptr(f["wn"]), ptr(f["ws"]), ptr(f["oldrhsw"]), ptr(f["pn"])),
                    "enter_field_data")

    def exit_field_data(self, f, g):
        self._check(self._c("exit_field_data", "mdx_exit_field_data", self.ctx), "exit_field_data")
        self._check(self._c("exit_field_data", "mdx_destroy", self.ctx), "mdx_destroy")
        self.ctx = C.c_void_p()
        self.ibm_sent = [None, None, None]
        self.ibm_stale = True

    # module mdx_ibm_sync
    def sync_ibm(self, ibm: Ibm):
        p = [a.ctypes.data for a in (ibm.coef_u, ibm.coef_v, ibm.coef_w)]
        if not self.ibm_stale and p == self.ibm_sent:
            return
        self._check(self._c("sync_ibm", "mdx_enter_ibm_data", self.ctx, *[C.c_void_p(q) for q in p]),
                    "enter_ibm_data")
        self.ibm_sent = p
        self.ibm_stale = False

    def ibm_coefficients_changed(self):
        self.ibm_stale = True

    # module boundary
    def sync_bc(self, bc: M.BcT):
        key = (tuple(bc.is_periodic), tuple(bc.bc_type), tuple(bc.bc_value))
        if self.last_bc == key:
            return
        self._check(self._c("sync_bc", "mdx_set_bc", self.ctx, C.byref(bc)), "mdx_set_bc")
        self.last_bc = key

    def apply_bc(self, f, g):
        self._check(self._c("apply_bc", "mdx_apply_bc", self.ctx), "apply_bc")

    def apply_bc_redblack(self, f, g, bc):
        self.sync_bc(bc)
        self._check(self._c("apply_bc_redblack", "mdx_apply_bc_redblack", self.ctx), "apply_bc_redblack")

    # module step
    def momentum(self, f, g, dt_alpha, dt_beta, dt_gamma, ibm, bc):
        self.sync_bc(bc)
        self.sync_ibm(ibm)
        self._check(self._c("momentum", "mdx_momentum", self.ctx, dt_alpha, dt_beta, dt_gamma), "momentum")

    def get_cfl(self, f, g):
        c = C.c_double(0.0)
        self._check(self._c("get_cfl", "mdx_get_cfl", self.ctx, C.byref(c)), "get_cfl")
        return c.value

    # module pressure_solver
    def init_pressure_solver(self, ps, g, redblack: bool):
        o = M.SolverOptsT()
        self._c("init_pressure_solver", "mdx_default_solver_opts", C.byref(o))
        if redblack:                                 # #ifdef USE_REDBLACK
            o.solver = M.SOLVER_REDBLACK
            o.n_iter = ps["nIter"]
            o.sor = ps["sor"]
        else:
            o.solver = M.SOLVER_FFT
        self._check(self._c("init_pressure_solver", "mdx_init_pressure_solver", self.ctx, C.byref(o)),
                    "init_pressure_solver")

    def pressure_projection(self, ps, f, g, dt_gamma, ibm, bc):
        self.sync_bc(bc)
        self.sync_ibm(ibm)
        self._check(self._c("pressure_projection", "mdx_pressure_projection", self.ctx, dt_gamma, None),
                    "pressure_projection")

    def destroy_pressure_solver(self, ps):
        self._check(self._c("destroy_pressure_solver", "mdx_destroy_pressure_solver", self.ctx),
                    "destroy_pressure_solver")

    # io.f90's `!$omp target update from(...)` before writing a field
    def update_host(self, f):
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        self._check(self.lib.mdx_update_host(self.ctx, ptr(f["un"]), ptr(f["vn"]), ptr(f["wn"]), ptr(f["pn"])),
                    "update_host")


def run_main(input_ini: str, redblack: bool):
    """src/main.f90:41-106 with this shim; returns (grid, bc, ps, host fields
    after the run, IBM coefficients, the shim's call log)."""
    g, bc, opts, run = M.read_runtime_config(input_ini)   # init_grid + init_bc + read_runtime_config
    ps = {"nIter": opts.n_iter, "sor": opts.sor}
    shim = Shim()
    shim.init_openmp_offload()
    pad = (g.nz + 2, g.ny + 2, g.nx + 2)
    inner = (g.nz, g.ny, g.nx)
    f = {n: np.zeros(pad) for n in ("un", "us", "vn", "vs", "wn", "ws", "pn")}         # init_field
    f.update({n: np.zeros(inner) for n in ("oldrhsu", "oldrhsv", "oldrhsw")})
    shim.enter_field_data(f, g)
    shim.init_pressure_solver(ps, g, redblack)
    ibm = Ibm(*M.set_ibm_coeff(g, M.ibm_reference(g)))   # init_ibm + set_ibm_coeff x3
    # enter_ibm_data(ibm, g): ibm.f90 unchanged, OpenMP directives only -- nothing to call
    a, b, c = M.rk_coeffs()
    for _ in range(g.nsteps):
        g.t_current = g.t_current + g.dt
        for st in range(3):
            dt_a, dt_b, dt_g = g.dt * a[st], g.dt * b[st], g.dt * c[st]
            shim.momentum(f, g, dt_a, dt_b, dt_g, ibm, bc)
            if not redblack:
                shim.apply_bc(f, g)
            shim.pressure_projection(ps, f, g, dt_g, ibm, bc)
            if redblack:
                shim.apply_bc_redblack(f, g, bc)
            else:
                shim.apply_bc(f, g)
        if g.cflmax > 0.0:
            g.cfl = shim.get_cfl(f, g)
            if g.cfl > 0.0:
                g.dt = min(g.cflmax / g.cfl, g.dtmax)
    shim.update_host(f)
    shim.destroy_pressure_solver(ps)
    # exit_ibm_data(ibm, g): unchanged, nothing to call
    shim.exit_field_data(f, g)
    return g, bc, ps, f, ibm, shim.calls
