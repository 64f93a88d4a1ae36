"""Shared helpers of the parity tests: seeded inputs and comparisons."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def random_fields(g: O.Grid, seed: int, ibm: str = "none", scale=1.0) -> O.Fields:
    """Seeded random state on every array, including ghosts and oldrhs."""
    rng = np.random.default_rng(seed)
    f = O.Fields(g)
    for n in O.FIELD_NAMES:
        getattr(f, n)[...] = scale * rng.uniform(-1.0, 1.0, g.padded)
    for n in O.RHS_NAMES:
        getattr(f, n)[...] = scale * rng.uniform(-1.0, 1.0, g.interior)
    if ibm in ("random", "zinv"):
        for n in O.COEF_NAMES:
            c = rng.uniform(0.0, 50.0, g.padded)
            c[rng.uniform(size=g.padded) < 0.6] = 0.0
            c[rng.uniform(size=g.padded) < 0.05] = 1e30 / g.re
            if ibm == "zinv":           # geometry depending on x and y only
                c[...] = c[0:1]
            getattr(f, n)[...] = c
    elif ibm == "reference":
        O.set_ibm_coeff(g, O.ibm_reference(g), f)
    return f


def to_device(M, g: O.Grid, bc: O.BC, f: O.Fields, device=0):
    """Create a Solver for an oracle state (same arrays, same layout)."""
    mg = M.make_grid(g.nx, g.ny, g.nz, g.lx, g.ly, g.lz, g.re, g.dt, g.forcing)
    mb = M.make_bc(bc.periodic)
    for t in range(24):
        mb.bc_type[t] = bc.bc_type[t]
        mb.bc_value[t] = bc.bc_value[t]
    s = M.Solver(mg, mb, device)
    s.enter_field_data(un=f.un, us=f.us, oldrhsu=f.oldrhsu, vn=f.vn, vs=f.vs, oldrhsv=f.oldrhsv,
                       wn=f.wn, ws=f.ws, oldrhsw=f.oldrhsw, pn=f.pn)
    s.enter_ibm_data(f.coef_u, f.coef_v, f.coef_w)
    return s


def compare_all(s, f: O.Fields, names=None):
    """Max abs difference per array between device and oracle."""
    out = {}
    for n in names or (O.FIELD_NAMES + O.RHS_NAMES):
        out[n] = float(np.max(np.abs(s.get(n) - getattr(f, n))))
    return out


def channel_case(nx, ny, nz, lx=2 * np.pi, ly=2.0, lz=np.pi, re=2000.0, dt=1e-3):
    g = O.Grid(nx, ny, nz, lx=lx, ly=ly, lz=lz, re=re, dt=dt, forcing=(2.0 / re, 0.0, 0.0))
    return g, O.channel_bc()


def oracle_channel_ic(g, bc, f, seed, solver=0, sor=1.7, tol=1e-10, max_iter=200000, check_every=10,
                      amp_u=0.1, amp_vw=0.01, y0=0.0, wave_amp=0.0, wave_lambda=1.0):
    """The seeded channel initial condition and t=0 projection, as mdx_channel_ic does it."""
    for n in O.FIELD_NAMES:
        getattr(f, n)[...] = 0.0
    for n in O.RHS_NAMES:
        getattr(f, n)[...] = 0.0
    O.channel_ic(g, f, seed, amp_u, amp_vw, y0, wave_amp, wave_lambda)
    f.us[...] = f.un
    f.vs[...] = f.vn
    f.ws[...] = f.wn
    res = None
    if solver == 0:
        O.apply_bc(g, f)
        O.pressure_projection_fft(g, f, 1.0)
        O.apply_bc(g, f)
    else:
        res = O.pressure_projection_redblack(g, bc, f, 1.0, sor=sor, tol=tol, max_iter=max_iter,
                                             check_every=check_every)
        O.apply_bc_redblack(g, bc, f)
    f.pn[...] = 0.0
    return res
