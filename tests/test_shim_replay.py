"""The Fortran drop-in, replayed through the C ABI.

CPU: every procedure of mobydiff_b200/fortran/mdx_shim.f90 makes exactly the
C calls the replay (tests/shim_replay.py) makes, in the same order, and every
C function the shim binds is declared in mdx_bindings.f90 and exported by the
library.

GPU: src/main.f90:41-106 run through the replayed shim -- input.ini, zero
initial fields, the reference's default IBM geometry (ibm.f90:45-50), a few
steps on the FFT path and on the red-black path -- against the oracle run
with the same coefficients: rel-L2 <= 1e-11 (FFT) and bit-exact (red-black
with the reference's fixed nIter).  A run of the oracle without the IBM
differs by far more, so the IBM coefficients demonstrably reach the device
through the shim's own calls.
"""
import os
import re
import textwrap

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import rel_l2
from tests.shim_replay import SHIM_CALLS, fortran_calls, run_main

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "mobydiff_b200", "fortran", "mdx_shim.f90")
BINDINGS = os.path.join(ROOT, "mobydiff_b200", "fortran", "mdx_bindings.f90")


def test_replay_matches_the_fortran_bodies():
    src = open(SHIM).read()
    got = fortran_calls(src)
    for proc, calls in SHIM_CALLS.items():
        assert proc in got, proc
        assert got[proc] == calls, (proc, got[proc], calls)
    # every procedure of the shim that calls the library is replayed
    missing = [p for p, c in got.items() if c and p not in SHIM_CALLS]
    assert not missing, missing


def test_shim_bindings_declared_and_exported():
    src = open(SHIM).read()
    used = {c for calls in fortran_calls(src).values() for c in calls if c.startswith("mdx_")}
    bound = set(re.findall(r'bind\(C,\s*name="(mdx_\w+)"\)', open(BINDINGS).read()))
    assert used <= bound, used - bound
    lib = M.lib()
    for name in used:
        assert hasattr(lib, name), name


def _ini(tmp_path, redblack):
    text = f"""
        [grid]
        nx = 32
        ny = 24
        nz = 16
        lx = 1.0
        ly = 1.0
        lz = 0.5
        [flow]
        re = 100.0
        [time]
        dt = 2.0e-4
        steps = 6
        [pressure]
        niter = 40
        omega = 1.5
        [boundary]
        periodic_y = {"no" if redblack else "yes"}
        y_min_p_type = neumann
        y_max_p_type = neumann
        """
    p = tmp_path / "input.ini"
    p.write_text(textwrap.dedent(text))
    return str(p)


def _oracle_run(g, bc, ps, redblack, ibm_on):
    og = O.Grid(g.nx, g.ny, g.nz, lx=g.lx, ly=g.ly, lz=g.lz, re=g.re, dt=g.dt,
                forcing=(g.forcing_x, g.forcing_y, g.forcing_z))
    ob = O.BC(tuple(bool(x) for x in bc.is_periodic))
    ob.bc_type[:] = list(bc.bc_type)
    ob.bc_value[:] = list(bc.bc_value)
    f = O.Fields(og)
    if ibm_on:
        O.set_ibm_coeff(og, O.ibm_reference(og), f)
    O.run(og, ob, f, og.dt, g.nsteps, solver=1 if redblack else 0, niter=ps["nIter"], sor=ps["sor"], tol=0.0)
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("redblack", [False, True])
def test_main_sequence_through_the_shim(tmp_path, redblack):
    g, bc, ps, f, ibm, calls = run_main(_ini(tmp_path, redblack), redblack)
    # the coefficients went up once, from the first predictor, through sync_ibm
    uploads = [c for c in calls if c[1] == "mdx_enter_ibm_data"]
    assert uploads == [("sync_ibm", "mdx_enter_ibm_data")], uploads
    first = [c[1] for c in calls].index("mdx_enter_ibm_data")
    assert [c[1] for c in calls].index("mdx_momentum") > first
    assert np.count_nonzero(ibm.coef_u) > 0
    ref = _oracle_run(g, bc, ps, redblack, ibm_on=True)
    plain = _oracle_run(g, bc, ps, redblack, ibm_on=False)
    # velocity components against the velocity vector's norm (w is round-off
    # noise in this flow: the geometry varies in x only), p against its own
    vel = np.sqrt(sum(np.linalg.norm(getattr(ref, n)) ** 2 for n in ("un", "vn", "wn")))
    for n in ("un", "vn", "wn", "pn"):
        b = getattr(ref, n)
        e = float(np.linalg.norm(f[n] - b)) / (vel if n != "pn" else float(np.linalg.norm(b)))
        if redblack:
            assert np.array_equal(f[n], b), (n, e)
        else:
            assert e <= 1e-11, (n, e)
    # without the coefficients the flow is another flow
    assert rel_l2(getattr(plain, "un"), ref.un) > 1e-3
