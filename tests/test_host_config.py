"""Host-side set-up of the library (no device): the input.ini reader with the
semantics of src/modules/config.f90 and the IBM coefficients of
src/modules/ibm.f90, the latter bit-exact against the oracle."""
import os
import textwrap

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O


def _ini(tmp_path, text):
    p = tmp_path / "input.ini"
    p.write_text(textwrap.dedent(text))
    return str(p)


def test_sections_keys_aliases(tmp_path, capfd):
    path = _ini(tmp_path, """
        ; a comment line
        [GRID]
        nx = 96          ; trailing comment
        NY=48
        nz 40
        lx = 6.2831853   # hash comment
        ly = 2
        lz = 3.14159d0
        [flow]
        Re = 2.0e3
        meanpx = 1.0D-3
        force_z = -0.5
        [time]
        dt = 5.0e-4
        steps = 12
        cflmax = 0.7
        [pressure]
        niter = 7
        omega = 1.8
        [boundary]
        periodic_y = no
        y_periodic = .false.
        x_is_periodic = T
        bottom_min_p_type = neumann
        y_min_p_type = neumann
        y_max_p_type = 1
        y_max_u_value = 0.25
        z_lo_w_type = gradient
        [output]
        interval = 0
        prefix = "run 1"
        h5_interval = 5
        [unknown]
        nx = 3
        [b200]
        solver = redblack
        tol = 1e-10
        max_iter = 5000
        check_every = 25
        ic = channel
        seed = 42
        ibm = wavy
        ibm_amp = 0.05
        guess = extrapolated
        inner_omega = 1.95
        residual_checks = fixed
        fft_kernel = stockham
        inner_form = faces
    """)
    g, b, o, r = M.read_runtime_config(path)
    assert (g.nx, g.ny, g.nz) == (96, 48, 40)
    assert g.lx == 6.2831853 and g.ly == 2.0 and g.lz == 3.14159
    assert g.re == 2000.0 and g.forcing_x == 1e-3 and g.forcing_z == -0.5
    assert g.dt == 5e-4 and g.nsteps == 12 and g.cflmax == 0.7
    assert g.dx == g.lx / 96 and g.t_final == g.dt * 12
    assert list(b.is_periodic) == [1, 0, 1]
    idx = lambda d, s, v: (d - 1) + 3 * (s + 2 * v)
    assert b.bc_type[idx(2, 0, 0)] == 1 and b.bc_type[idx(2, 1, 0)] == 1
    assert b.bc_value[idx(2, 1, 1)] == 0.25 and b.bc_type[idx(3, 0, 3)] == 1
    assert o.n_iter == 7 and o.sor == 1.8
    assert o.solver == M.SOLVER_REDBLACK and o.tol == 1e-10 and o.max_iter == 5000 and o.check_every == 25
    assert r.output_interval == 0 and r.output_prefix == b"run 1" and r.field_interval == 5
    assert r.ic == 1 and r.seed == 42 and r.ibm == 1 and r.ibm_amp == 0.05
    assert r.guess == M.GUESS_EXTRAPOLATED and o.inner_sor == 1.95 and o.check_mode == 1
    assert o.fft_kernel == 1 and o.inner_form == 1
    out = capfd.readouterr().out
    assert "unknown boundary key" in out      # bottom_min_p_type: "bottom" is not a direction


def test_t_final_sets_nsteps(tmp_path):
    path = _ini(tmp_path, """
        [time]
        dt = 0.003
        t_final = 0.01
    """)
    g, *_ = M.read_runtime_config(path)
    assert g.nsteps == 4                      # ceiling(0.01/0.003)


def test_missing_file_keeps_defaults(tmp_path, capfd):
    g, b, o, r = M.read_runtime_config(str(tmp_path / "nope.ini"))
    assert (g.nx, g.ny, g.nz, g.nsteps) == (200, 200, 200, 10000)
    assert g.re == 100.0 and g.dt == 1e-4 and g.forcing_x == 1.0
    assert list(b.is_periodic) == [1, 1, 1]
    assert r.output_interval == 1 and r.output_prefix == b"data" and r.field_prefix == b"field"
    assert "input file not found" in capfd.readouterr().out


def test_bad_values_warn_and_keep(tmp_path, capfd):
    path = _ini(tmp_path, """
        [grid]
        nx = 12.5
        ny = abc
        nz =
        [pressure]
        niter = -2
        [boundary]
        periodic_x = maybe
        x_min_u_type = robin
        x_min_u_flavour = 1
    """)
    g, b, o, r = M.read_runtime_config(path)
    assert (g.nx, g.ny, g.nz) == (200, 200, 200)
    assert o.n_iter == 3 and b.is_periodic[0] == 1
    assert r.warnings == 7
    out = capfd.readouterr().out
    assert out.count("warning") == 7


@pytest.mark.parametrize("geom", ["reference", "wavy"])
def test_ibm_coefficients_match_oracle(geom):
    g = M.make_grid(40, 24, 6, lx=2 * np.pi, ly=2.25, lz=1.0, re=3000.0)
    og = O.Grid(40, 24, 6, lx=2 * np.pi, ly=2.25, lz=1.0, re=3000.0)
    if geom == "reference":
        mg, oi = M.ibm_reference(g), O.ibm_reference(og)
    else:
        mg, oi = M.ibm_wavy(0.05, g.lx / 2, 0.125), O.ibm_wavy(0.05, og.lx / 2, 0.125)
    cu, cv, cw = M.set_ibm_coeff(g, mg)
    f = O.Fields(og)
    O.set_ibm_coeff(og, oi, f)
    assert np.array_equal(cu, f.coef_u)
    assert np.array_equal(cv, f.coef_v)
    assert np.array_equal(cw, f.coef_w)
    assert (cu > 0).any() and (cu < 1e30 / 3000.0).any()


def test_inner_form_values(tmp_path):
    for text, want in (("potential", 0), ("faces", 1), ("potential_all", 2), ("2", 2)):
        path = _ini(tmp_path, f"""
            [b200]
            inner_form = {text}
        """)
        _, _, o, _ = M.read_runtime_config(path)
        assert o.inner_form == want, text
