"""The standalone driver (mdx_main, the reference's main program): a short
channel run from an input.ini that writes field files and VTK files every two
steps.  The field files carry the run's time and the oracle's state after the
same steps (rel-L2 <= 1e-11, FFT path); the VTK files have the byte layout of
the reference's data_output (src/modules/io.f90:224-259) -- its header lines
and the Fortran edit descriptors I0 and ES20.12, emulated here independently
-- and hold the centre velocities of center_vel (io.f90:184-222) of the
state written beside them."""
import os
import subprocess

import numpy as np
import pytest

import mobydiff_b200 as M
from oracle import oracle as O
from tests.helpers import channel_case, oracle_channel_ic, rel_l2

MAIN = os.path.join(os.path.dirname(M.__file__), "mdx_main")


def fortran_es(x: float, w: int = 20, d: int = 12) -> str:
    """Fortran ESw.d output of one value: d digits after the point; exponent
    E+dd, or +ddd without the letter when it needs three digits."""
    mant, exp = f"{x:.{d}E}".split("E")
    e = int(exp)
    sign = "+" if e >= 0 else "-"
    t = f"{mant}E{sign}{abs(e):02d}" if abs(e) <= 99 else f"{mant}{sign}{abs(e):03d}"
    return t.rjust(w)


def test_fortran_es_emulation():
    assert fortran_es(1.0) == "  1.000000000000E+00"
    assert fortran_es(-2.5e-3) == " -2.500000000000E-03"
    assert fortran_es(0.0) == "  0.000000000000E+00"
    assert fortran_es(1.5e-120) == "  1.500000000000-120"


@pytest.mark.gpu
def test_driver_writes_field_files(tmp_path):
    ini = tmp_path / "input.ini"
    ini.write_text("""
[grid]
nx = 32
ny = 16
nz = 16
lx = 6.283185307179586
ly = 2.0
lz = 3.141592653589793
[flow]
re = 2000.0
forcing_x = 1e-3
[time]
dt = 1e-3
nsteps = 4
[boundary]
periodic_y = no
y_min_p_type = neumann
y_max_p_type = neumann
[output]
interval = 2
prefix = vel
h5_interval = 2
field_prefix = chk
[b200]
ic = channel
seed = 5
""")
    r = subprocess.run([MAIN, str(ini)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "main loop ended" in r.stdout
    for step in (2, 4):
        name = f"chk_{step}.h5"
        assert f"field filename: {name}" in r.stdout
        h = M.h5_read_header(str(tmp_path / name))
        assert (h["nx"], h["ny"], h["nz"]) == (32, 16, 16)
        assert abs(h["t_current"] - step * 1e-3) <= 1e-15 and h["re"] == 2000.0
        un, vn, wn, pn = M.h5_read_field(str(tmp_path / name), 32, 16, 16)
        assert np.isfinite(un).all() and np.abs(un).max() > 0.5    # the channel flow
    assert not os.path.exists(tmp_path / "chk_1.h5") and not os.path.exists(tmp_path / "chk_3.h5")

    # the state after 4 steps against the oracle (same input, same seeded start,
    # the reference's IBM bump that the driver applies by default like
    # src/main.f90:57-61)
    g, bc = channel_case(32, 16, 16, re=2000.0, dt=1e-3)
    g.forcing = (1e-3, 0.0, 0.0)
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_reference(g), f)
    oracle_channel_ic(g, bc, f, 5)
    O.run(g, bc, f, g.dt, 4, solver=0)
    fields = M.h5_read_field(str(tmp_path / "chk_4.h5"), 32, 16, 16)
    for n, a in zip(("un", "vn", "wn", "pn"), fields):
        assert rel_l2(a, getattr(f, n)) <= 1e-11, n
    # the VTK files: the reference's layout, values of center_vel of the state
    for step in (2, 4):
        lines = (tmp_path / f"vel_{step}.vtk").read_text().split("\n")
        un, vn, wn, _ = M.h5_read_field(str(tmp_path / f"chk_{step}.h5"), 32, 16, 16)
        h = M.h5_read_header(str(tmp_path / f"chk_{step}.h5"))
        head = ["# vtk DataFile Version 3.0", "3D velocity field", "ASCII", "DATASET STRUCTURED_POINTS",
                "DIMENSIONS 33 17 17", "ORIGIN " + fortran_es(0.0) * 3,
                "SPACING " + fortran_es(h["dx"]) + fortran_es(h["dy"]) + fortran_es(h["dz"]),
                "FIELD FieldData 1", "TIME 1 1 double", fortran_es(h["t_current"]), "CELL_DATA 8192",
                "VECTORS U double"]
        assert lines[:12] == head
        uc = 0.5 * (un[1:-1, 1:-1, 1:-1] + un[1:-1, 1:-1, 2:])
        vc = 0.5 * (vn[1:-1, 1:-1, 1:-1] + vn[1:-1, 2:, 1:-1])
        wc = 0.5 * (wn[1:-1, 1:-1, 1:-1] + wn[2:, 1:-1, 1:-1])
        body = [fortran_es(a) + fortran_es(b) + fortran_es(c)
                for a, b, c in zip(uc.ravel(), vc.ravel(), wc.ravel())]
        assert lines[12:12 + len(body)] == body
        assert lines[12 + len(body):] == [""]


@pytest.mark.gpu
def test_driver_adaptive_dt(tmp_path):
    """cflmax > 0 in input.ini: the driver's steps take dt = min(cflmax/cfl,
    dtmax) after every step (src/main.f90:92-97), computed on the device; the
    field file's dt and t_current and its state match the oracle's adaptive
    loop."""
    ini = tmp_path / "input.ini"
    ini.write_text("""
[grid]
nx = 32
ny = 16
nz = 16
lx = 6.283185307179586
ly = 2.0
lz = 3.141592653589793
[flow]
re = 2000.0
forcing_x = 1e-3
[time]
dt = 1e-3
nsteps = 5
cflmax = 0.02
dtmax = 5e-3
[boundary]
periodic_y = no
y_min_p_type = neumann
y_max_p_type = neumann
[output]
h5_interval = 5
field_prefix = chk
[b200]
ic = channel
seed = 5
""")
    r = subprocess.run([MAIN, str(ini)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    h = M.h5_read_header(str(tmp_path / "chk_5.h5"))
    g, bc = channel_case(32, 16, 16, re=2000.0, dt=1e-3)
    g.forcing = (1e-3, 0.0, 0.0)
    f = O.Fields(g)
    O.set_ibm_coeff(g, O.ibm_reference(g), f)
    oracle_channel_ic(g, bc, f, 5)
    dt, t = 1e-3, 0.0
    for _ in range(5):
        t += dt
        O.run(g, bc, f, dt, 1, solver=0)
        dt = min(0.02 / O.get_cfl(g, f), 5e-3)
    assert dt != 1e-3
    assert abs(h["t_current"] - t) <= 1e-12 * t and abs(h["dt"] - dt) <= 1e-10 * dt
    fields = M.h5_read_field(str(tmp_path / "chk_5.h5"), 32, 16, 16)
    for n, a in zip(("un", "vn", "wn", "pn"), fields):
        assert rel_l2(a, getattr(f, n)) <= 1e-10, n
