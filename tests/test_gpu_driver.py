"""The standalone driver (mdx_main, the reference's main program): a short
channel run from an input.ini that writes field files every two steps;
the files carry the run's time and restart the same state."""
import os
import subprocess

import numpy as np
import pytest

import mobydiff_b200 as M

pytestmark = pytest.mark.gpu

MAIN = os.path.join(os.path.dirname(M.__file__), "mdx_main")


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
interval = 0
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
