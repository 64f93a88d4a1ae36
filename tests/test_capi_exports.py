"""The C-ABI library loads and exports every entry point the header declares."""
import os
import re
import subprocess

import pytest

import mobydiff_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(mdx_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_all_declared_symbols():
    M.lib()
    out = subprocess.check_output(["nm", "-D", "--defined-only", M.LIB_PATH], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = _declared()
    assert len(declared) >= 30
    missing = sorted(declared - exported)
    assert not missing, missing


def test_version_and_defaults():
    assert "sm_100a" in M.version()
    g = M.make_grid(8, 8, 8)
    assert g.dx == 1.0 / 8
    o = M.make_solver_opts()
    assert o.n_iter == 3 and o.sor == 1.5     # pressure_workspace.f90:7-8


def test_no_device_fails_loudly():
    if M.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(M.MdxError) as e:
        M.Solver(M.make_grid(8, 8, 8), M.channel_bc())
    assert e.value.code == M.MDX_ERR_NO_DEVICE
