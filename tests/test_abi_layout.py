"""The ctypes mirror of the public structs (mobydiff_b200/__init__.py) has
the C header's layout: a probe compiled with gcc against
include/mobydiff_b200.h prints sizeof and every field's offsetof, and each
must equal the ctypes value."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

import mobydiff_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [
    (M.GridT, "mdx_grid_t"),
    (M.BcT, "mdx_bc_t"),
    (M.SolverOptsT, "mdx_solver_opts_t"),
    (M.SolveStatsT, "mdx_solve_stats_t"),
    (M.UnetOptsT, "mdx_unet_opts_t"),
    (M.UnetStatsT, "mdx_unet_stats_t"),
    (M.MemberT, "mdx_member_t"),
    (M.TimingT, "mdx_timing_t"),
    (M.RunConfigT, "mdx_run_config_t"),
    (M.IbmGeomT, "mdx_ibm_geom_t"),
]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mobydiff_b200.h"', "int main(void) {"]
    expect = []
    for cls, cname in PAIRS:
        lines.append(f'    printf("%zu\\n", sizeof({cname}));')
        expect.append((cname, "sizeof", C.sizeof(cls)))
        for f in cls._fields_:
            name = f[0]
            cfield = name[:-1] if name.endswith("_") else name    # lambda_ mirrors C's lambda
            lines.append(f'    printf("%zu\\n", offsetof({cname}, {cfield}));')
            expect.append((cname, name, getattr(cls, name).offset))
    lines += ["    return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.check_call(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)], text=True).split()]
    assert len(got) == len(expect)
    bad = [(s, f, e, g) for (s, f, e), g in zip(expect, got) if e != g]
    assert not bad, bad
