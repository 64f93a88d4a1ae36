"""Build libmobyb200.so in-tree with nvcc for sm_100a (and the mdx_main driver).

Usage:  python -m mobydiff_b200.build [--force]

Each CUDA source is compiled separately so that the FP64 parity kernels keep
-fmad=false (no FMA contraction, the arithmetic of the reference's x86-64
gfortran -O2 build) while other files may choose their own flags.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmobyb200.so")
MAIN = os.path.join(HERE, "mdx_main")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
               "--expt-relaxed-constexpr"]

# source -> extra nvcc flags
CUDA_SOURCES = {
    "capi.cu": ["-fmad=false"],
    "k_step.cu": ["-fmad=false"],
    "k_fft.cu": ["-fmad=false"],
    "k_sor.cu": ["-fmad=false"],
    "k_sor_mixed.cu": [],   # FP32 sweeps inside FP64 defect correction: FMA allowed
    "k_warm.cu": ["-fmad=false"],
    "k_unet.cu": [],        # BF16 network with FP32 accumulation: FMA allowed
    "k_ensemble.cu": ["-fmad=false"],
    "k_ibm.cu": ["-fmad=false"],   # IBM coefficients: the host routine's arithmetic
}
CXX_SOURCES = ["host_config.cpp", "h5_field.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "mobydiff_b200.h"))
    objs = []
    for src, extra in CUDA_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc, *ARCH, *NVCC_COMMON, *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers + [__file__]):
            cmd = [_cxx(), "-O2", "-ffp-contract=off", "-std=c++17", "-fPIC", "-Wall", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    main_src = os.path.join(CSRC, "mdx_main.cpp")
    if os.path.exists(main_src) and (force or _stale(MAIN, [main_src, LIB] + headers)):
        cmd = [_cxx(), "-O2", "-std=c++17", "-o", MAIN, main_src, "-L" + HERE, "-lmobyb200",
               "-Wl,-rpath,$ORIGIN", "-I" + os.path.join(ROOT, "include")]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
