"""Builds libomvgba_cuda.so (C ABI + sm_100a kernels) in-tree with nvcc.

Usage: python openmvg-rs_b200/build.py [--debug]
The library lands in openmvg-rs_b200/openmvg_ba_cuda/_lib/ so it travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "openmvg_ba_cuda", "_lib")
LIB = os.path.join(OUT_DIR, "libomvgba_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["gpu_solver.cu", "residual.cu", "residual_static.cu", "sfm_refresh.cu"]
CPP_SOURCES = ["host.cpp", "fixed_rotation.cpp", "sfm_prepare.cpp"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [s for s in CU_SOURCES + CPP_SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "ba_cuda.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    opt = ["-O0", "-g", "-G"] if debug else ["-O3"]
    for src in sources():
        path = os.path.join(CSRC, src)
        obj = os.path.join(obj_dir, src + ".o")
        cmd = [nvcc(), *ARCH, "-lineinfo", "-std=c++17", *opt, "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
               "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include"), "-c", path, "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        else:
            cmd += ["-x", "c++"]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    link = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"]
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, verbose="--verbose" in sys.argv))
