"""Builds libfieldgrid.so in-tree (next to this file) with nvcc for sm_100a.

Usage: python -m fieldgrid_b200.build   (or __graft_entry__.build()).
The library is rebuilt only when a source is newer than it, unless force=True.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfieldgrid.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def host_cxx() -> str:
    # the image's default CXX has no OpenMP runtime; the system g++ does
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
    deps.append(os.path.join(ROOT, "include", "fieldgrid.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cxx = host_cxx()
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if src.endswith(".cu"):
            cmd = [nvcc, "-ccbin", cxx, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-c", src, "-o", obj,
                   "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", "-Xptxas", "-O3",
                   # no a*b+c contraction: the kernels round like the reference's CPU path
                   "--fmad=false",
                   "-I", os.path.join(ROOT, "include")]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        else:
            # host code: the setup arithmetic must not be contracted into FMAs
            cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-c", src, "-o", obj,
                   "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"compiling {os.path.basename(src)} failed")
        if verbose and (r.stdout or r.stderr):
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = OUT + ".tmp"
    cmd = [nvcc, "-ccbin", cxx, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp",
           "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("linking libfieldgrid.so failed")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
