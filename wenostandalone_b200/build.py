"""Build libweno_sb.so (and the harness driver) in-tree for sm_100a.

    python -m wenostandalone_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libweno_sb.so")
DRIVER = os.path.join(HERE, "weno_standalone_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _sources():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    deps.append(os.path.join(INCLUDE, "weno_sb.h"))
    return deps


def build_lib(force: bool = False, verbose: bool = False) -> str:
    deps = _sources()
    if not force and _newer(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-shared", f"-I{INCLUDE}", "-o", LIB,
           os.path.join(CSRC, "weno_sb.cu")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


def build_driver(force: bool = False, verbose: bool = False) -> str | None:
    src = os.path.join(CSRC, "weno_driver.cpp")
    if not os.path.exists(src):
        return None
    deps = _sources() + [LIB]
    if not force and _newer(DRIVER, deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", f"-I{INCLUDE}", "-o", DRIVER, src,
           f"-L{HERE}", "-lweno_sb", f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force, verbose)
    build_driver(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
