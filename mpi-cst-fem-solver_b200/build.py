"""Build recipe of the sm_100a library (libcstfem_b200.so, in-tree next to this file).

nvcc compiles csrc/*.cu for sm_100a only (-gencode arch=compute_100a,code=sm_100a) into a
shared library with the C ABI of include/cstfem_b200.h. Host code is compiled with
-ffp-contract=off so its arithmetic (constitutive matrix, traction loads) matches the
reference's g++ -O3 build bit for bit.
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcstfem_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def sources() -> list:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _deps() -> list:
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.h*"))) + \
        sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        [os.path.join(REPO, "include", "cstfem_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile the library unless it is newer than every source; returns its path."""
    if not force and up_to_date():
        return LIB
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-ccbin", "/usr/bin/g++",
           "-o", LIB + ".tmp"] + sources()
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    import sys
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
