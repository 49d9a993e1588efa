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


def _flags() -> list:
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
            "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", "/usr/bin/g++"]


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile the library unless it is newer than every source; returns its path. Each source
    is compiled to its own object (in parallel, one nvcc per file) and the objects are linked."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    headers = [p for p in _deps() if not p.endswith(".cu")]
    newest_header = max(os.path.getmtime(p) for p in headers)
    jobs = []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
        stale = force or not os.path.exists(obj) or \
            os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header)
        cmd = [NVCC] + (["-Xptxas=-v"] if verbose else []) + _flags() + ["-c", src, "-o", obj + ".tmp"]
        jobs.append((obj, cmd if stale else None))

    def run(job):
        obj, cmd = job
        if cmd is None:
            return obj
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(obj + ".tmp", obj)
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(run, jobs))
    subprocess.run([NVCC] + _flags() + ["-shared", "-o", LIB + ".tmp"] + objs, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    import sys
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
