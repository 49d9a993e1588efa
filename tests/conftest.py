import glob
import hashlib
import importlib
import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GROUPS = ("hole", "left_sym", "bottom_sym", "right", "top")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("mpi-cst-fem-solver_b200")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


class Golden:
    def __init__(self, name):
        p = os.path.join(GOLDEN, name)
        self.npz = np.load(p + ".npz") if os.path.exists(p + ".npz") else None
        self.meta = json.load(open(p + ".json")) if os.path.exists(p + ".json") else {}

    def __getitem__(self, k):
        return self.npz[k]

    def mesh(self, pkg):
        groups = {g: self.npz["group_" + g] for g in GROUPS if "group_" + g in self.npz}
        return pkg.plate.Mesh(xy=self.npz["xy"], triangles=self.npz["tri"], boundary_edges=groups)


@pytest.fixture(scope="session")
def golden():
    return Golden


@pytest.fixture(scope="session")
def gpu_lib(pkg):
    """The built sm_100a library (built in-tree when missing)."""
    pkg.build.build_library()
    return pkg.native.load()


@pytest.fixture
def ctx(pkg, gpu_lib):
    c = pkg.Context(0)
    yield c
    c.close()
