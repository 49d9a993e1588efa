"""CPU tests: the synthetic plate generator, the C-ABI library's exports, and the host mirror
of the reference interface (no device calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO


def test_plate_geometry(pkg):
    p = pkg.plate.quarter_plate(40, 80)
    assert p.num_nodes == 41 * 81 == 3321 and p.num_triangles == 2 * 40 * 80
    P = p.xy.reshape(-1, 2)
    t = p.triangles.reshape(-1, 3)
    A = 0.5 * ((P[t[:, 1], 0] - P[t[:, 0], 0]) * (P[t[:, 2], 1] - P[t[:, 0], 1])
               - (P[t[:, 2], 0] - P[t[:, 0], 0]) * (P[t[:, 1], 1] - P[t[:, 0], 1]))
    assert (A > 0).all()  # counter-clockwise
    assert abs(A.sum() - (100.0 - np.pi / 4.0)) < 1e-2  # polygonal hole
    g = {k: np.unique(v) for k, v in p.boundary_edges.items()}
    assert np.all(P[g["right"], 0] == 10.0) and np.all(P[g["top"], 1] == 10.0)
    assert np.all(P[g["left_sym"], 0] == 0.0) and np.all(P[g["bottom_sym"], 1] == 0.0)
    assert np.allclose(np.hypot(P[g["hole"], 0], P[g["hole"], 1]), 1.0, atol=1e-15)
    corner = np.intersect1d(g["right"], g["top"])
    assert corner.size == 1 and P[corner[0]].tolist() == [10.0, 10.0]
    # graded: last/first radial ratio of the 40-cell mesh is 1.05^39
    r = np.hypot(P[:41, 0], P[:41, 1])
    assert abs((r[40] - r[39]) / (r[1] - r[0]) - 1.05 ** 39) < 1e-9


def test_plate_sizes_of_the_workloads(pkg):
    # DOF counts of the named plates ((n_r + 1)(n_theta + 1) nodes, 2 DOFs each)
    dofs = lambda nr, nt: 2 * (nr + 1) * (nt + 1)
    assert dofs(40, 80) == 6642
    assert dofs(400, 1250) == 1_003_302
    assert dofs(565, 1766) == 2_000_244
    with pytest.raises(ValueError):
        pkg.plate.quarter_plate(10, 21)


def test_symmetry_dirichlet_and_batch(pkg):
    p = pkg.plate.quarter_plate(6, 12)
    d, v = pkg.plate.symmetry_dirichlet(p)
    assert (np.diff(d) > 0).all() and not v.any()
    assert d.size == 7 + 7
    b1 = pkg.plate.random_batch(64, seed=2026)
    b2 = pkg.plate.random_batch(64, seed=2026)
    assert b1 == b2 and len(b1) == 64
    assert all(20 <= s.n_r <= 200 and s.n_theta == 2 * s.n_r and 0.5 <= s.a <= 2.0 for s in b1)


def _header_symbols():
    src = open(os.path.join(REPO, "include", "cstfem_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cstg_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg, gpu_lib):
    syms = _header_symbols()
    assert len(syms) >= 20
    lib = ctypes.CDLL(pkg.native.library_path())
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.native.library_path()],
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(cstg_[a-z_0-9]+)\b", out))
    assert set(syms) <= exported


def test_library_is_built_for_sm100a_only(pkg):
    """The build compiles every source for sm_100a and nothing else (the runtime check of the
    loaded kernels' architecture is tests/test_gpu_pcg.py::test_kernels_are_sm100a)."""
    flags = pkg.build._flags()
    assert flags[flags.index("-gencode") + 1] == "arch=compute_100a,code=sm_100a"
    assert flags.count("-gencode") == 1 and not any(f.startswith("-arch") for f in flags)


def test_host_only_calls(pkg, gpu_lib):
    o = pkg.native.default_options()
    assert o.rtol == 1e-10 and o.max_iter == 20000 and o.precision == 0
    assert gpu_lib.cstg_version() >= 1
    import torch
    if not torch.cuda.is_available():
        st = ctypes.c_int(0)
        assert gpu_lib.cstg_create(0, ctypes.byref(st)) is None
        assert st.value == pkg.native.ERR_CUDA


def test_host_mirror(pkg, oracle):
    for plane in (0, 1):
        for E, nu in ((1.0, 0.3), (210e9, 0.3), (0.7, 0.45)):
            assert np.array_equal(pkg.constitutive_matrix(E, nu, plane),
                                  oracle.constitutive_matrix(E, nu, bool(plane)))
    d = pkg.DirichletDofs()
    d.add(4, 1.0)
    d.add(4, 1.0)
    assert d.size() == 1
    with pytest.raises(pkg.CstgError, match=r"conflicting Dirichlet values for node 2 \(0-based\) component ux"):
        d.add(4, 2.0)
    p = pkg.plate.quarter_plate(4, 8)
    with pytest.raises(pkg.CstgError, match="unknown boundary group 'nowhere'"):
        pkg.add_dirichlet_group(p, "nowhere", 0, 0.0, pkg.DirichletDofs())
    dd = pkg.DirichletDofs()
    pkg.add_dirichlet_group(p, "left_sym", 0, 0.0, dd)
    pkg.add_dirichlet_group(p, "bottom_sym", 1, 0.0, dd)
    a, v = dd.arrays()
    assert np.array_equal(a, pkg.plate.symmetry_dirichlet(p)[0])
    o = pkg.SolverOptions(precision="mixed", true_residual_stop=True).native()
    assert o.precision == 1 and o.true_residual_stop == 1
