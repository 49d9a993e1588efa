"""GPU Jacobi-PCG against the reference (golden fixtures) and the oracle.

Tolerance: displacements within relative 1e-8 (2-norm) of the reference's FP64 serial CG at
the same rtol, the correctness bar of this path; the iteration count within 2 %. The only
difference in arithmetic is the summation order of the dot products (tree reductions).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _dense_csr(pkg, A):
    n = A.shape[0]
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    cols = np.tile(np.arange(n, dtype=np.int32), n)
    return pkg.GpuCsrMatrix.from_csr(rp, cols, A.reshape(-1))


def test_random_spd_vs_reference(pkg, gpu_lib, golden):
    # test_pcg.cpp:75-102 (numpy-seeded construction): error vs direct < 1e-9
    g = golden("spd")
    for n in (5, 40, 120):
        A, b = g[f"A{n}"], g[f"b{n}"]
        K = _dense_csr(pkg, A)
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=1000, record_history=True))
        s.setup(K)
        x = np.zeros(n)
        st = s.solve(b, x)
        xd = np.linalg.solve(A, b)
        assert st.converged and st.rel_residual < 1e-12
        assert np.abs(x - xd).max() / np.abs(xd).max() < 1e-9
        assert abs(st.iterations - int(g[f"iters{n}"])) <= max(2, 0.02 * st.iterations)
        assert len(st.residual_history) == st.iterations + 1
        assert st.residual_history[0] == 1.0 and st.residual_history[-1] < 1e-12
        assert st.message.startswith(f"converged in {st.iterations} iterations")
        K.ctx.close()


def test_edge_cases(pkg, gpu_lib, golden):
    A = golden("spd")["A40"]
    K = _dense_csr(pkg, A)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    x = np.full(40, 123.0)
    st = s.solve(np.zeros(40), x)  # zero right-hand side (test_pcg.cpp:104-113)
    assert st.converged and st.iterations == 0 and not x.any()
    assert st.message == "zero right-hand side, x = 0"
    s2 = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-14, max_iter=2))
    s2.setup(K)
    st = s2.solve(np.ones(40))  # max_iter (test_pcg.cpp:115-128)
    assert not st.converged and st.iterations == 2 and "NOT converged" in st.message
    assert st.true_rel_residual > 0.0 and not st.warning
    with pytest.raises(pkg.LogicError, match="before setup"):
        pkg.CgJacobiSolver().solve(np.ones(3))
    bad = pkg.GpuCsrMatrix.from_csr([0, 2, 4], [0, 1, 0, 1], [2.0, 1.0, 1.0, -1.0], ctx=K.ctx)
    with pytest.raises(pkg.CstgError, match="non-positive diagonal at row 1"):  # test_pcg.cpp:204-208
        pkg.CgJacobiSolver().setup(bad)
    # indefinite matrix with a positive diagonal: breakdown p'Ap <= 0 (solver.cpp:65-71)
    ind = pkg.GpuCsrMatrix.from_csr([0, 2, 4], [0, 1, 0, 1], [1.0, 3.0, 3.0, 1.0], ctx=K.ctx)
    s3 = pkg.CgJacobiSolver()
    s3.setup(ind)
    st = s3.solve(np.array([1.0, -1.0]))
    assert not st.converged and st.status == pkg.native.SOLVE_BREAKDOWN
    assert st.message.startswith("CG breakdown at iteration 1: p'Ap = ")
    K.ctx.close()


@pytest.mark.parametrize("name,plane", [("kirsch_L0", "stress"), ("kirsch_L0", "strain"),
                                        ("kirsch_L1", "stress"), ("kirsch_L1", "strain")])
def test_kirsch_solution_vs_reference(pkg, gpu_lib, golden, name, plane):
    g = golden(name)
    mesh = g.mesh(pkg)
    K = pkg.build_stiffness_pattern(mesh)
    pkg.assemble_stiffness(mesh, pkg.constitutive_matrix(210e9, 0.3, plane == "strain"), 0.01, K)
    b = g[f"{plane}_f"].copy()
    pkg.apply_dirichlet((g["dir_dofs"], g["dir_vals"]), K, b)
    for rtol, rt in ((1e-10, "10"), (1e-12, "12")):
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=rtol, record_history=True))
        s.setup(K)
        x = np.zeros(mesh.num_dofs)
        st = s.solve(b, x)
        ref_it = g.meta[f"{plane}_iters{rt}"]
        assert st.converged and abs(st.iterations - ref_it) <= max(2, 0.02 * ref_it)
        assert _rel(x, g[f"{plane}_u{rt}"]) < REL_TOL
        assert st.true_rel_residual < 10 * rtol and not st.warning
    K.ctx.close()


def test_plate_40x80_solution_and_scf(pkg, gpu_lib, golden):
    g = golden("plate_40x80")
    p = pkg.plate.quarter_plate(40, 80)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(p), K, b)
    st = pkg.pcg_jacobi(K, b, x := np.zeros(p.num_dofs))
    assert st.converged and abs(st.iterations - g.meta["iters"]) <= 0.02 * g.meta["iters"]
    assert _rel(x, g["u"]) < REL_TOL
    es = pkg.compute_element_stresses(K, x, 1.0, 0.3)
    scf, e = pkg.scf_at_hole(es, 1.0)
    assert e == g.meta["scf_element"] and abs(scf - g.meta["scf"]) < 1e-8
    assert 3.0 < scf < 3.2  # finite plate: slightly above Kirsch's 3
    K.ctx.close()


def test_element_stresses_bitexact(pkg, gpu_lib, golden):
    from conftest import sha
    g = golden("kirsch_L0")
    mesh = g.mesh(pkg)
    K = pkg.build_stiffness_pattern(mesh)
    for plane, tag in ((0, "stress"), (1, "strain")):
        es = pkg.compute_element_stresses(K, g[f"{tag}_u10"], 210e9, 0.3, plane)
        for k in ("sxx", "syy", "txy", "von_mises", "szz", "cx", "cy", "area"):
            assert sha(es[k]) == g.meta[f"{tag}_stress_{k}_sha"], k
    K.ctx.close()


def test_spmv_vs_oracle(pkg, gpu_lib, oracle):
    p = pkg.plate.quarter_plate(30, 60)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.3, 0.25, 1), 1.0, K)
    rp, cols, vals = K.download()
    x = np.random.default_rng(0).standard_normal(p.num_dofs)
    y = K.multiply(x)
    y_o = oracle.multiply(rp, cols, vals, x)
    assert np.abs(y - y_o).max() <= 1e-13 * np.abs(y_o).max()
    C = pkg.GpuCsrMatrix.from_csr(rp, cols, vals)  # same matrix on the scalar-CSR path
    assert np.abs(C.multiply(x) - y_o).max() <= 1e-13 * np.abs(y_o).max()
    K.ctx.close()
    C.ctx.close()


def test_device_vectors(pkg, gpu_lib):
    import torch
    p = pkg.plate.quarter_plate(20, 40)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    d, v = pkg.plate.symmetry_dirichlet(p)
    bd = torch.from_numpy(b).cuda()
    pkg.apply_dirichlet((torch.from_numpy(d).cuda(), torch.from_numpy(v).cuda()), K, bd)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    xd = torch.zeros_like(bd)
    st = s.solve(bd, xd)
    x = np.zeros(p.num_dofs)
    st2 = s.solve(bd.cpu().numpy(), x)
    assert st.converged and st.iterations == st2.iterations
    assert np.array_equal(xd.cpu().numpy(), x)  # deterministic reductions: same bits
    K.ctx.close()


def test_true_residual_stop_on_2m_plate(pkg, gpu_lib):
    """The 2M-DOF plate at rtol 1e-10 on the FP64 TRUE residual (residual replacement), and
    the reference's rule side by side: same matrix, both converge, solutions agree."""
    p = pkg.plate.quarter_plate(565, 1766)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(p), K, b)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=100000, true_residual_stop=True))
    s.setup(K)
    x = np.zeros(p.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual < 1e-10
    r = b - K.multiply(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    s2 = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=100000))
    s2.setup(K)
    x2 = np.zeros(p.num_dofs)
    st2 = s2.solve(b, x2)
    assert st2.converged and st2.iterations <= st.iterations
    assert _rel(x2, x) < REL_TOL
    es = pkg.compute_element_stresses(K, x, 1.0, 0.3)
    scf, _ = pkg.scf_at_hole(es, 1.0)
    assert 3.0 < scf < 3.1
    K.ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_matches_graph_path(pkg, gpu_lib, golden, precision):
    """The persistent cooperative kernel (default for mesh matrices) and the graph-replayed
    per-phase kernels run the same recurrence: same convergence, solutions within 1e-10."""
    g = golden("plate_40x80")
    p = pkg.plate.quarter_plate(40, 80)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(p), K, b)
    out = {}
    for launch in ("graph", "persistent"):
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, precision=precision, launch=launch,
                                                 record_history=True))
        s.setup(K)
        x = np.zeros(p.num_dofs)
        out[launch] = (s.solve(b, x), x)
    (sg, xg), (sp_, xp) = out["graph"], out["persistent"]
    assert sg.converged and sp_.converged
    assert abs(sg.iterations - sp_.iterations) <= 2
    assert _rel(xp, xg) < 1e-10 and _rel(xp, g["u"]) < REL_TOL
    assert len(sp_.residual_history) == sp_.iterations + 1
    K.ctx.close()


def test_true_residual_warning(pkg, gpu_lib, golden, oracle):
    """The reference's warning path (solver.cpp:123-129, tests/test_pcg.cpp:130-181): with an rtol
    below what FP64 can reach on an ill-conditioned SPD system (D A D, diagonal spread over three
    decades), the recursive residual converges while the true residual stays above 10 rtol. The
    GPU solver (a caller CSR on the graph path) reports it with the reference's text, as does the
    CPU oracle on the same system; a reachable rtol gives no warning."""
    g = golden("spd")
    A, b = g["A120"], g["b120"]
    n = b.size
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    cols = np.tile(np.arange(n, dtype=np.int32), n)
    K = pkg.GpuCsrMatrix.from_csr(rp, cols, A.reshape(-1))
    rtol = 1e-19
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=rtol, max_iter=5000, launch="graph"))
    s.setup(K)
    x = np.zeros(n)
    st = s.solve(b, x)
    _, so = oracle.pcg_jacobi(rp, cols, A.reshape(-1), b, rtol=rtol, max_iter=5000)
    assert so["converged"] and so["true_rel_residual"] > 10 * rtol  # the same situation on the CPU
    assert st.converged and st.true_rel_residual > 10 * rtol, st.message
    assert st.warning.startswith("WARNING: CG recursive residual converged (")
    assert "but the true residual ||b - Ax|| / ||b|| = " in st.warning and "exceeds 10 * rtol = 1e-18" in st.warning
    s2 = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=5000, launch="graph"))
    s2.setup(K)
    st2 = s2.solve(b, np.zeros(n))
    assert st2.converged and not st2.warning
    K.ctx.close()


def test_kernels_are_sm100a(pkg, gpu_lib):
    """The CUDA runtime reports the loaded kernels' architecture as sm_100 (binaryVersion 100)."""
    import ctypes as C
    v = C.c_int(0)
    assert gpu_lib.cstg_binary_version(0, C.byref(v)) == pkg.native.OK
    assert v.value == 100
