"""The CPU oracle (oracle/cst_oracle.c) pinned against the reference.

Two kinds of pins: the reference's own known answers (tests/test_element.cpp,
tests/test_bc.cpp, tests/test_pcg.cpp, tests/test_csr.cpp of FreddyJuka/mpi-cst-fem-solver),
and bit-for-bit equality with outputs of the reference's compiled serial core stored under
tests/golden/ (made by tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from conftest import sha


def test_ke_reference_triangle(oracle):
    # test_element.cpp:60-84: (0,0), (1,0), (0,1); E = 1, nu = 0, t = 1, plane stress.
    expected = np.array([0.75, 0.25, -0.5, -0.25, -0.25, 0.0,
                         0.25, 0.75, 0.0, -0.25, -0.25, -0.5,
                         -0.5, 0.0, 0.5, 0.0, 0.0, 0.0,
                         -0.25, -0.25, 0.0, 0.25, 0.25, 0.0,
                         -0.25, -0.25, 0.0, 0.25, 0.25, 0.0,
                         0.0, -0.5, 0.0, 0.0, 0.0, 0.5])
    K = oracle.cst_stiffness([0, 0, 1, 0, 0, 1], oracle.constitutive_matrix(1.0, 0.0), 1.0)
    assert np.max(np.abs(K - expected)) <= 1e-14


def test_constitutive_closed_form(oracle):
    # test_element.cpp:121-136
    Ds = oracle.constitutive_matrix(1.0, 0.3, False)
    De = oracle.constitutive_matrix(1.0, 0.3, True)
    Ds_ref = np.array([1 / 0.91, 0.3 / 0.91, 0, 0.3 / 0.91, 1 / 0.91, 0, 0, 0, 0.35 / 0.91])
    De_ref = np.array([0.7 / 0.52, 0.3 / 0.52, 0, 0.3 / 0.52, 0.7 / 0.52, 0, 0, 0, 0.2 / 0.52])
    assert np.max(np.abs(Ds - Ds_ref)) <= 1e-15
    assert np.max(np.abs(De - De_ref)) <= 1e-15
    assert De[0] > Ds[0]


def test_ke_golden_bitexact(oracle, golden):
    g = golden("element")
    for plane in (0, 1):
        D = oracle.constitutive_matrix(210e9, 0.3, bool(plane))
        assert np.array_equal(D, g[f"D{plane}"])
        for t, Kref in zip(g["xy"], g[f"K{plane}"]):
            K = oracle.cst_stiffness(t, D, 0.01)
            assert np.array_equal(K.view(np.int64), Kref.view(np.int64))


def test_ke_properties(oracle, golden):
    # test_element.cpp:86-119: exact symmetry, rigid-body modes, positive strain energy
    g = golden("element")
    for plane in (0, 1):
        for t, K in zip(g["xy"], g[f"K{plane}"]):
            K = K.reshape(6, 6)
            assert np.array_equal(K, K.T)
            kmax = np.abs(K).max()
            tx = np.tile([1.0, 0.0], 3)
            ty = np.tile([0.0, 1.0], 3)
            rot = np.ravel(np.stack([-t[1::2], t[0::2]], axis=1))
            rmax = np.abs(t).max()
            for r, s in ((tx, 1.0), (ty, 1.0), (rot, rmax)):
                assert np.abs(K @ r).max() <= 1e-12 * s * kmax


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_pattern_and_assembly_golden(oracle, golden, name):
    g = golden(name)
    xy, tri = g["xy"], g["tri"]
    rp, cols = oracle.build_stiffness_pattern(xy.size // 2, tri)
    assert sha(rp) == g.meta["row_ptr_sha"] and sha(cols) == g.meta["cols_sha"]
    # test_csr.cpp:36-62: nnz = 4 (nodes + 2 edges), sorted columns, diagonal present
    t = tri.reshape(-1, 3)
    e = np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), axis=1)
    n_edges = np.unique(e, axis=0).shape[0]
    assert cols.size == 4 * (xy.size // 2 + 2 * n_edges)
    for i in range(rp.size - 1):
        row = cols[rp[i]:rp[i + 1]]
        assert np.all(np.diff(row) > 0) and i in row
    for plane, tag in ((False, "stress"), (True, "strain")):
        D = oracle.constitutive_matrix(210e9, 0.3, plane)
        vals = oracle.assemble_stiffness(xy, tri, D, 0.01, rp, cols)
        assert sha(vals) == g.meta[f"{tag}_K_sha"]


def test_symmetric_elimination_known_answer(oracle):
    # test_bc.cpp:169-184
    rp = np.array([0, 2, 5, 7], dtype=np.int32)
    cols = np.array([0, 1, 0, 1, 2, 1, 2], dtype=np.int32)
    vals = np.array([4, 1, 1, 3, 1, 1, 2], dtype=np.float64)
    b = np.ones(3)
    oracle.apply_dirichlet(rp, cols, vals, [1], [2.0], b)
    assert b.tolist() == [-1.0, 6.0, -1.0]
    assert vals.tolist() == [4, 0, 0, 3, 0, 0, 2]


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_loads_dirichlet_pcg_golden(oracle, golden, name):
    g = golden(name)
    xy, tri = g["xy"], g["tri"]
    rp, cols = oracle.build_stiffness_pattern(xy.size // 2, tri)
    for plane, tag in ((False, "stress"), (True, "strain")):
        D = oracle.constitutive_matrix(210e9, 0.3, plane)
        vals = oracle.assemble_stiffness(xy, tri, D, 0.01, rp, cols)
        f = np.zeros(xy.size)
        oracle.add_traction(xy, tri, g["group_right"], 0.01, 100e6, 0.0, f)
        assert np.array_equal(f, g[f"{tag}_f"])
        oracle.apply_dirichlet(rp, cols, vals, g["dir_dofs"], g["dir_vals"], f)
        assert sha(vals) == g.meta[f"{tag}_Kbc_sha"]
        assert np.array_equal(f, g[f"{tag}_b"])
        for rtol, rt in ((1e-10, "10"), (1e-12, "12")):
            x, st = oracle.pcg_jacobi(rp, cols, vals, f, rtol, 20000, record_history=True)
            assert st["iterations"] == g.meta[f"{tag}_iters{rt}"]
            assert np.array_equal(x, g[f"{tag}_u{rt}"])
            assert np.array_equal(st["residual_history"], g[f"{tag}_hist{rt}"])
            assert st["true_rel_residual"] == g.meta[f"{tag}_true{rt}"]
            assert st["message"] == g.meta[f"{tag}_msg{rt}"]


def test_published_iteration_counts(golden):
    # docs/VERIFICATION.md:66-67 and the plane-strain table: L0 148 / 157, L1 295 / 313 at rtol 1e-12
    assert golden("kirsch_L0").meta["stress_iters12"] == 148
    assert golden("kirsch_L1").meta["stress_iters12"] == 295
    assert golden("kirsch_L0").meta["strain_iters12"] == 157
    assert golden("kirsch_L1").meta["strain_iters12"] == 313


def test_plate_golden(oracle, golden, pkg):
    g = golden("plate_40x80")
    p = pkg.plate.quarter_plate(40, 80)
    assert sha(p.xy) == g.meta["xy_sha"] and sha(p.triangles) == g.meta["tri_sha"]
    rp, cols = oracle.build_stiffness_pattern(p.num_nodes, p.triangles)
    vals = oracle.assemble_stiffness(p.xy, p.triangles, oracle.constitutive_matrix(1.0, 0.3), 1.0, rp, cols)
    assert sha(vals) == g.meta["K_sha"]
    f = np.zeros(p.num_dofs)
    oracle.add_traction(p.xy, p.triangles, p.boundary_edges["right"], 1.0, 1.0, 0.0, f)
    d, v = pkg.plate.symmetry_dirichlet(p)
    assert np.array_equal(d, g["dir_dofs"])
    oracle.apply_dirichlet(rp, cols, vals, d, v, f)
    assert sha(vals) == g.meta["Kbc_sha"] and sha(f) == g.meta["b_sha"]
    x, st = oracle.pcg_jacobi(rp, cols, vals, f, 1e-10, 20000)
    assert st["iterations"] == g.meta["iters"] == 897
    assert np.array_equal(x, g["u"])


def test_pcg_spd_golden(oracle, golden):
    # test_pcg.cpp:75-102 construction (numpy-seeded): bit-equal to the reference, < 1e-9 vs direct
    g = golden("spd")
    for n in (5, 40, 120):
        A, b = g[f"A{n}"], g[f"b{n}"]
        rp = np.arange(0, n * n + 1, n, dtype=np.int32)
        cols = np.tile(np.arange(n, dtype=np.int32), n)
        x, st = oracle.pcg_jacobi(rp, cols, A.reshape(-1), b, 1e-12, 1000, record_history=True)
        assert st["converged"] and st["iterations"] == int(g[f"iters{n}"])
        assert np.array_equal(x, g[f"x{n}"])
        xd = np.linalg.solve(A, b)
        assert np.abs(x - xd).max() / np.abs(xd).max() < 1e-9
        assert len(st["residual_history"]) == st["iterations"] + 1
        assert st["residual_history"][0] == 1.0


def test_pcg_edge_cases(oracle, golden):
    g = golden("spd")
    A = g["A40"]
    n = 40
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    cols = np.tile(np.arange(n, dtype=np.int32), n)
    # zero right-hand side (test_pcg.cpp:104-113)
    x, st = oracle.pcg_jacobi(rp, cols, A.reshape(-1), np.zeros(n))
    assert st["converged"] and st["iterations"] == 0 and not x.any()
    # max_iter (test_pcg.cpp:115-128)
    x, st = oracle.pcg_jacobi(rp, cols, A.reshape(-1), np.ones(n), 1e-14, 2)
    assert not st["converged"] and st["iterations"] == 2 and "NOT converged" in st["message"]
    # non-positive diagonal (test_pcg.cpp:204-208)
    from oracle import OracleError
    with pytest.raises(OracleError, match="non-positive diagonal"):
        oracle.pcg_jacobi(np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                          np.array([2.0, 1.0, 1.0, -1.0]), np.ones(2))


def test_traction_equilibrium(oracle, golden):
    # test_bc.cpp:213-232: the nodal forces sum to thickness * traction * length
    g = golden("kirsch_L0")
    xy, tri = g["xy"], g["tri"]
    for grp in ("hole", "left_sym", "bottom_sym", "right", "top"):
        e = g["group_" + grp]
        P = xy.reshape(-1, 2)
        length = np.hypot(*(P[e[:, 1]] - P[e[:, 0]]).T).sum()
        f = np.zeros(xy.size)
        oracle.add_traction(xy, tri, e, 0.01, 3.0e6, -2.0e6, f)
        assert abs(f[0::2].sum() - 0.01 * 3.0e6 * length) <= 1e-12 * 0.01 * 3.0e6 * length
        assert abs(f[1::2].sum() + 0.01 * 2.0e6 * length) <= 1e-12 * 0.01 * 2.0e6 * length
