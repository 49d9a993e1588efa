"""GPU pattern + assembly + Dirichlet elimination, bit-for-bit against the reference
(golden fixtures) and the oracle, plus size-independent properties at the 2M-DOF plate."""
import numpy as np
import pytest

from conftest import sha

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_kirsch_meshes_bitexact(pkg, gpu_lib, golden, name):
    g = golden(name)
    mesh = g.mesh(pkg)
    K = pkg.build_stiffness_pattern(mesh)
    for plane, tag in ((0, "stress"), (1, "strain")):
        pkg.assemble_stiffness(mesh, pkg.constitutive_matrix(210e9, 0.3, plane), 0.01, K)
        rp, cols, vals = K.download()
        assert sha(rp) == g.meta["row_ptr_sha"] and sha(cols) == g.meta["cols_sha"]
        assert sha(vals) == g.meta[f"{tag}_K_sha"]
        f = np.zeros(mesh.num_dofs)
        pkg.add_traction(K, mesh.boundary_edges["right"], 0.01, 100e6, 0.0, f)
        assert _bits_equal(f, g[f"{tag}_f"])
        pkg.apply_dirichlet((g["dir_dofs"], g["dir_vals"]), K, f)
        _, _, kbc = K.download()
        assert sha(kbc) == g.meta[f"{tag}_Kbc_sha"]
        assert _bits_equal(f, g[f"{tag}_b"])
    K.ctx.close()


def test_plate_40x80_bitexact(pkg, gpu_lib, golden):
    g = golden("plate_40x80")
    p = pkg.plate.quarter_plate(40, 80)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    rp, cols, vals = K.download()
    assert sha(rp) == g.meta["row_ptr_sha"] and sha(cols) == g.meta["cols_sha"]
    assert sha(vals) == g.meta["K_sha"]
    f = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, f)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(p), K, f)
    assert sha(K.download()[2]) == g.meta["Kbc_sha"] and sha(f) == g.meta["b_sha"]
    K.ctx.close()


def _permuted_plate(pkg, n_r, n_t, seed):
    """A plate whose nodes and triangles are randomly renumbered (no structured ordering)."""
    rng = np.random.default_rng(seed)
    p = pkg.plate.quarter_plate(n_r, n_t, a=float(rng.uniform(0.5, 2.0)))
    perm = rng.permutation(p.num_nodes)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    xy = p.xy.reshape(-1, 2)[perm].reshape(-1).copy()
    tri = inv[p.triangles.reshape(-1, 3)]
    tri = tri[rng.permutation(tri.shape[0])]
    rot = rng.integers(0, 3, tri.shape[0])  # rotate corner order, keeps orientation
    tri = np.stack([np.roll(t, -r) for t, r in zip(tri, rot)]).astype(np.int32).reshape(-1)
    groups = {k: inv[v].astype(np.int32) for k, v in p.boundary_edges.items()}
    return pkg.plate.Mesh(xy=xy, triangles=tri, boundary_edges=groups)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_plates_bitexact_vs_oracle(pkg, gpu_lib, oracle, seed):
    rng = np.random.default_rng(100 + seed)
    mesh = _permuted_plate(pkg, int(rng.integers(3, 30)), 2 * int(rng.integers(2, 30)), seed)
    E, nu, plane = float(rng.uniform(0.5, 2.0)), float(rng.uniform(0.2, 0.45)), int(rng.integers(0, 2))
    D = pkg.constitutive_matrix(E, nu, plane)
    rp_o, cols_o = oracle.build_stiffness_pattern(mesh.num_nodes, mesh.triangles)
    vals_o = oracle.assemble_stiffness(mesh.xy, mesh.triangles, D, 0.7, rp_o, cols_o)
    K = pkg.build_stiffness_pattern(mesh)
    pkg.assemble_stiffness(mesh, D, 0.7, K)
    rp, cols, vals = K.download()
    assert np.array_equal(rp, rp_o) and np.array_equal(cols, cols_o)
    assert _bits_equal(vals, vals_o)
    f = np.zeros(mesh.num_dofs)
    f_o = f.copy()
    pkg.add_traction(K, mesh.boundary_edges["top"], 0.7, 0.3, -1.1, f)
    oracle.add_traction(mesh.xy, mesh.triangles, mesh.boundary_edges["top"], 0.7, 0.3, -1.1, f_o)
    assert _bits_equal(f, f_o)
    dofs, vals_d = pkg.plate.symmetry_dirichlet(mesh)
    vals_d = rng.uniform(-1e-3, 1e-3, vals_d.size)  # non-homogeneous prescribed values
    pkg.apply_dirichlet((dofs, vals_d), K, f)
    oracle.apply_dirichlet(rp_o, cols_o, vals_o, dofs, vals_d, f_o)
    assert _bits_equal(K.download()[2], vals_o) and _bits_equal(f, f_o)
    K.ctx.close()


def test_symmetric_elimination_known_answer(pkg, gpu_lib):
    # test_bc.cpp:169-184 on the generic CSR path
    K = pkg.GpuCsrMatrix.from_csr([0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2], [4, 1, 1, 3, 1, 1, 2])
    b = np.ones(3)
    d = pkg.DirichletDofs()
    d.add(1, 2.0)
    pkg.apply_dirichlet(d, K, b)
    assert b.tolist() == [-1.0, 6.0, -1.0]
    assert K.download()[2].tolist() == [4, 0, 0, 3, 0, 0, 2]
    K.ctx.close()


def test_error_paths(pkg, gpu_lib):
    p = pkg.plate.quarter_plate(4, 8)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    with pytest.raises(pkg.CstgError, match=r"DOF 9999 out of range"):
        pkg.apply_dirichlet((np.array([3, 9999], np.int32), np.zeros(2)), K, b)
    with pytest.raises(pkg.CstgError, match=r"conflicting Dirichlet values for node 1 \(0-based\) component uy"):
        pkg.apply_dirichlet((np.array([3, 3], np.int32), np.array([0.0, 1.0])), K, b)
    bad = pkg.plate.Mesh(xy=p.xy, triangles=np.where(p.triangles == 5, 10 ** 6, p.triangles).astype(np.int32),
                         boundary_edges=p.boundary_edges)
    with pytest.raises(pkg.CstgError, match="node index outside"):
        pkg.build_stiffness_pattern(bad, ctx=K.ctx)
    with pytest.raises(pkg.LogicError):
        pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)  # K now has no pattern
    # non-positive diagonal on a prescribed row (bc.cpp:151-153)
    Z = pkg.GpuCsrMatrix.from_csr([0, 1, 2], [0, 1], [1.0, 0.0])
    with pytest.raises(pkg.CstgError, match="non-positive diagonal at DOF 1"):
        pkg.apply_dirichlet((np.array([1], np.int32), np.array([1.0])), Z, np.zeros(2))
    K.ctx.close()
    Z.ctx.close()


def test_empty_and_isolated(pkg, gpu_lib):
    empty = pkg.plate.Mesh(xy=np.zeros(0), triangles=np.zeros(0, np.int32), boundary_edges={})
    K = pkg.build_stiffness_pattern(empty)
    assert K.nnz() == 0 and K.num_rows == 0
    # one triangle plus an isolated node: the isolated node keeps its own 2x2 block
    m = pkg.plate.Mesh(xy=np.array([0, 0, 1, 0, 0, 1, 5, 5.0]), triangles=np.array([0, 1, 2], np.int32),
                       boundary_edges={})
    K2 = pkg.build_stiffness_pattern(m, ctx=K.ctx)
    rp, cols, _ = K2.download(values=False)
    assert K2.nnz() == 4 * (4 + 2 * 3) and cols[rp[6]:rp[7]].tolist() == [6, 7]
    K.ctx.close()


def test_reference_triangle_known_answer(pkg, gpu_lib):
    """The reference's element known answer (its tests/test_element.cpp:60-84) through the GPU
    pattern and assembly: one triangle (0,0), (1,0), (0,1), E = 1, nu = 0, t = 1, plane stress;
    the assembled 6 x 6 matrix equals the closed-form Ke within 1e-14."""
    expected = np.array([[0.75, 0.25, -0.5, -0.25, -0.25, 0.0],
                         [0.25, 0.75, 0.0, -0.25, -0.25, -0.5],
                         [-0.5, 0.0, 0.5, 0.0, 0.0, 0.0],
                         [-0.25, -0.25, 0.0, 0.25, 0.25, 0.0],
                         [-0.25, -0.25, 0.0, 0.25, 0.25, 0.0],
                         [0.0, -0.5, 0.0, 0.0, 0.0, 0.5]])
    m = pkg.plate.Mesh(xy=np.array([0, 0, 1, 0, 0, 1.0]), triangles=np.array([0, 1, 2], np.int32),
                       boundary_edges={})
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, pkg.constitutive_matrix(1.0, 0.0), 1.0, K)
    rp, cols, vals = K.download()
    Kd = np.zeros((6, 6))
    for i in range(6):
        Kd[i, cols[rp[i]:rp[i + 1]]] = vals[rp[i]:rp[i + 1]]
    assert np.max(np.abs(Kd - expected)) <= 1e-14
    K.ctx.close()


@pytest.fixture(scope="module")
def big_plate(pkg):
    return pkg.plate.quarter_plate(565, 1766)  # 2,000,244 DOFs


def test_full_size_assembly_properties(pkg, gpu_lib, big_plate):
    """Size-independent checks on the 2M-DOF plate: nnz = 4 (nodes + 2 edges), K exactly
    symmetric (same contributions, same order for (i, j) and (j, i)), rigid-body modes in
    the null space (test_csr.cpp:64-98) and the 2x2 block layout."""
    p = big_plate
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    rp, cols, vals = K.download()
    n_r, n_t = 565, 1766
    edges = n_r * (n_t + 1) + (n_r + 1) * n_t + n_r * n_t
    assert cols.size == 4 * (p.num_nodes + 2 * edges)
    import scipy.sparse as sp
    A = sp.csr_matrix((vals, cols, rp), shape=(p.num_dofs, p.num_dofs))
    assert (A != A.T).nnz == 0
    P = p.xy.reshape(-1, 2)
    knorm = np.abs(A).sum(axis=1).max()
    for r in (np.tile([1.0, 0.0], p.num_nodes), np.tile([0.0, 1.0], p.num_nodes),
              np.stack([-P[:, 1], P[:, 0]], axis=1).reshape(-1)):
        y = K.multiply(r)
        assert np.abs(y).max() / (knorm * np.abs(r).max()) <= 1e-12
    K.ctx.close()
