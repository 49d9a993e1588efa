"""Batched solves: many plates of uneven size x load cases in one persistent launch, checked
plate by plate against the oracle.

Bars (the batch is the reference's single-plate path applied to every plate and load case):
* each plate's block of K and each eliminated load vector are bit-identical to the oracle's
  single-plate assembly (assembly.cpp:54-74), traction loads (bc.cpp:190-253) and
  elimination (bc.cpp:137-166);
* every (plate, load case) converged on the FP64 true residual <= 1e-10, recomputed here on the
  host from the downloaded matrix;
* displacements within relative 1e-8 of the oracle's FP64 Jacobi-PCG at rtol 1e-10;
* for a fixed launch shape the results are the same bits on every run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _oracle_plate(oracle, pkg, spec, cases):
    m = pkg.plate.quarter_plate(spec.n_r, spec.n_theta, a=spec.a)
    D = oracle.constitutive_matrix(spec.E, spec.nu, spec.plane_strain)
    rp, cols = oracle.build_stiffness_pattern(m.num_nodes, m.triangles)
    vals = oracle.assemble_stiffness(m.xy, m.triangles, D, 1.0, rp, cols)
    d, v = pkg.plate.symmetry_dirichlet(m)
    bs, K = [], None
    for parts in cases.values():
        f = np.zeros(m.num_dofs)
        for g, tx, ty in parts:
            oracle.add_traction(m.xy, m.triangles, m.boundary_edges[g], 1.0, tx, ty, f)
        kv = vals.copy()
        oracle.apply_dirichlet(rp, cols, kv, d, v, f)
        bs.append(f)
        K = kv
    return rp, cols, K, bs


def _host_true_residuals(batch, K, b, x):
    """||b - K x|| / ||b|| per (plate, case) from the downloaded CSR (scipy, FP64)."""
    import scipy.sparse as sp
    rp, cols, vals = K.download()
    A = sp.csr_matrix((vals, cols, rp), shape=(rp.size - 1, rp.size - 1))
    out = np.zeros((batch.n_plates, batch.n_cases))
    for q in range(batch.n_cases):
        r = b[q] - A @ x[q]
        for s in range(batch.n_plates):
            sl = batch.dof_range(s)
            out[s, q] = np.linalg.norm(r[sl]) / np.linalg.norm(b[q][sl])
    return out


@pytest.fixture(scope="module")
def small(pkg, gpu_lib):
    specs = pkg.plate.random_batch(count=5, seed=7, n_r_range=(4, 14))
    batch = pkg.build_batch(specs)
    solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=100000))
    K = solver.setup(batch)
    yield specs, batch, solver, K
    solver.close()


def test_batch_matches_oracle_per_plate(pkg, oracle, small):
    specs, batch, solver, K = small
    rp_all, cols_all, vals_all = K.download()
    sol = solver.solve()
    assert sol.x.shape == (4, batch.mesh.num_dofs)
    for s, spec in enumerate(specs):
        rp, cols, Kel, bs = _oracle_plate(oracle, pkg, spec, pkg.plate.LOAD_CASES)
        sl = batch.dof_range(s)
        lo, hi = rp_all[sl.start], rp_all[sl.stop]
        assert np.array_equal(rp_all[sl.start:sl.stop + 1] - lo, rp)
        assert np.array_equal(cols_all[lo:hi] - sl.start, cols)
        assert np.array_equal(vals_all[lo:hi], Kel)
        for q in range(4):
            assert np.array_equal(solver.b[q][sl], bs[q])
            x_ref, st = oracle.pcg_jacobi(rp, cols, Kel, bs[q], rtol=1e-10, max_iter=100000)
            assert st["converged"]
            assert sol.status[s, q] == pkg.native.SOLVE_CONVERGED
            assert sol.true_rel_residual[s, q] <= 1e-10
            assert _rel(sol.x[q][sl], x_ref) < REL_TOL, (s, q)
    host = _host_true_residuals(batch, K, solver.b, sol.x)
    assert np.all(host <= 1.0001e-10), host


def test_batch_shapes_and_determinism(pkg, small):
    specs, batch, solver, K = small
    a = solver.solve(config=(2, 256))
    b = solver.solve(config=(2, 256))
    assert np.array_equal(a.x, b.x) and np.array_equal(a.iterations, b.iterations)
    c = solver.solve(config=(16, 512))
    d = solver.solve(config=(1, 512))
    for sol in (a, c, d):
        assert np.all(sol.converged) and np.all(sol.true_rel_residual <= 1e-10)
    for q in range(4):
        assert _rel(c.x[q], a.x[q]) < REL_TOL and _rel(d.x[q], a.x[q]) < REL_TOL


def test_batch_fp64_and_autotune(pkg, small):
    specs, batch, solver, K = small
    mixed = solver.solve()
    s64 = pkg.BatchSolver(pkg.SolverOptions(precision="fp64", max_iter=100000))
    s64.setup(batch, device_rhs=True)
    sol = s64.solve(device=True)
    x = sol.x.cpu().numpy()
    assert np.all(sol.converged) and np.all(sol.fp64 == 1)
    for q in range(4):
        assert _rel(x[q], mixed.x[q]) < REL_TOL
    cfg, sec = s64.autotune(max_iter=200)
    assert cfg in {(c, t) for c in (1, 2, 4, 8, 16) for t in (256, 512)} and sec > 0
    again = s64.solve(device=True)
    assert again.config == cfg and np.all(again.converged)
    s64.close()


def test_batch_many_load_cases_linearity(pkg, gpu_lib):
    """Six load cases (two groups: 4 + 2): a doubled load gives a doubled displacement."""
    specs = pkg.plate.random_batch(count=3, seed=11, n_r_range=(6, 10))
    cases = dict(pkg.plate.LOAD_CASES)
    cases["tension_x_twice"] = [("right", 2.0, 0.0)]
    cases["compression_y"] = [("top", 0.0, -1.0)]
    batch = pkg.build_batch(specs, cases)
    solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=100000))
    solver.setup(batch)
    sol = solver.solve()
    assert sol.iterations.shape == (3, 6) and np.all(sol.converged)
    assert _rel(sol.x[4], 2.0 * sol.x[0]) < REL_TOL
    assert _rel(sol.x[5], -sol.x[1]) < REL_TOL
    solver.close()


def test_batch_rejects_coupled_systems(pkg, small):
    specs, batch, solver, K = small
    offs = batch.node_offsets.copy()
    offs[1] -= 3  # splits plate 0: its last nodes now "belong" to plate 1 but couple to plate 0
    bad = pkg.PlateBatch(**{**batch.__dict__, "node_offsets": offs})
    solver.batch = bad
    try:
        with pytest.raises(pkg.CstgError, match="coupled"):
            solver.solve()
    finally:
        solver.batch = batch
    assert np.all(solver.solve().converged)


def test_batch_64_plates_4_load_cases(pkg, oracle, gpu_lib):
    """The uneven batch workload: 64 seeded plates (n_r 20..200, n_theta = 2 n_r), 4 load cases,
    one persistent launch. Every system converged on the host-recomputed FP64 true residual; a
    stratified sample of 8 plates by size (the smallest and the largest included) checked against
    the oracle's FP64 Jacobi-PCG: every load case of the smallest and the largest, one case each
    (in turn) of the six between."""
    specs = pkg.plate.random_batch(count=64, seed=2026)
    batch = pkg.build_batch(specs)
    solver = pkg.BatchSolver(pkg.SolverOptions(precision="mixed", max_iter=200000))
    K = solver.setup(batch)
    sol = solver.solve()
    assert np.all(sol.converged), sol.status
    host = _host_true_residuals(batch, K, solver.b, sol.x)
    assert np.all(host <= 1.0001e-10), host.max()
    sizes = batch.node_offsets[1:] - batch.node_offsets[:-1]
    order = np.argsort(sizes, kind="stable")
    sample = [int(order[int(round(k * (len(order) - 1) / 7))]) for k in range(8)]
    assert sample[0] == int(order[0]) and sample[-1] == int(order[-1]) and len(set(sample)) == 8
    for i, s in enumerate(sample):
        rp, cols, Kel, bs = _oracle_plate(oracle, pkg, specs[s], pkg.plate.LOAD_CASES)
        cases = range(4) if i in (0, 7) else [i % 4]
        for q in cases:
            x_ref, _ = oracle.pcg_jacobi(rp, cols, Kel, bs[q], rtol=1e-10, max_iter=100000)
            assert _rel(sol.x[q][batch.dof_range(s)], x_ref) < REL_TOL, (s, q)
    solver.close()
