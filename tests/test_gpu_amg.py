"""Smoothed-aggregation multigrid preconditioner on the GPU, checked like the other methods against
the reference's FP64 Jacobi-PCG solution.

Bars: solutions within relative 1e-8 of the reference's (rtol 1e-10, FP64 true residual);
the V-cycle is a symmetric positive operator (<Mu, v> = <u, Mv> to 1e-8 relative: the finest
smoother uses the FP32 difference-form operator, whose rounded off-diagonal blocks leave its
diagonal blocks asymmetric at the FP32 level; <Mu, u> > 0),
the hierarchy coarsens (levels >= 2, DOFs decreasing) and the solve is bit-reproducible; far
fewer iterations than Jacobi-PCG."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _plate(pkg, n_r, n_t, load="right"):
    m = pkg.plate.quarter_plate(n_r, n_t)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges[load], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    return m, K, b


def _amg(precision="fp64"):
    import importlib
    pkg = importlib.import_module("mpi-cst-fem-solver_b200")
    return pkg.SolverOptions(rtol=1e-10, max_iter=5000, precision=precision, preconditioner="amg",
                             true_residual_stop=True)


def test_amg_plate_matches_reference(pkg, gpu_lib, golden):
    g = golden("plate_40x80")
    m, K, b = _plate(pkg, 40, 80)
    s = pkg.CgJacobiSolver(_amg())
    s.setup(K)
    info = pkg.amg_setup(K)
    assert info["levels"] >= 2 and all(a > c for a, c in zip(info["dofs"], info["dofs"][1:]))
    x1, x2 = np.zeros(m.num_dofs), np.zeros(m.num_dofs)
    st = s.solve(b, x1)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert _rel(x1, g["u"]) < REL_TOL
    assert st.iterations < g.meta["iters"] / 10, st.iterations
    st2 = s.solve(b, x2)
    assert np.array_equal(x1, x2) and st2.iterations == st.iterations
    K.ctx.close()


def test_amg_vcycle_is_symmetric_positive(pkg, gpu_lib):
    import torch
    m, K, b = _plate(pkg, 30, 60)
    s = pkg.CgJacobiSolver(_amg())
    s.setup(K)
    rng = np.random.default_rng(0)
    u = torch.from_numpy(rng.standard_normal(m.num_dofs)).cuda()
    v = torch.from_numpy(rng.standard_normal(m.num_dofs)).cuda()
    Mu, Mv = pkg.amg_apply(K, u), pkg.amg_apply(K, v)
    a, c = float(torch.dot(Mu, v)), float(torch.dot(u, Mv))
    assert abs(a - c) <= 1e-8 * max(abs(a), abs(c))
    assert float(torch.dot(Mu, u)) > 0 and float(torch.dot(Mv, v)) > 0
    # timing the cycle leaves the preconditioner unchanged
    t = pkg.amg_time(K, reps=3)
    assert 0 < t["sweep_s"] < t["vcycle_s"]
    assert torch.equal(pkg.amg_apply(K, u), Mu)
    K.ctx.close()


@pytest.mark.parametrize("name", ["kirsch_L0", "kirsch_L1"])
def test_amg_kirsch_meshes(pkg, gpu_lib, golden, name):
    g = golden(name)
    mesh = g.mesh(pkg)
    K = pkg.build_stiffness_pattern(mesh)
    pkg.assemble_stiffness(mesh, pkg.constitutive_matrix(210e9, 0.3), 0.01, K)
    b = g["stress_f"].copy()
    pkg.apply_dirichlet((g["dir_dofs"], g["dir_vals"]), K, b)
    s = pkg.CgJacobiSolver(_amg("mixed"))
    s.setup(K)
    x = np.zeros(mesh.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert _rel(x, g["stress_u10"]) < REL_TOL
    K.ctx.close()


def test_amg_mixed_larger_plate(pkg, gpu_lib):
    m, K, b = _plate(pkg, 200, 400)
    ref = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=100000))
    ref.setup(K)
    x_ref = np.zeros(m.num_dofs)
    st_ref = ref.solve(b, x_ref)
    s = pkg.CgJacobiSolver(_amg("mixed"))
    s.setup(K)
    x = np.zeros(m.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert _rel(x, x_ref) < REL_TOL
    assert st.iterations * 20 < st_ref.iterations, (st.iterations, st_ref.iterations)
    K.ctx.close()


def test_amg_cluster_tail_matches_per_level_cycle(pkg, gpu_lib):
    """The one-cluster launch of the small coarse levels gives the bits of the per-level
    launches, and solves agree bit for bit either way."""
    import torch
    m, K, b = _plate(pkg, 200, 400)  # 161k DOFs: a level of ~1.4k DOFs above the dense coarsest
    s = pkg.CgJacobiSolver(_amg())
    s.setup(K)
    info = pkg.amg_setup(K)
    assert info["levels"] >= 3 and info["tail_level"] >= 1 and info["tail_cluster"] in (8, 16), info
    r = torch.from_numpy(np.random.default_rng(3).standard_normal(m.num_dofs)).cuda()
    z_tail = pkg.amg_apply(K, r)
    x_tail = np.zeros(m.num_dofs)
    st_tail = s.solve(b, x_tail)
    pkg.amg_set_tail(K, False)
    assert pkg.amg_setup(K)["tail_level"] == 0
    z_lvl = pkg.amg_apply(K, r)
    x_lvl = np.zeros(m.num_dofs)
    st_lvl = s.solve(b, x_lvl)
    assert torch.equal(z_tail, z_lvl)
    assert np.array_equal(x_tail, x_lvl) and st_tail.iterations == st_lvl.iterations
    assert st_tail.converged and st_tail.true_rel_residual <= 1e-10
    pkg.amg_set_tail(K, True)
    assert pkg.amg_setup(K)["tail_level"] == info["tail_level"]
    assert torch.equal(pkg.amg_apply(K, r), z_tail)
    K.ctx.close()


def test_amg_chebyshev_beats_jacobi_smoothing(pkg, gpu_lib):
    """Both smoothers reach the FP64 Jacobi-PCG solution; degree-2 Chebyshev (the default) needs
    fewer iterations than damped Jacobi for the same number of operator applications."""
    m, K, b = _plate(pkg, 200, 400)
    ref = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=100000))
    ref.setup(K)
    x_ref = np.zeros(m.num_dofs)
    ref.solve(b, x_ref)
    its = {}
    for kind in ("jacobi", "chebyshev"):
        pkg.amg_set_smoother(K, kind)
        s = pkg.CgJacobiSolver(_amg())
        s.setup(K)
        x = np.zeros(m.num_dofs)
        st = s.solve(b, x)
        assert st.converged and st.true_rel_residual <= 1e-10, (kind, st.message)
        assert _rel(x, x_ref) < REL_TOL, kind
        its[kind] = st.iterations
    assert its["chebyshev"] < 0.9 * its["jacobi"], its
    K.ctx.close()


def test_amg_random_plates(pkg, gpu_lib):
    """Seeded plates of the uneven-size batch workload (hole radius, modulus, Poisson ratio, plane
    stress or strain, each of the four load cases) all reach the FP64 Jacobi-PCG solution."""
    specs = pkg.plate.random_batch(count=4, seed=7, n_r_range=(20, 60))
    for k, (spec, case) in enumerate(zip(specs, sorted(pkg.plate.LOAD_CASES))):
        m = pkg.plate.quarter_plate(spec.n_r, spec.n_theta, a=spec.a)
        K = pkg.build_stiffness_pattern(m)
        plane = pkg.PlaneCondition.Strain if spec.plane_strain else pkg.PlaneCondition.Stress
        pkg.assemble_stiffness(m, pkg.constitutive_matrix(spec.E, spec.nu, plane), 1.0, K)
        b = np.zeros(m.num_dofs)
        for group, tx, ty in pkg.plate.LOAD_CASES[case]:
            pkg.add_traction(K, m.boundary_edges[group], 1.0, tx, ty, b)
        pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
        ref = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=100000))
        ref.setup(K)
        x_ref = np.zeros(m.num_dofs)
        assert ref.solve(b, x_ref).converged
        s = pkg.CgJacobiSolver(_amg("mixed" if k % 2 else "fp64"))
        s.setup(K)
        x = np.zeros(m.num_dofs)
        st = s.solve(b, x)
        assert st.converged and st.true_rel_residual <= 1e-10, (spec, case, st.message)
        assert _rel(x, x_ref) < REL_TOL, (spec, case)
        K.ctx.close()


def test_amg_coarse_strength_filter(pkg, gpu_lib):
    """Aggregating the coarse levels over strong connections only (the default) keeps the first
    coarsening, gives smaller aggregates below it and fewer iterations than aggregating over
    every connection; both reach the FP64 Jacobi-PCG solution."""
    m, K, b = _plate(pkg, 200, 400)
    ref = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=100000))
    ref.setup(K)
    x_ref = np.zeros(m.num_dofs)
    ref.solve(b, x_ref)
    out = {}
    for theta_c in (0.0, 0.03):
        pkg.amg_set_strength(K, 0.0, theta_c)
        s = pkg.CgJacobiSolver(_amg())
        s.setup(K)
        info = pkg.amg_setup(K)
        x = np.zeros(m.num_dofs)
        st = s.solve(b, x)
        assert st.converged and st.true_rel_residual <= 1e-10, (theta_c, st.message)
        assert _rel(x, x_ref) < REL_TOL, theta_c
        out[theta_c] = (info["dofs"], st.iterations)
    (d0, it0), (d1, it1) = out[0.0], out[0.03]
    assert d0[:2] == d1[:2] and d1[2] > d0[2], out
    assert it1 < it0, out
    with pytest.raises(pkg.CstgError):
        pkg.amg_set_strength(K, 0.0, 1.5)
    K.ctx.close()
