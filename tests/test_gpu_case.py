"""The case-file front end end-to-end on the GPU: a reference-style case on the reference's
Kirsch mesh (written from the golden fixture) reproduces the reference's displacements
(relative 1e-8) and iteration count; the analytical Kirsch traction case recovers SCF ~ 3."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASE = """# Kirsch L0 with a constant traction (the golden fixture's loads)
mesh             = {mesh}
plane            = plane_stress
E                = 210e9
nu               = 0.3
thickness        = 0.01
solver           = {solver}
rtol             = 1e-10
max_iter         = 20000
output_dir       = {out}
bc.dirichlet     = left_sym:ux=0 ; bottom_sym:uy=0
bc.traction      = {traction}
kirsch.sigma_inf = 1
kirsch.a         = {a}
"""


def _run(pkg, tmp_path, mesh, solver="cg_jacobi", traction="right:tx=100e6,ty=0", a=1.0):
    from importlib import import_module
    import io
    case = import_module("mpi-cst-fem-solver_b200.case")
    mp = str(tmp_path / "mesh.msh")
    pkg.write_gmsh(mesh, mp)
    out_dir = str(tmp_path / "out")
    cp = str(tmp_path / "k.case")
    open(cp, "w").write(CASE.format(mesh=mp, out=out_dir, solver=solver, traction=traction, a=repr(a)))
    out, err = io.StringIO(), io.StringIO()
    rc = case.run_case(cp, out, err)
    return rc, out.getvalue(), err.getvalue(), out_dir


def test_case_kirsch_L0_matches_reference(pkg, gpu_lib, golden, tmp_path):
    g = golden("kirsch_L0")
    rc, out, err, d = _run(pkg, tmp_path, g.mesh(pkg))
    assert rc == 0, out + err
    u = np.load(os.path.join(d, "displacement.npy"))
    assert np.linalg.norm(u - g["stress_u10"]) <= 1e-8 * np.linalg.norm(g["stress_u10"])
    t = json.load(open(os.path.join(d, "timings.json")))
    assert t["path"] == "gpu" and t["solver"]["converged"] and t["dofs"] == u.size
    assert t["solver"]["iterations"] == g.meta["stress_iters10"]
    # instrument = true (the default): the reference's solve_breakdown entries from CUDA events
    bd = t["solve_breakdown"]
    names = ["setup", "spmv_local", "halo_post", "halo_wait", "spmv_ghost", "dot_local", "allreduce",
             "vector_ops", "unaccounted", "total", "time_per_iteration", "accounted_fraction",
             "halo_bytes_sent_per_iteration", "halo_messages_sent_per_iteration"]
    assert list(bd) == names
    assert all(set(v) == {"min", "max", "mean"} for v in bd.values())
    assert bd["total"]["mean"] > 0 and bd["spmv_local"]["mean"] > 0 and bd["vector_ops"]["mean"] > 0
    # (the rest of the total is the device idling between batches while the host reads the state;
    # on this 1.5k-DOF mesh that is ~15 % of a 150-iteration solve)
    assert 0.5 <= bd["accounted_fraction"]["mean"] <= 1.0 + 1e-9


def test_instrumented_solve_matches_graph_path(pkg, gpu_lib):
    """The instrumented launch runs the graph path's kernels one by one: the same iterations
    and the same bits; its phase times add up to the device time of the solve."""
    m = pkg.plate.quarter_plate(30, 60)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    xs = {}
    for launch in ("graph", "instrumented"):
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, launch=launch))
        s.setup(K)
        x = np.zeros(m.num_dofs)
        st = s.solve(b, x)
        assert st.converged
        xs[launch] = (x, st.iterations)
    assert xs["graph"][1] == xs["instrumented"][1]
    assert np.array_equal(xs["graph"][0], xs["instrumented"][0])
    bd = s.breakdown()
    assert bd["spmv_calls"] == xs["instrumented"][1] + 1
    acc = bd["setup"] + bd["spmv_local"] + bd["dot_local"] + bd["vector_ops"]
    assert 0.5 * bd["total"] <= acc <= bd["total"] * (1 + 1e-9)
    K.ctx.close()


@pytest.mark.parametrize("solver", ["gpu_cg", "gpu_cg_mixed", "gpu_cg_amg"])
def test_case_kirsch_exact_scf(pkg, gpu_lib, tmp_path, solver):
    mesh = pkg.plate.quarter_plate(40, 80)
    rc, out, err, d = _run(pkg, tmp_path, mesh, solver=solver, traction="kirsch_exact")
    assert rc == 0, out + err
    t = json.load(open(os.path.join(d, "timings.json")))
    k = t["kirsch"]
    assert 2.8 < k["scf"]["numerical"] < 3.2 and k["l2_rel_stress_error"] < 0.1
    assert t["solver"]["true_rel_residual"] <= 1e-10


def test_case_kirsch_refinement_lowers_the_error(pkg, gpu_lib, golden, tmp_path):
    """The reference's end-to-end check (its tests/check_e2e.cmake) on the GPU path: its committed
    Kirsch meshes L0 and L1 (L = 1, hole radius 0.1) under the exact Kirsch traction, solved
    through the case-file front end: converged, true residual below 1e-9, and the relative L2
    error of the element stresses against the analytical field lower on L1 than on L0."""
    errs = []
    for name in ("kirsch_L0", "kirsch_L1"):
        (tmp_path / name).mkdir()
        rc, out, err, d = _run(pkg, tmp_path / name, golden(name).mesh(pkg), solver="gpu_cg",
                               traction="kirsch_exact", a=0.1)
        assert rc == 0, out + err
        t = json.load(open(os.path.join(d, "timings.json")))
        assert t["solver"]["converged"] and t["solver"]["true_rel_residual"] < 1e-9, t["solver"]
        errs.append(t["kirsch"]["l2_rel_stress_error"])
    assert 0.0 < errs[1] < errs[0], errs
