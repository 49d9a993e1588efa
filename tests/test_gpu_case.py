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
kirsch.a         = 1
"""


def _run(pkg, tmp_path, mesh, solver="cg_jacobi", traction="right:tx=100e6,ty=0"):
    from importlib import import_module
    import io
    case = import_module("mpi-cst-fem-solver_b200.case")
    mp = str(tmp_path / "mesh.msh")
    pkg.write_gmsh(mesh, mp)
    out_dir = str(tmp_path / "out")
    cp = str(tmp_path / "k.case")
    open(cp, "w").write(CASE.format(mesh=mp, out=out_dir, solver=solver, traction=traction))
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


@pytest.mark.parametrize("solver", ["gpu_cg", "gpu_cg_mixed", "gpu_cg_amg"])
def test_case_kirsch_exact_scf(pkg, gpu_lib, tmp_path, solver):
    mesh = pkg.plate.quarter_plate(40, 80)
    rc, out, err, d = _run(pkg, tmp_path, mesh, solver=solver, traction="kirsch_exact")
    assert rc == 0, out + err
    t = json.load(open(os.path.join(d, "timings.json")))
    k = t["kirsch"]
    assert 2.8 < k["scf"]["numerical"] < 3.2 and k["l2_rel_stress_error"] < 0.1
    assert t["solver"]["true_rel_residual"] <= 1e-10
