"""Parity with the reference at the benchmark sizes: the reference serial core was run to
convergence on the 1M-DOF plate (O-grid 400 x 1250, 1,003,302 DOFs) and on the 2M-DOF plate
(565 x 1766, 2,000,244 DOFs) by tests/golden/make_golden_large.py, which stored SHA-256 digests
of its pattern, K, the loads and K / b after the Dirichlet elimination, its iteration count and
residuals, its stress concentration factor and its displacements (all of them at 1M DOFs, every
8th node at 2M DOFs).

Bars: the integer pattern and the FP64 assembly, loads and elimination bit-identical; FP64
Jacobi-PCG under the reference's stopping rule within 2 % of its iterations; every solution
(plain FP64, mixed precision, the multigrid cycle, the learned cycle and the network alone)
within relative 1e-8 (2-norm) of the reference's displacements; the element stresses of the
reference's displacements bit-identical; the SCF within 1e-8 of the reference's.
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REL_TOL = 1e-8


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _golden(tag):
    meta = json.load(open(os.path.join(HERE, "golden", f"plate_{tag}.json")))
    npz = np.load(os.path.join(HERE, "golden", f"plate_{tag}.npz"))
    if "u_sub" in npz.files:
        nodes = np.arange(0, meta["n_dofs"] // 2, meta["u_stride_nodes"])
        idx = np.stack([2 * nodes, 2 * nodes + 1], axis=1).reshape(-1)
        return meta, npz["u_sub"], idx
    return meta, npz["u"], None


def _rel(x, u, idx):
    xs = x if idx is None else x[idx]
    return np.linalg.norm(xs - u) / np.linalg.norm(u)


def _system(pkg, meta):
    import torch
    m = pkg.plate.quarter_plate(meta["n_r"], meta["n_theta"])
    assert sha(m.xy) == meta["xy_sha"] and sha(m.triangles) == meta["tri_sha"]
    D = pkg.constitutive_matrix(1.0, 0.3)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    f = torch.zeros(m.num_dofs, dtype=torch.float64, device="cuda")
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, f)  # on the GPU
    return m, D, K, f


@pytest.mark.parametrize("tag", ["400x1250", "565x1766"])
def test_assembly_loads_and_elimination_bit_exact(pkg, gpu_lib, tag):
    meta, _, _ = _golden(tag)
    m, D, K, f = _system(pkg, meta)
    rp, cols, kv = K.download()
    assert int(cols.size) == meta["nnz"]
    assert sha(rp) == meta["row_ptr_sha"] and sha(cols) == meta["cols_sha"]
    assert sha(kv) == meta["K_sha"]
    fh = f.cpu().numpy()
    assert sha(fh) == meta["f_sha"]
    dofs, vals = pkg.plate.symmetry_dirichlet(m)
    assert sha(dofs) == meta["dir_dofs_sha"]
    pkg.apply_dirichlet((dofs, vals), K, f)
    _, _, kbc = K.download()
    assert sha(kbc) == meta["Kbc_sha"] and sha(f.cpu().numpy()) == meta["b_sha"]
    K.ctx.close()


def _solve(pkg, K, b, **kw):
    import torch
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=400000, **kw))
    s.setup(K)
    x = torch.zeros_like(b)
    st = s.solve(b, x)
    return x.cpu().numpy(), st


@pytest.mark.parametrize("tag", ["400x1250", "565x1766"])
def test_solutions_match_reference_displacements(pkg, gpu_lib, tag):
    meta, u, idx = _golden(tag)
    m, D, K, f = _system(pkg, meta)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, f)
    # the reference's method and stopping rule
    x, st = _solve(pkg, K, f)
    assert st.converged
    assert abs(st.iterations - meta["iters"]) <= 0.02 * meta["iters"], (st.iterations, meta["iters"])
    assert _rel(x, u, idx) < REL_TOL
    errors = {"reference_rule": _rel(x, u, idx)}
    # every method of this library, on the FP64 true residual
    mat = pkg.learned.node_material(D, m.num_nodes)
    cases = [("plain_fp64", {}, None), ("jacobi_mixed", {"precision": "mixed"}, None),
             ("amg_mixed", {"precision": "mixed", "preconditioner": "amg"}, None),
             ("learned_cycle_mixed", {"precision": "mixed", "preconditioner": "learned_mg"}, "cycle"),
             ("learned_local_mixed", {"precision": "mixed", "preconditioner": "learned"}, "local")]
    for name, kw, weights in cases:
        s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=400000, true_residual_stop=True, **kw))
        s.setup(K)
        if weights:
            pkg.learned.setup(K, pkg.learned.load_weights(mode=weights), mat)
        import torch
        xx = torch.zeros_like(f)
        st = s.solve(f, xx)
        assert st.converged and st.true_rel_residual <= 1e-10, (name, st.message)
        errors[name] = _rel(xx.cpu().numpy(), u, idx)
        assert errors[name] < REL_TOL, (name, errors[name])
    print(f"relative error against the reference's displacements ({tag}):", errors)
    K.ctx.close()


def test_stresses_and_scf_of_reference_displacements(pkg, gpu_lib):
    """At 1M DOFs the reference's full displacement field is stored: the GPU element stresses of
    those displacements are bit-identical to the reference's, and so is the SCF."""
    meta, u, idx = _golden("400x1250")
    assert idx is None
    m, D, K, f = _system(pkg, meta)
    st = pkg.compute_element_stresses(K, u, 1.0, 0.3)
    assert sha(st["sxx"]) == meta["sxx_sha"]
    scf, e = pkg.scf_at_hole(st, 1.0)
    assert e == meta["scf_element"] and scf == meta["scf"]
    K.ctx.close()
