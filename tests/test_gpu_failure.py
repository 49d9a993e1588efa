"""Failure detection without a GPU fault: every device wait of the library is bounded, and a
wait that gives up comes back to the host as CSTG_ERR_TIMEOUT with the context still usable.

The waits are made to run out by setting their poll limits to zero (cstg_set_wait_limits): the
persistent solve's grid barrier (every block but the last to arrive gives up at once) and the
learned network's tensor-core wait (it gives up, then lets the matrix multiply finish before the
kernel releases its memory). Afterwards the limits go back to their defaults and the same
context must solve correctly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(pkg, n_r=40, n_t=80):
    m = pkg.plate.quarter_plate(n_r, n_t)
    D = pkg.constitutive_matrix(1.0, 0.3)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    return m, D, K, b


def test_persistent_barrier_timeout_then_recovery(pkg, gpu_lib, golden):
    g = golden("plate_40x80")
    m, D, K, b = _system(pkg)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, launch="persistent"))
    s.setup(K)
    K.ctx.set_wait_limits(barrier_polls=0)
    x = np.zeros(m.num_dofs)
    with pytest.raises(pkg.CstgError) as ei:
        s.solve(b, x)
    assert ei.value.code == pkg.native.ERR_TIMEOUT
    assert "grid barrier" in str(ei.value)
    # the same context, default limits: the reference's solution
    K.ctx.set_wait_limits()
    st = s.solve(b, x)
    assert st.converged, st.message
    assert np.linalg.norm(x - g["u"]) <= 1e-8 * np.linalg.norm(g["u"])
    K.ctx.close()


def test_timeout_status_in_stats(pkg, gpu_lib):
    """Through the C ABI: the status code and stats.status of a solve whose barrier gave up."""
    import ctypes as C
    m, D, K, b = _system(pkg, 20, 40)
    ctx = K.ctx
    ctx.check(ctx.L.cstg_pcg_setup(ctx.h))
    ctx.set_wait_limits(0, -1)
    o = pkg.SolverOptions(rtol=1e-10, launch="persistent").native()
    st = pkg.native.Stats()
    x = np.zeros(m.num_dofs)
    rc = ctx.L.cstg_pcg_solve(ctx.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(st), None)
    assert rc == pkg.native.ERR_TIMEOUT
    assert st.status == pkg.native.SOLVE_TIMEOUT
    ctx.set_wait_limits()
    rc = ctx.L.cstg_pcg_solve(ctx.h, b.ctypes.data, x.ctypes.data, C.byref(o), C.byref(st), None)
    assert rc == pkg.native.OK and st.converged
    ctx.close()


def test_tensor_core_wait_timeout_then_recovery(pkg, gpu_lib):
    import torch
    m, D, K, b = _system(pkg, 20, 40)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10))
    s.setup(K)
    w = pkg.learned.load_weights()
    pkg.learned.setup(K, w, pkg.learned.node_material(D, m.num_nodes))
    r = torch.from_numpy(np.random.default_rng(0).standard_normal(m.num_dofs)).cuda()
    z_ok = pkg.learned.apply(K, r).cpu().numpy()
    K.ctx.set_wait_limits(mma_polls=0)
    with pytest.raises(pkg.CstgError) as ei:
        pkg.learned.apply(K, r)
    assert ei.value.code == pkg.native.ERR_TIMEOUT
    K.ctx.set_wait_limits()
    z = pkg.learned.apply(K, r).cpu().numpy()
    assert np.array_equal(z, z_ok)
    # and a learned solve on the same context
    s2 = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=100000, preconditioner="learned",
                                              true_residual_stop=True))
    s2.A = K
    x = np.zeros(m.num_dofs)
    st = s2.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    K.ctx.close()


def test_wait_limits_reject_bad_values(pkg, gpu_lib, ctx):
    with pytest.raises(pkg.CstgError):
        ctx.set_wait_limits(-5, 0)
