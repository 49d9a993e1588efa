"""The solve that allocates nothing (cstg_pcg_solve_static), through the C ABI.

It exists for callers that cannot allocate device memory where they solve (fixed memory
budgets with their own pool allocator, callbacks where cudaMalloc would stall the device,
real-time loops); its work vectors live in a static device array of at most 65,536 rows.
Its output is checked against the context-based solve (cstg_pcg_solve on the same CSR) within
the parity tolerance of the other solver tests, on two calls in a row (the second call finds
the first call's contents in the shared array), and against the CPU oracle's Jacobi-PCG (the
reference's recurrence) on the same system. Kept last in collection order.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


def _plate_system(pkg):
    p = pkg.plate.quarter_plate(40, 80)
    K = pkg.build_stiffness_pattern(p)
    pkg.assemble_stiffness(p, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    b = np.zeros(p.num_dofs)
    pkg.add_traction(K, p.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(p), K, b)
    rp, cols, vals = K.download()
    K.ctx.close()
    return rp, cols, vals, b


def test_static_solve_matches_context_solve(pkg, gpu_lib, oracle):
    import torch
    rp, cols, vals, b = _plate_system(pkg)
    n = rp.size - 1
    assert n <= pkg.native.STATIC_MAX_ROWS
    x_or, st_or = oracle.pcg_jacobi(rp, cols, vals, b, rtol=1e-10, max_iter=20000)
    assert st_or["converged"]
    # the existing entry point: the context solve on the same CSR
    A = pkg.GpuCsrMatrix.from_csr(rp, cols, vals)
    s = pkg.CgJacobiSolver()
    s.setup(A)
    x_ref = np.zeros(n)
    st_ref = s.solve(b, x_ref)
    A.ctx.close()
    assert st_ref.converged

    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_cols = torch.from_numpy(cols).to(dev)
    d_vals = torch.from_numpy(vals).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.empty(n, dtype=torch.float64, device=dev)
    opt = pkg.native.default_options()
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    for call in range(2):
        d_x.fill_(float("nan"))
        torch.cuda.synchronize()
        st = pkg.native.Stats()
        rc = gpu_lib.cstg_pcg_solve_static(n, d_rp.data_ptr(), d_cols.data_ptr(), d_vals.data_ptr(),
                                           d_b.data_ptr(), d_x.data_ptr(), C.byref(opt), C.byref(st),
                                           stream)
        assert rc == pkg.native.OK, st.message.decode()
        x = d_x.cpu().numpy()
        assert st.converged and st.iterations == st_ref.iterations, (call, st.message)
        assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < REL_TOL, call
        assert np.linalg.norm(x - x_or) / np.linalg.norm(x_or) < REL_TOL, call
        assert abs(st.iterations - st_or["iterations"]) <= max(2, st_or["iterations"] // 50), call
        assert abs(st.true_rel_residual - st_ref.true_rel_residual) <= 1e-3 * st_ref.true_rel_residual
        assert st.message.decode() == st_ref.message


def test_static_solve_rejects_oversize(pkg, gpu_lib):
    st = pkg.native.Stats()
    rc = gpu_lib.cstg_pcg_solve_static(pkg.native.STATIC_MAX_ROWS + 1, None, None, None, None, None,
                                       None, C.byref(st), None)
    assert rc == pkg.native.ERR_INVALID_ARGUMENT
    assert "outside the static scratch" in st.message.decode()
