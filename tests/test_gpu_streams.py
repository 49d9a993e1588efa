"""Stream ordering between torch and a context.

A context runs its kernels on its own stream. The Python device wrappers order each call after
torch's pending work (inputs written by torch kernels) and torch's later work after the call
(outputs, including the calls that only enqueue). These tests write the input with a torch
kernel right before the call, on a busy stream, and read the output on torch's stream with no
explicit synchronisation; the values must be the oracle's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plate(pkg, n_r=60, n_t=120):
    m = pkg.plate.quarter_plate(n_r, n_t)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, pkg.constitutive_matrix(1.0, 0.3), 1.0, K)
    return m, K


def _busy(torch, dev):
    # a long chain of torch kernels ahead of the input's last write
    a = torch.randn(4096, 4096, device=dev)
    for _ in range(8):
        a = a @ a
        a = a / a.norm()
    return a


def test_spmv_orders_with_torch_stream(pkg, oracle, gpu_lib):
    import torch
    dev = torch.device("cuda:0")
    m, K = _plate(pkg)
    rp, cols, vals = K.download()
    rng = np.random.default_rng(5)
    x_h = rng.standard_normal(m.num_dofs)
    # the same kernel through the host path (synchronous): the device path must give its bits
    y_ref = K.multiply(x_h)
    assert np.linalg.norm(y_ref - oracle.multiply(rp, cols, vals, x_h)) <= 1e-13 * np.linalg.norm(y_ref)
    for _ in range(3):
        _busy(torch, dev)
        x = torch.zeros(m.num_dofs, dtype=torch.float64, device=dev)
        x.add_(torch.from_numpy(x_h).to(dev, non_blocking=False))  # last write on torch's stream
        y = K.multiply(x)
        y2 = y * 1.0  # a torch kernel reading y, no synchronize in between
        assert np.array_equal(y2.cpu().numpy(), y_ref)
    K.ctx.close()


def test_mixed_spmv_orders_with_torch_stream(pkg, gpu_lib):
    import torch
    dev = torch.device("cuda:0")
    m, K = _plate(pkg)
    b = np.zeros(m.num_dofs)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    rng = np.random.default_rng(6)
    x_h = rng.standard_normal(m.num_dofs)
    x0 = torch.from_numpy(x_h).to(dev)
    y_ref = K.multiply(x0).cpu().numpy()
    for _ in range(3):
        _busy(torch, dev)
        x = torch.zeros_like(x0)
        x.add_(x0)
        y = K.multiply_mixed(x)
        y2 = y * 1.0
        assert np.linalg.norm(y2.cpu().numpy() - y_ref) <= 1e-6 * np.linalg.norm(y_ref)
    K.ctx.close()


def test_device_solve_reads_torch_written_rhs(pkg, oracle, gpu_lib):
    import torch
    dev = torch.device("cuda:0")
    m, K = _plate(pkg, 20, 40)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    rp, cols, vals = K.download()
    x_ref, _ = oracle.pcg_jacobi(rp, cols, vals, b, rtol=1e-10, max_iter=20000)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    _busy(torch, dev)
    d_b = torch.zeros(m.num_dofs, dtype=torch.float64, device=dev)
    d_b.add_(torch.from_numpy(b).to(dev))
    x = torch.empty_like(d_b)
    st = s.solve(d_b, x)
    x2 = x * 1.0
    assert st.converged
    xr = x2.cpu().numpy()
    assert np.linalg.norm(xr - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    K.ctx.close()
