"""The learned preconditioner's CPU oracle (oracle/mpnn_oracle.c) checked against finite
differences: the FP64 backward pass must match central differences of the loss, so that the
oracle can check the GPU gradients. CPU only."""
import numpy as np
import pytest


def node_graph(rp, cols):
    """Node-block pattern (self included) from the reference CSR: rows 2n list 2m, 2m+1."""
    N = (rp.size - 1) // 2
    node_ptr = np.zeros(N + 1, dtype=np.int32)
    nbr = []
    for n in range(N):
        c = cols[rp[2 * n]:rp[2 * n + 1]:2] // 2
        nbr.extend(c.tolist())
        node_ptr[n + 1] = len(nbr)
    return node_ptr, np.array(nbr, dtype=np.int32)


def small_problem(pkg, oracle, n_r=3, n_t=4, seed=0):
    m = pkg.plate.quarter_plate(n_r, n_t)
    D = oracle.constitutive_matrix(1.0, 0.3)
    rp, cols = oracle.build_stiffness_pattern(m.num_nodes, m.triangles)
    vals = oracle.assemble_stiffness(m.xy, m.triangles, D, 1.0, rp, cols)
    d, v = pkg.plate.symmetry_dirichlet(m)
    b = np.zeros(m.num_dofs)
    oracle.apply_dirichlet(rp, cols, vals, d, v, b)
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(m.num_dofs)
    Kd = np.zeros((m.num_dofs, m.num_dofs))
    for i in range(m.num_dofs):
        Kd[i, cols[rp[i]:rp[i + 1]]] = vals[rp[i]:rp[i + 1]]
    e = np.linalg.solve(Kd, r)
    invd = 1.0 / np.diag(Kd)
    mat = np.tile([np.log(D[0]), D[1] / D[0]], m.num_nodes)
    return m, rp, cols, vals, r, e, invd, mat


def random_params(oracle, seed=1, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(oracle.mp_param_count()) * scale


def test_mpnn_oracle_gradient_matches_finite_differences(pkg, oracle):
    m, rp, cols, vals, r, e, invd, mat = small_problem(pkg, oracle)
    node_ptr, nbr = node_graph(rp, cols)
    X, s = oracle.mp_features(r, invd, m.xy, mat)
    P = random_params(oracle)

    def loss(P):
        Y, _ = oracle.mp_forward(node_ptr, nbr, X, P, q=False)
        return oracle.mp_loss(rp, cols, vals, r, e, invd, s, Y, grad=False)[0]

    Y, cache = oracle.mp_forward(node_ptr, nbr, X, P, q=False)
    L0, dY = oracle.mp_loss(rp, cols, vals, r, e, invd, s, Y)
    assert 0.0 <= L0 <= 1.0
    g = oracle.mp_backward(node_ptr, nbr, X, P, cache, dY, q=False)
    rng = np.random.default_rng(3)
    idx = np.concatenate([rng.choice(P.size, 60, replace=False), [P.size - 1, P.size - 2, 0, 520]])
    h = 1e-6
    fd = []
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd.append((loss(Pp) - loss(Pm)) / (2 * h))
    fd = np.array(fd)
    assert np.linalg.norm(g[idx] - fd) <= 1e-5 * np.linalg.norm(fd) + 1e-12


def test_mpnn_oracle_zero_network_is_jacobi(pkg, oracle):
    """With all parameters zero the network outputs Y = 0: z = D^-1 r, the Jacobi step."""
    m, rp, cols, vals, r, e, invd, mat = small_problem(pkg, oracle)
    node_ptr, nbr = node_graph(rp, cols)
    X, s = oracle.mp_features(r, invd, m.xy, mat)
    Y, _ = oracle.mp_forward(node_ptr, nbr, X, np.zeros(oracle.mp_param_count()))
    assert np.all(Y == 0.0)
    assert np.array_equal(oracle.mp_apply(r, invd, s, Y), invd * r)


def test_mpnn_oracle_homogeneous_in_r(pkg, oracle):
    """z(c r) = c z(r): the input is r / RMS(r) and the output is scaled back by RMS(r)."""
    m, rp, cols, vals, r, e, invd, mat = small_problem(pkg, oracle)
    node_ptr, nbr = node_graph(rp, cols)
    P = random_params(oracle, seed=5)
    zs = []
    for c in (1.0, 8.0):
        X, s = oracle.mp_features(c * r, invd, m.xy, mat)
        Y, _ = oracle.mp_forward(node_ptr, nbr, X, P, q=False)
        zs.append(oracle.mp_apply(c * r, invd, s, Y))
    assert np.allclose(zs[1], 8.0 * zs[0], rtol=1e-12, atol=0)


def test_mpnn_oracle_cycle_gradient_matches_finite_differences(pkg, oracle):
    """The learned multigrid cycle's loss: the network reads the residual r2 left after the
    cycle's fixed part x_fix and adds omega D^-1 (r2 + s Y); the gradient of the loss of the
    cycle's output (against the sample's r and e) must match central differences."""
    m, rp, cols, vals, r, e, invd, mat = small_problem(pkg, oracle, seed=4)
    node_ptr, nbr = node_graph(rp, cols)
    rng = np.random.default_rng(8)
    xfix = 0.5 * e + 0.1 * rng.standard_normal(e.size) * np.abs(e).max()
    r2 = r - oracle.multiply(rp, cols, vals, xfix)
    winvd = 0.6 * invd
    X, s = oracle.mp_features(r2, invd, m.xy, mat)
    P = random_params(oracle, seed=2)

    def loss(P):
        Y, _ = oracle.mp_forward(node_ptr, nbr, X, P, q=False)
        return oracle.mp_loss_cycle(rp, cols, vals, r, e, xfix, r2, winvd, s, Y, grad=False)[0]

    Y, cache = oracle.mp_forward(node_ptr, nbr, X, P, q=False)
    L0, dY = oracle.mp_loss_cycle(rp, cols, vals, r, e, xfix, r2, winvd, s, Y)
    assert 0.0 <= L0 <= 1.0
    g = oracle.mp_backward(node_ptr, nbr, X, P, cache, dY, q=False)
    idx = np.concatenate([rng.choice(P.size, 60, replace=False), [P.size - 1, P.size - 2, 0, 520]])
    h = 1e-6
    fd = []
    for k in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd.append((loss(Pp) - loss(Pm)) / (2 * h))
    fd = np.array(fd)
    assert np.linalg.norm(g[idx] - fd) <= 1e-5 * np.linalg.norm(fd) + 1e-12
    # with the network at zero the cycle's post-smoothing is one damped-Jacobi step
    Y0, _ = oracle.mp_forward(node_ptr, nbr, X, np.zeros(P.size), q=False)
    z0 = xfix + winvd * (r2 + s * Y0)
    assert np.array_equal(z0, xfix + winvd * r2)
