"""Learned preconditioner on the GPU: the tensor-core forward pass and the training gradients
against the FP64 oracle (oracle/mpnn_oracle.c), training, and the flexible-CG solve with its
Jacobi fallback, checked against the reference's FP64 Jacobi-PCG solution.

Bars: forward z within relative 1e-2 of the oracle (BF16 activations on both sides; the rest
is FP32-vs-FP64 accumulation); gradients within relative 5e-2; solves converged on the FP64 true
residual <= 1e-10 with displacements within relative 1e-8 of the oracle's FP64 Jacobi-PCG."""
import numpy as np
import pytest

from test_oracle_mpnn import node_graph

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _plate(pkg, n_r=6, n_t=12, E=1.0, nu=0.3):
    m = pkg.plate.quarter_plate(n_r, n_t)
    D = pkg.constitutive_matrix(E, nu)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    return m, D, K, b


def _bf16_params(oracle, pkg, seed=4, out_scale=0.3):
    p = pkg.learned.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    p[-130:] = rng.standard_normal(130) * out_scale  # a non-zero output layer
    p = p.astype(np.float32)
    # the oracle sees what the GPU computes with: BF16 weights, FP32 biases
    q = p.astype(np.float64)
    o = 0
    w_idx = []
    w_idx.append(np.arange(0, 64 * 8))
    o = 64 * 8 + 64
    for _ in range(3):
        w_idx.append(np.arange(o, o + 64 * 128))
        o += 64 * 128 + 64
    w_idx.append(np.arange(o, o + 128))
    for idx in w_idx:
        q[idx] = oracle.mp_round_bf16(q[idx])
    return p, q


def test_learned_forward_matches_oracle(pkg, oracle, gpu_lib):
    import torch
    m, D, K, b = _plate(pkg)
    p, q = _bf16_params(oracle, pkg)
    mat = pkg.learned.node_material(D, m.num_nodes)
    pkg.learned.setup(K, p, mat)
    rng = np.random.default_rng(0)
    r = rng.standard_normal(m.num_dofs)
    z = pkg.learned.apply(K, torch.from_numpy(r).cuda()).cpu().numpy()
    rp, cols, vals = K.download()
    invd = 1.0 / vals[[np.searchsorted(cols[rp[i]:rp[i + 1]], i) + rp[i] for i in range(rp.size - 1)]]
    node_ptr, nbr = node_graph(rp, cols)
    X, s = oracle.mp_features(r, invd, m.xy, mat.astype(np.float64))
    Y, _ = oracle.mp_forward(node_ptr, nbr, X, q, q=True)
    z_ref = oracle.mp_apply(r, invd, s, Y)
    assert np.abs(Y).max() > 1e-3  # the network is not trivially zero
    assert _rel(z, z_ref) < 1e-2
    # the network's own part (z - D^-1 r) is what the tensor cores compute
    assert _rel(z - invd * r, z_ref - invd * r) < 2e-2
    K.ctx.close()


def test_learned_gradients_match_oracle(pkg, oracle, gpu_lib):
    import torch
    m, D, K, b = _plate(pkg)
    p, q = _bf16_params(oracle, pkg, seed=9)
    mat = pkg.learned.node_material(D, m.num_nodes)
    pkg.learned.setup(K, p, mat)
    rp, cols, vals = K.download()
    Kd = np.zeros((m.num_dofs, m.num_dofs))
    for i in range(m.num_dofs):
        Kd[i, cols[rp[i]:rp[i + 1]]] = vals[rp[i]:rp[i + 1]]
    rng = np.random.default_rng(1)
    r = rng.standard_normal(m.num_dofs)
    e = np.linalg.solve(Kd, r)
    invd = 1.0 / np.diag(Kd)
    tr = pkg.learned.Trainer(p)
    loss = tr.accumulate(K, torch.from_numpy(r[None, :]).cuda(), torch.from_numpy(e[None, :]).cuda())
    _, g = tr.params(grads=True)
    node_ptr, nbr = node_graph(rp, cols)
    X, s = oracle.mp_features(r, invd, m.xy, mat.astype(np.float64))
    Y, cache = oracle.mp_forward(node_ptr, nbr, X, q, q=True)
    L, dY = oracle.mp_loss(rp, cols, vals, r, e, invd, s, Y)
    g_ref = oracle.mp_backward(node_ptr, nbr, X, q, cache, dY, q=True)
    assert abs(loss[0] - L) < 1e-3 * max(1.0, abs(L))
    assert _rel(g, g_ref) < 5e-2
    # each block of the parameter vector separately (encoder, 3 layers, decoder)
    bounds = [0, 576, 576 + 8256, 576 + 2 * 8256, 576 + 3 * 8256, 25474]
    for a, c in zip(bounds[:-1], bounds[1:]):
        assert _rel(g[a:c], g_ref[a:c]) < 5e-2, (a, c)
    tr.close()
    K.ctx.close()


def test_zero_network_flexible_cg_is_jacobi_pcg(pkg, oracle, gpu_lib, golden):
    """With all weights zero, z = D^-1 r: flexible CG reproduces Jacobi-PCG (same iterations
    within 1 %, same solution to 1e-8)."""
    g = golden("plate_40x80")
    m = pkg.plate.quarter_plate(40, 80)
    D = pkg.constitutive_matrix(1.0, 0.3)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=100000, preconditioner="learned",
                                             true_residual_stop=True))
    s.setup(K)
    pkg.learned.setup(K, np.zeros(pkg.learned.N_PARAMS, np.float32), pkg.learned.node_material(D, m.num_nodes))
    x = np.zeros(m.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert abs(st.iterations - g.meta["iters"]) <= 0.01 * g.meta["iters"] + 2
    assert _rel(x, g["u"]) < REL_TOL
    K.ctx.close()


def test_fallback_on_a_bad_network(pkg, gpu_lib, golden):
    """A network with large random weights: the solve still converges (Jacobi takes over) to the
    reference's solution."""
    g = golden("plate_40x80")
    m = pkg.plate.quarter_plate(40, 80)
    D = pkg.constitutive_matrix(1.0, 0.3)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=200000, preconditioner="learned",
                                             true_residual_stop=True))
    s.setup(K)
    p = (np.random.default_rng(3).standard_normal(pkg.learned.N_PARAMS) * 3.0).astype(np.float32)
    pkg.learned.setup(K, p, pkg.learned.node_material(D, m.num_nodes))
    x = np.zeros(m.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert _rel(x, g["u"]) < REL_TOL
    K.ctx.close()


def test_training_lowers_the_loss(pkg, gpu_lib):
    """A few Adam steps on one plate's pairs lower the mean loss from its Jacobi value."""
    import torch
    spec = pkg.plate.PlateSpec(n_r=16, n_theta=32, a=1.0, E=1.0, nu=0.3, plane_strain=False)
    p0 = pkg.learned.init_params(0)
    prob = pkg.learned.harvest(spec, 24, p0, seed=0)
    tr = pkg.learned.Trainer(p0)
    first = tr.accumulate(prob.K, prob.R, prob.E).mean()
    tr.zero_grad()
    for _ in range(60):
        losses = tr.accumulate(prob.K, prob.R, prob.E)
        tr.step(3e-3, 1.0 / len(losses))
    last = tr.accumulate(prob.K, prob.R, prob.E).mean()
    assert np.isfinite(first) and last < 0.9 * first, (first, last)
    tr.close()
    prob.K.ctx.close()


def test_trained_network_gain_on_held_out_plates(pkg, gpu_lib):
    """What the packaged (trained) network gains over the method without it, measured on plates
    it was not trained on: its loss (the energy-norm angle between M(r) and the error) is lower
    than the Jacobi step's (the network with its output layer at zero), and the flexible-CG
    solve with it still converges to the FP64 solution (Jacobi takes over on stagnation)."""
    w = pkg.learned.load_weights()
    jac = w.copy()
    jac[-130:] = 0.0  # output layer off: z = D^-1 r
    specs = pkg.plate.random_batch(count=3, seed=99, n_r_range=(20, 60))
    gains = []
    for i, spec in enumerate(specs):
        prob = pkg.learned.harvest(spec, 40, w, seed=100 + i)
        losses = {}
        for name, p in (("trained", w), ("jacobi", jac)):
            tr = pkg.learned.Trainer(p)
            losses[name] = tr.accumulate(prob.K, prob.R, prob.E).mean()
            tr.close()
        gains.append(losses["jacobi"] - losses["trained"])
        prob.K.ctx.close()
    assert np.mean(gains) > 0.0, gains

    m = pkg.plate.quarter_plate(30, 60)
    D = pkg.constitutive_matrix(1.0, 0.3)
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    b = np.zeros(m.num_dofs)
    pkg.add_traction(K, m.boundary_edges["right"], 1.0, 1.0, 0.0, b)
    pkg.apply_dirichlet(pkg.plate.symmetry_dirichlet(m), K, b)
    ref = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=100000))
    ref.setup(K)
    x_ref = np.zeros(m.num_dofs)
    assert ref.solve(b, x_ref).converged
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-10, max_iter=200000, precision="mixed",
                                             preconditioner="learned", true_residual_stop=True))
    s.setup(K)
    pkg.learned.setup(K, w, pkg.learned.node_material(D, m.num_nodes))
    x = np.zeros(m.num_dofs)
    st = s.solve(b, x)
    assert st.converged and st.true_rel_residual <= 1e-10, st.message
    assert _rel(x, x_ref) < REL_TOL
    K.ctx.close()


def _mesh_system(pkg, m, D):
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, D, 1.0, K)
    s = pkg.CgJacobiSolver()
    s.setup(K)
    return K


def _plan_fallback_tiles(m):
    """Tiles of 128 nodes the layers' gather plan cannot take (more than 8 runs of consecutive
    rows, more than 400 rows, a span over 4096 nodes or a node of more than 7 neighbours), counted
    on the host from the mesh alone."""
    tri = np.asarray(m.triangles).reshape(-1, 3).astype(np.int64)
    N = m.num_nodes
    a = np.unique(np.concatenate([tri[:, i] * N + tri[:, j] for i in range(3) for j in range(3)]))
    src, dst = a // N, a % N
    ptr = np.searchsorted(src, np.arange(N + 1))
    out = 0
    for t in range(0, N, 128):
        u = np.unique(dst[ptr[t]:ptr[min(N, t + 128)]])
        deg = np.diff(ptr[t:min(N, t + 128) + 1])
        runs = 1 + int(np.sum(np.diff(u) > 1))
        out += int(u[-1] - u[0] + 1 > 4096 or u.size > 400 or runs > 8 or deg.max() - 1 > 7)
    return out, (N + 127) // 128


def _renumbered_plate(pkg, n_r, n_t, first, seed):
    """The quarter plate with the nodes from `first` on numbered at random."""
    m = pkg.plate.quarter_plate(n_r, n_t)
    N = m.num_nodes
    perm = np.arange(N)
    perm[first:] = first + np.random.default_rng(seed).permutation(N - first)
    xy = np.empty_like(np.asarray(m.xy).reshape(-1, 2))
    xy[perm] = np.asarray(m.xy).reshape(-1, 2)
    tri = perm[np.asarray(m.triangles).reshape(-1, 3)].astype(np.int32)
    return pkg.plate.Mesh(xy=xy.reshape(-1), triangles=tri.reshape(-1), boundary_edges={})


def test_gather_plan_matches_row_gather(pkg, oracle, gpu_lib, golden, monkeypatch):
    """The layers read each tile's rows either through its gather plan (bulk copies of runs of
    consecutive rows into shared memory) or row by row; both sum the same neighbours in the same
    order, so z and the training loss and gradients are bit-identical. Meshes: an O-grid plate
    (every tile planned: the plan kernel), the Kirsch L1 mesh (no tile planned: the row kernel
    either way) and a plate renumbered at random past its 1000th node (27 % of the tiles planned:
    the plan kernel with row-by-row fallback tiles in the same launch)."""
    import torch
    D = pkg.constitutive_matrix(1.0, 0.3)
    meshes = {"plate": pkg.plate.quarter_plate(60, 150), "kirsch_L1": golden("kirsch_L1").mesh(pkg),
              "mixed": _renumbered_plate(pkg, 40, 80, 1000, 5),
              "tiny": pkg.plate.quarter_plate(2, 4),           # 15 nodes: one ragged tile
              "ragged": pkg.plate.quarter_plate(8, 14)}        # 135 nodes: a full tile and 7 nodes
    kinds = {k: _plan_fallback_tiles(m) for k, m in meshes.items()}
    assert kinds["plate"][0] == 0 and kinds["kirsch_L1"][0] == kinds["kirsch_L1"][1]
    assert kinds["tiny"] == (0, 1) and kinds["ragged"] == (0, 2), kinds
    assert 0 < kinds["mixed"][0] < kinds["mixed"][1], kinds
    p, _ = _bf16_params(oracle, pkg, seed=6)
    for name, m in meshes.items():
        rng = np.random.default_rng(11)
        r = rng.standard_normal((2, m.num_dofs))
        e = rng.standard_normal((2, m.num_dofs))
        mat = pkg.learned.node_material(D, m.num_nodes)
        out = {}
        for gather in ("plan", "rows"):
            if gather == "rows":
                monkeypatch.setenv("CSTG_MP_GATHER", "rows")
            else:
                monkeypatch.delenv("CSTG_MP_GATHER", raising=False)
            K = _mesh_system(pkg, m, D)
            pkg.learned.setup(K, p, mat)
            z = pkg.learned.apply(K, torch.from_numpy(r[0]).cuda()).cpu().numpy()
            tr = pkg.learned.Trainer(p)
            loss = tr.accumulate(K, torch.from_numpy(r).cuda(), torch.from_numpy(e).cuda())
            _, g = tr.params(grads=True)
            out[gather] = (z, loss, g)
            tr.close()
            K.ctx.close()
        monkeypatch.delenv("CSTG_MP_GATHER", raising=False)
        for a, b in zip(out["plan"], out["rows"]):
            assert np.array_equal(a, b), name
