"""The reference's patch tests (tests/test_patch.cpp:52-135) on the GPU path, on its kirsch_L0
mesh (golden fixture read by the reference's reader): linear displacement fields must be
reproduced exactly by the CST elements, through GPU assembly, GPU loads, GPU elimination and
the GPU Jacobi-PCG at rtol 1e-12.

  * Dirichlet patch: u = a0 + a1 x + a2 y, v = b0 + b1 x + b2 y prescribed on every boundary
    group; max |u - u_exact| / max |u_exact| < 1e-9 (plane stress and plane strain).
  * Neumann patch: the uniform stress (sxx, syy, 0) with symmetry BCs and the traction sigma . n
    on right, top and hole; the exact field ux = exx x, uy = eyy y; uniaxial and biaxial; < 1e-9.
  * Flipped normal: with the traction of one loaded group reversed the error exceeds 1e-2.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E, NU, T = 210e9, 0.3, 0.01
GROUPS = ("hole", "left_sym", "bottom_sym", "right", "top")


def _mesh(pkg, golden):
    return golden("kirsch_L0").mesh(pkg)


def _rel_error(m, u, exact):
    xy = np.asarray(m.xy).reshape(-1, 2)
    ue = np.array([exact(x, y) for x, y in xy])
    return np.abs(u.reshape(-1, 2) - ue).max() / np.abs(ue).max()


def _solve(pkg, m, plane, dofs, f):
    import torch
    K = pkg.build_stiffness_pattern(m)
    pkg.assemble_stiffness(m, pkg.constitutive_matrix(E, NU, plane), T, K)
    f = f if hasattr(f, "is_cuda") else torch.from_numpy(f).cuda()
    pkg.apply_dirichlet(dofs, K, f)
    s = pkg.CgJacobiSolver(pkg.SolverOptions(rtol=1e-12, max_iter=20000))
    s.setup(K)
    u = torch.empty_like(f)
    st = s.solve(f, u)
    K.ctx.close()
    return u.cpu().numpy(), st


@pytest.mark.parametrize("plane", [0, 1])
def test_dirichlet_patch(pkg, gpu_lib, golden, plane):
    m = _mesh(pkg, golden)
    a = (1e-4, 2e-3, -1e-3)
    b = (-5e-4, 1e-3, 3e-3)

    def exact(x, y):
        return (a[0] + a[1] * x + a[2] * y, b[0] + b[1] * x + b[2] * y)
    dofs = pkg.DirichletDofs()
    for g in GROUPS:
        pkg.add_dirichlet_group(m, g, 0, lambda x, y: exact(x, y)[0], dofs)
        pkg.add_dirichlet_group(m, g, 1, lambda x, y: exact(x, y)[1], dofs)
    u, st = _solve(pkg, m, plane, dofs, np.zeros(m.num_dofs))
    assert st.converged, st.message
    assert _rel_error(m, u, exact) < 1e-9


def _neumann_patch(pkg, m, plane, sxx, syy, flip=""):
    import torch
    stress = plane == 0
    Ep = E if stress else E / (1 - NU * NU)
    nup = NU if stress else NU / (1 - NU)
    exx, eyy = (sxx - nup * syy) / Ep, (syy - nup * sxx) / Ep
    K = pkg.build_stiffness_pattern(m)  # (a context for the loads: the pattern's node incidence)
    f = torch.zeros(m.num_dofs, dtype=torch.float64, device="cuda")
    for g in ("right", "top", "hole"):
        sgn = -1.0 if flip == g else 1.0
        pkg.add_stress_traction(K, m.boundary_edges[g], T, sgn * sxx, sgn * syy, f)
    K.ctx.close()
    dofs = pkg.DirichletDofs()
    pkg.add_dirichlet_group(m, "left_sym", 0, 0.0, dofs)
    pkg.add_dirichlet_group(m, "bottom_sym", 1, 0.0, dofs)
    u, st = _solve(pkg, m, plane, dofs, f)
    assert st.converged, st.message
    return _rel_error(m, u, lambda x, y: (exx * x, eyy * y))


@pytest.mark.parametrize("plane", [0, 1])
def test_neumann_patch(pkg, gpu_lib, golden, plane):
    m = _mesh(pkg, golden)
    s0 = 100e6
    assert _neumann_patch(pkg, m, plane, s0, 0.0) < 1e-9  # uniaxial
    assert _neumann_patch(pkg, m, plane, s0, -0.4 * s0) < 1e-9  # biaxial


@pytest.mark.parametrize("group", ["right", "top", "hole"])
def test_neumann_patch_detects_flipped_normal(pkg, gpu_lib, golden, group):
    m = _mesh(pkg, golden)
    assert _neumann_patch(pkg, m, 0, 100e6, -40e6, flip=group) > 1e-2
