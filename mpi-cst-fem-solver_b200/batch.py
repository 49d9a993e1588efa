"""Batched plates: many O-grid plates of uneven size, each with several load cases, solved in one
persistent launch (cstg_batch_solve).

The reference solves one plate and one load per run (src/driver.cpp:164-188). A batch is that
path applied to every (plate, load case): `build_batch` generates the plates, concatenates their
meshes (node indices offset per plate, so the global matrix is block diagonal), and computes
each case's consistent loads with the reference's traction rule (`cstg_add_traction`,
bc.cpp:190-253). `BatchSolver.setup` builds the pattern, assembles every plate with its own
material (`cstg_assemble_materials`), eliminates the symmetry conditions for all load vectors at
once (`cstg_apply_dirichlet_multi`) and sets up Jacobi; `solve` runs the batched Jacobi-PCG.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import native
from .native import CstgError
from .plate import LOAD_CASES, Mesh, quarter_plate, symmetry_dirichlet
from .solver import Context, GpuCsrMatrix, PlaneCondition, SolverOptions, _f64, _i32, _ptr, constitutive_matrix


@dataclasses.dataclass
class PlateBatch:
    """Concatenated plates: global mesh, per-plate node ranges, materials, BCs and loads."""
    specs: list
    mesh: Mesh                  # all plates, node indices offset per plate
    node_offsets: np.ndarray    # int32 [n_plates + 1]
    D: np.ndarray               # float64 [n_plates, 9]
    thickness: np.ndarray       # float64 [n_plates]
    material: np.ndarray        # int32 [n_triangles]: plate of each triangle
    dirichlet: tuple            # (dofs int32, values float64), sorted
    case_names: list
    loads: np.ndarray           # float64 [n_cases, n_dofs], before elimination

    @property
    def n_plates(self) -> int:
        return len(self.specs)

    @property
    def n_cases(self) -> int:
        return len(self.case_names)

    def dof_range(self, s: int) -> slice:
        return slice(2 * int(self.node_offsets[s]), 2 * int(self.node_offsets[s + 1]))


def build_batch(specs, cases: dict | None = None, ctx: Context | None = None) -> PlateBatch:
    """Generates the plates of `specs` (PlateSpec list) and the load vectors of `cases`
    ({name: [(group, tx, ty), ...]}, default the four LOAD_CASES) on their concatenation."""
    cases = cases or LOAD_CASES
    meshes = [quarter_plate(s.n_r, s.n_theta, a=s.a) for s in specs]
    offs = np.zeros(len(specs) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([m.num_nodes for m in meshes])
    if offs[-1] > np.iinfo(np.int32).max // 2:
        raise CstgError(native.ERR_INVALID_ARGUMENT, "build_batch: too many nodes for int32 DOFs")
    xy = np.concatenate([m.xy for m in meshes])
    tri = np.concatenate([m.triangles + np.int32(o) for m, o in zip(meshes, offs[:-1])]).astype(np.int32)
    groups = {g: np.concatenate([m.boundary_edges[g] + np.int32(o) for m, o in zip(meshes, offs[:-1])])
              for g in meshes[0].boundary_edges}
    mesh = Mesh(xy=xy, triangles=tri, boundary_edges=groups)
    D = np.stack([constitutive_matrix(s.E, s.nu, PlaneCondition.Strain if s.plane_strain
                                      else PlaneCondition.Stress) for s in specs])
    thickness = np.ones(len(specs))
    material = np.concatenate([np.full(m.num_triangles, k, dtype=np.int32) for k, m in enumerate(meshes)])
    dd, dv = zip(*(symmetry_dirichlet(m) for m in meshes))
    dofs = np.concatenate([d + np.int32(2 * o) for d, o in zip(dd, offs[:-1])]).astype(np.int32)
    vals = np.concatenate(dv)
    own = ctx is None
    ctx = ctx or Context()
    try:
        ctx.set_mesh(mesh)
        loads = np.zeros((len(cases), mesh.num_dofs))
        L = ctx.L
        for q, parts in enumerate(cases.values()):
            for group, tx, ty in parts:
                e = _i32(groups[group].reshape(-1))
                # thickness 1 on every plate: one call per (case, group) covers all plates
                ctx.check(L.cstg_add_traction(ctx.h, e.size // 2, _ptr(e), 1.0, float(tx), float(ty),
                                              _ptr(loads[q])))
    finally:
        if own:
            ctx.close()
    return PlateBatch(specs=list(specs), mesh=mesh, node_offsets=offs.astype(np.int32), D=D,
                      thickness=thickness, material=material, dirichlet=(dofs, vals),
                      case_names=list(cases), loads=loads)


@dataclasses.dataclass
class BatchSolution:
    x: object                  # [n_cases, n_dofs]: numpy (host solve) or a CUDA tensor (device solve)
    iterations: np.ndarray     # int [n_plates, n_cases]
    status: np.ndarray
    refinements: np.ndarray
    fp64: np.ndarray
    rel_residual: np.ndarray
    true_rel_residual: np.ndarray
    seconds: float
    config: tuple              # (cluster_ctas, threads) the solve ran with

    @property
    def converged(self) -> np.ndarray:
        return self.status == native.SOLVE_CONVERGED


class BatchSolver:
    """Batched Jacobi-PCG over a PlateBatch (one persistent launch of thread-block clusters)."""

    def __init__(self, options: SolverOptions | None = None, ctx: Context | None = None,
                 config: tuple | None = None):
        self.options = options or SolverOptions(precision="mixed", max_iter=200000)
        self.ctx = ctx or Context()
        self.config = config
        self.batch = None
        self.b = None
        self.d_b = self.d_x = None

    def setup(self, batch: PlateBatch, device_rhs: bool = False) -> GpuCsrMatrix:
        """Pattern, per-plate assembly, Dirichlet elimination of every load vector, Jacobi."""
        ctx, L = self.ctx, self.ctx.L
        ctx.set_mesh(batch.mesh)
        nnz = C.c_int64(0)
        ctx.check(L.cstg_build_pattern(ctx.h, C.byref(nnz)))
        D = _f64(batch.D.reshape(-1))
        t = _f64(batch.thickness)
        mat = _i32(batch.material)
        ctx.check(L.cstg_assemble_materials(ctx.h, batch.n_plates, _ptr(D), _ptr(t), _ptr(mat)))
        d, v = _i32(batch.dirichlet[0]), _f64(batch.dirichlet[1])
        b = np.ascontiguousarray(batch.loads, dtype=np.float64).copy()
        ctx.check(L.cstg_apply_dirichlet_multi(ctx.h, d.size, _ptr(d), _ptr(v), batch.n_cases, _ptr(b)))
        ctx.check(L.cstg_pcg_setup(ctx.h))
        self.batch = batch
        self.b = b
        if device_rhs:
            import torch
            self.d_b = torch.from_numpy(b).to(f"cuda:{ctx.device}")
            self.d_x = torch.zeros_like(self.d_b)
        K = GpuCsrMatrix(ctx)
        K.mesh = batch.mesh
        return K

    def _cfg(self, config):
        config = config or self.config
        if config is None:
            return None
        c = native.BatchConfig()
        c.cluster_ctas, c.threads = int(config[0]), int(config[1])
        return C.byref(c)

    def autotune(self, max_iter: int | None = None) -> tuple:
        """Times every feasible launch shape on this batch (device vectors) and keeps the
        fastest for later solves. max_iter bounds each trial solve."""
        import torch
        ctx, batch = self.ctx, self.batch
        if batch is None:
            raise CstgError(native.ERR_STATE, "autotune: call setup first")
        d_b = self.d_b if self.d_b is not None else torch.from_numpy(self.b).to(f"cuda:{ctx.device}")
        d_x = torch.zeros_like(d_b)
        o = self.options.native()
        if max_iter is not None:
            o.max_iter = int(max_iter)
        best = native.BatchConfig()
        sec = C.c_double(0.0)
        offs = _i32(batch.node_offsets)
        with ctx.ordered(d_b.device):
            ctx.check(ctx.L.cstg_batch_autotune(ctx.h, batch.n_plates, _ptr(offs), batch.n_cases, _ptr(d_b),
                                                _ptr(d_x), C.byref(o), C.byref(best), C.byref(sec)))
        self.config = (best.cluster_ctas, best.threads)
        return self.config, sec.value

    def solve(self, config: tuple | None = None, device: bool = False) -> BatchSolution:
        """Solves every (plate, load case). device=True: vectors stay on the GPU (setup with
        device_rhs=True) and x is returned as a tensor."""
        ctx, batch = self.ctx, self.batch
        if batch is None:
            raise CstgError(native.ERR_STATE, "batch_solve: call setup first")
        n_p, n_c = batch.n_plates, batch.n_cases
        res = (native.BatchResult * (n_p * n_c))()
        sec = C.c_double(0.0)
        o = self.options.native()
        offs = _i32(batch.node_offsets)
        cfg = self._cfg(config)
        if device:
            if self.d_b is None:
                raise CstgError(native.ERR_STATE, "batch_solve: setup(device_rhs=True) first")
            x = self.d_x
            with ctx.ordered(self.d_b.device):
                ctx.check(ctx.L.cstg_batch_solve_device(ctx.h, n_p, _ptr(offs), n_c, _ptr(self.d_b), _ptr(x),
                                                        C.byref(o), cfg, res, C.byref(sec)))
        else:
            x = np.zeros_like(self.b)
            ctx.check(ctx.L.cstg_batch_solve(ctx.h, n_p, _ptr(offs), n_c, _ptr(self.b), _ptr(x), C.byref(o),
                                             cfg, res, C.byref(sec)))

        def field(name, dtype):
            return np.array([getattr(r, name) for r in res], dtype=dtype).reshape(n_p, n_c)

        used = config or self.config or (8, 512)
        return BatchSolution(x=x, iterations=field("iterations", np.int64), status=field("status", np.int64),
                             refinements=field("refinements", np.int64), fp64=field("fp64", np.int64),
                             rel_residual=field("rel_residual", np.float64),
                             true_rel_residual=field("true_rel_residual", np.float64),
                             seconds=sec.value, config=tuple(used))

    def close(self):
        self.ctx.close()
