"""Host-side mirror of the reference's serial-core interface, over the C ABI.

Names, argument meaning and error behaviour follow FreddyJuka/mpi-cst-fem-solver:

==============================  =======================================================
reference (include/cstfem/...)  here
==============================  =======================================================
constitutive_matrix             constitutive_matrix          (element.hpp:18)
build_stiffness_pattern         build_stiffness_pattern      (assembly.hpp:15)
assemble_stiffness              assemble_stiffness           (assembly.hpp:22)
CsrMatrix / multiply            GpuCsrMatrix / .multiply     (csr.hpp:14-32)
DirichletDofs, add_dirichlet*   DirichletDofs, add_dirichlet_group (bc.hpp:28-48)
apply_dirichlet                 apply_dirichlet              (bc.hpp:53)
add_traction (constant)         add_traction                 (bc.hpp:74-75)
SolverOptions / SolverStats     SolverOptions / SolverStats  (solver.hpp:93-107)
CgJacobiSolver setup/solve      CgJacobiSolver               (solver.hpp:131-146)
pcg_jacobi                      pcg_jacobi                   (solver.hpp:115-118)
compute_element_stresses        compute_element_stresses     (postprocess.hpp:67-68)
==============================  =======================================================

The matrix lives on the GPU inside a Context (one matrix per context); exceptions of the
reference become CstgError (std::runtime_error) or LogicError (std::logic_error).
Vectors are numpy float64 arrays (host) or torch CUDA float64 tensors (device, no copies).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import dataclasses

import numpy as np

from . import native
from .native import CstgError, LogicError


class PlaneCondition:
    Stress = 0
    Strain = 1


def constitutive_matrix(E: float, nu: float, plane: int = PlaneCondition.Stress) -> np.ndarray:
    """Isotropic 3x3 D, row-major (element.cpp:7-15; same operations, so the same bits)."""
    if plane == PlaneCondition.Stress:
        c = E / (1.0 - nu * nu)
        return np.array([c, c * nu, 0.0, c * nu, c, 0.0, 0.0, 0.0, c * (1.0 - nu) / 2.0])
    c = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return np.array([c * (1.0 - nu), c * nu, 0.0, c * nu, c * (1.0 - nu), 0.0,
                     0.0, 0.0, c * (1.0 - 2.0 * nu) / 2.0])


def _is_device(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _f64(a):
    if _is_device(a):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise CstgError(native.ERR_INVALID_ARGUMENT, "device vectors must be contiguous float64")
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    if _is_device(a):
        import torch
        if a.dtype != torch.int32 or not a.is_contiguous():
            raise CstgError(native.ERR_INVALID_ARGUMENT, "device index arrays must be contiguous int32")
        return a
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One cstg_ctx: a device, a stream, and the mesh / matrix / solver buffers."""

    def __init__(self, device: int = 0):
        self.L = native.load()
        st = C.c_int(0)
        self.h = self.L.cstg_create(device, C.byref(st))
        if not self.h:
            raise CstgError(st.value, f"cstg_create(device={device}) failed (status {st.value})")
        self.device = device
        self.mesh = None

    def check(self, rc, what=""):
        native.check(self.L, self.h, rc, what)

    def set_stream(self, stream) -> None:
        """stream: a torch.cuda.Stream, a raw cudaStream_t (int) or None (own stream)."""
        ptr = getattr(stream, "cuda_stream", stream)
        self.check(self.L.cstg_set_stream(self.h, ptr or None))
        self._ext = None

    def set_wait_limits(self, barrier_polls: int = -1, mma_polls: int = -1) -> None:
        """Polls before a device wait gives up (cstg_set_wait_limits; -1: the default, 0: at once)."""
        self.check(self.L.cstg_set_wait_limits(self.h, int(barrier_polls), int(mma_polls)))

    def stream_handle(self) -> int:
        """The cudaStream_t the context's work is ordered on (cstg_get_stream)."""
        s = C.c_void_p(0)
        self.check(self.L.cstg_get_stream(self.h, C.byref(s)))
        return s.value or 0

    @contextlib.contextmanager
    def ordered(self, device):
        """Orders a device call between torch's current stream and the context's stream.

        The context works on its own stream, which torch does not know about: before the call
        the context's stream waits (an event, not a host synchronisation) for everything torch
        has queued so far, so inputs written by torch kernels or copies are complete; after it
        torch's current stream waits for the context's, so torch work issued afterwards sees
        the outputs, also of the entry points that return before their kernels have run."""
        import torch
        dev = torch.device(device)
        ext = getattr(self, "_ext", None)
        if ext is None:
            ext = torch.cuda.ExternalStream(self.stream_handle(), device=dev)
            self._ext = ext
        cur = torch.cuda.current_stream(dev)
        ext.wait_stream(cur)
        try:
            yield
        finally:
            cur.wait_stream(ext)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.cstg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_mesh(self, mesh) -> None:
        xy, tri = mesh.xy, mesh.triangles
        if _is_device(xy):
            with self.ordered(xy.device):
                self.check(self.L.cstg_set_mesh_device(self.h, xy.numel() // 2, _ptr(_f64(xy)),
                                                       tri.numel() // 3, _ptr(_i32(tri))))
        else:
            xy, tri = _f64(xy), _i32(tri)
            self.check(self.L.cstg_set_mesh(self.h, xy.size // 2, _ptr(xy), tri.size // 3, _ptr(tri)))
        self.mesh = mesh


class GpuCsrMatrix:
    """The reference's CsrMatrix (csr.hpp:14-32) held on the GPU by a Context: row_ptr int32,
    cols int32 sorted per row, vals float64, first_row = 0, num_rows = num_cols."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.first_row = 0

    @property
    def num_rows(self) -> int:
        n = C.c_int(0)
        nnz = C.c_int64(0)
        self.ctx.check(self.ctx.L.cstg_matrix_size(self.ctx.h, C.byref(n), C.byref(nnz)))
        return n.value

    num_cols = num_rows

    def nnz(self) -> int:
        n = C.c_int(0)
        nnz = C.c_int64(0)
        self.ctx.check(self.ctx.L.cstg_matrix_size(self.ctx.h, C.byref(n), C.byref(nnz)))
        return nnz.value

    def download(self, values: bool = True):
        """(row_ptr, cols, vals) as host arrays; vals is None when values=False."""
        n, nnz = self.num_rows, self.nnz()
        rp = np.zeros(n + 1, dtype=np.int32)
        cols = np.zeros(nnz, dtype=np.int32)
        vals = np.zeros(nnz) if values else None
        self.ctx.check(self.ctx.L.cstg_get_csr(self.ctx.h, _ptr(rp), _ptr(cols), _ptr(vals)))
        return rp, cols, vals

    @classmethod
    def from_csr(cls, row_ptr, cols, vals, ctx: Context | None = None) -> "GpuCsrMatrix":
        ctx = ctx or Context()
        rp, c, v = _i32(row_ptr), _i32(cols), _f64(vals)
        ctx.check(ctx.L.cstg_set_csr(ctx.h, rp.size - 1, _ptr(rp), _ptr(c), _ptr(v)))
        return cls(ctx)

    def multiply(self, x, y=None):
        """y = A x (csr.cpp:19-26)."""
        x = _f64(x)
        if _is_device(x):
            import torch
            y = torch.empty_like(x) if y is None else y
            with self.ctx.ordered(x.device):
                self.ctx.check(self.ctx.L.cstg_multiply_device(self.ctx.h, _ptr(x), _ptr(y)))
            return y
        y = np.zeros(self.num_rows) if y is None else y
        self.ctx.check(self.ctx.L.cstg_multiply(self.ctx.h, _ptr(x), _ptr(y)))
        return y

    def multiply_mixed(self, x, y=None):
        """y = K x with the mixed-precision SpMV (FP32 difference-form matrix, FP64 vectors and
        accumulation); torch CUDA float64 tensors; needs the mesh pattern and a solver setup on
        this matrix. Asynchronous on the context's stream."""
        import torch
        if not (_is_device(x) and x.dtype == torch.float64 and x.is_contiguous()):
            raise CstgError(native.ERR_INVALID_ARGUMENT, "multiply_mixed: x must be a contiguous CUDA float64 tensor")
        y = torch.empty_like(x) if y is None else y
        with self.ctx.ordered(x.device):
            self.ctx.check(self.ctx.L.cstg_multiply_mixed_device(self.ctx.h, _ptr(x), _ptr(y)))
        return y


def build_stiffness_pattern(mesh, ctx: Context | None = None) -> GpuCsrMatrix:
    """Sparsity pattern of K: one 2x2 block per pair of nodes sharing a triangle, self
    included, sorted (assembly.cpp:9-42). Values are left unassembled."""
    ctx = ctx or Context()
    ctx.set_mesh(mesh)
    nnz = C.c_int64(0)
    ctx.check(ctx.L.cstg_build_pattern(ctx.h, C.byref(nnz)))
    K = GpuCsrMatrix(ctx)
    K.mesh = mesh
    return K


def assemble_stiffness(mesh, D, thickness: float, K: GpuCsrMatrix) -> None:
    """Zeroes K's values and adds Ke of every triangle (assembly.cpp:54-74), bit-identical to
    the reference. K must carry the pattern built from this mesh."""
    if getattr(K, "mesh", None) is not mesh:
        raise LogicError(native.ERR_STATE, "assemble_stiffness: K does not have the pattern of this mesh")
    D = np.ascontiguousarray(D, dtype=np.float64).reshape(9)
    K.ctx.check(K.ctx.L.cstg_assemble(K.ctx.h, _ptr(D), float(thickness)))


class DirichletDofs:
    """Prescribed DOF values keyed by DOF index (bc.hpp:28-38)."""

    def __init__(self):
        self._v = {}

    def add(self, dof: int, value: float) -> None:
        old = self._v.setdefault(int(dof), float(value))
        if old != value:
            raise CstgError(native.ERR_DIRICHLET_CONFLICT,
                            f"conflicting Dirichlet values for node {dof // 2} (0-based) component "
                            f"{'ux' if dof % 2 == 0 else 'uy'}: {old!r} vs {value!r}")

    def values(self) -> dict:
        return dict(sorted(self._v.items()))

    def size(self) -> int:
        return len(self._v)

    def arrays(self):
        items = sorted(self._v.items())
        return (np.array([k for k, _ in items], dtype=np.int32),
                np.array([v for _, v in items], dtype=np.float64))


def add_dirichlet_group(mesh, group: str, component: int, value, dofs: DirichletDofs) -> None:
    """Prescribes component (0 = ux, 1 = uy) on every node of a line group (bc.cpp:118-130).
    value: a number or a callable f(x, y)."""
    if group not in mesh.boundary_edges:
        raise CstgError(native.ERR_INVALID_ARGUMENT, f"unknown boundary group '{group}'")
    xy = np.asarray(mesh.xy).reshape(-1, 2)
    for a, b in np.asarray(mesh.boundary_edges[group]).reshape(-1, 2):
        for n in (int(a), int(b)):
            v = value(xy[n, 0], xy[n, 1]) if callable(value) else value
            dofs.add(2 * n + component, v)


def apply_dirichlet(dofs, K: GpuCsrMatrix, b) -> None:
    """Symmetric elimination on K (on the GPU) and b (in place), bc.cpp:137-166.
    dofs: DirichletDofs or a (dofs int32, values float64) pair."""
    d, v = dofs.arrays() if isinstance(dofs, DirichletDofs) else dofs
    if _is_device(b):
        import torch
        d = torch.as_tensor(d, dtype=torch.int32, device=b.device).contiguous()
        v = torch.as_tensor(v, dtype=torch.float64, device=b.device).contiguous()
        with K.ctx.ordered(b.device):
            K.ctx.check(K.ctx.L.cstg_apply_dirichlet_device(K.ctx.h, d.numel(), _ptr(d), _ptr(v), _ptr(b)))
        return
    if not (isinstance(b, np.ndarray) and b.dtype == np.float64 and b.flags.c_contiguous):
        raise CstgError(native.ERR_INVALID_ARGUMENT, "apply_dirichlet: b must be a float64 C array")
    d, v = _i32(d), _f64(v)
    K.ctx.check(K.ctx.L.cstg_apply_dirichlet(K.ctx.h, d.size, _ptr(d), _ptr(v), _ptr(b)))


def add_traction(K_or_ctx, group_edges, thickness: float, tx: float, ty: float, f) -> None:
    """Consistent nodal forces of a constant traction on line edges (bc.cpp:190-253), added to
    f. Host f (numpy): computed on the host from the context's host mesh. CUDA f (torch): on the
    GPU with the pattern's node incidence (cstg_add_traction_device); same bits either way."""
    ctx = K_or_ctx.ctx if isinstance(K_or_ctx, GpuCsrMatrix) else K_or_ctx
    if _is_device(f):
        _traction_device(ctx, group_edges, thickness, native.TRACTION_CONSTANT, tx, ty, f)
        return
    e = _i32(np.asarray(group_edges).reshape(-1))
    ctx.check(ctx.L.cstg_add_traction(ctx.h, e.size // 2, _ptr(e), float(thickness), float(tx),
                                      float(ty), _ptr(f)))


def add_kirsch_traction(K_or_ctx, group_edges, thickness: float, a: float, sigma_inf: float, f) -> None:
    """Traction sigma . n of the analytical Kirsch field (kirsch.cpp:40-45) on line edges, added
    to the CUDA tensor f on the GPU."""
    ctx = K_or_ctx.ctx if isinstance(K_or_ctx, GpuCsrMatrix) else K_or_ctx
    if not _is_device(f):
        raise CstgError(native.ERR_INVALID_ARGUMENT, "add_kirsch_traction: f must be a CUDA float64 tensor")
    _traction_device(ctx, group_edges, thickness, native.TRACTION_KIRSCH, a, sigma_inf, f)


def add_stress_traction(K_or_ctx, group_edges, thickness: float, sxx: float, syy: float, f) -> None:
    """Traction sigma . n of the uniform stress diag(sxx, syy) on line edges (outward normals),
    added to the CUDA tensor f on the GPU: the loads of the reference's Neumann patch tests."""
    ctx = K_or_ctx.ctx if isinstance(K_or_ctx, GpuCsrMatrix) else K_or_ctx
    if not _is_device(f):
        raise CstgError(native.ERR_INVALID_ARGUMENT, "add_stress_traction: f must be a CUDA float64 tensor")
    _traction_device(ctx, group_edges, thickness, native.TRACTION_STRESS, sxx, syy, f)


def _traction_device(ctx, group_edges, thickness, kind, p0, p1, f):
    # cstg_add_traction_device only enqueues its kernels on the context's stream: ctx.ordered
    # puts them after torch's pending work (the edge list copy, f) and torch's later work after them
    import torch
    e = torch.as_tensor(np.asarray(group_edges).reshape(-1) if not _is_device(group_edges) else group_edges,
                        dtype=torch.int32, device=f.device).contiguous()
    f = _f64(f)
    with ctx.ordered(f.device):
        ctx.check(ctx.L.cstg_add_traction_device(ctx.h, e.numel() // 2, _ptr(e), float(thickness), int(kind),
                                                 float(p0), float(p1), _ptr(f)))


@dataclasses.dataclass
class SolverOptions:
    """solver.hpp:93-97 plus precision / true-residual stopping / refinement controls."""
    rtol: float = 1e-10
    max_iter: int = 20000
    record_history: bool = False
    precision: str = "fp64"  # "fp64" | "mixed"
    true_residual_stop: bool = False
    max_refinements: int = 16
    check_interval: int = 0
    launch: str = "auto"  # "auto" | "persistent" | "graph" | "instrumented" (phase times: breakdown())
    # "jacobi" | "learned" (the network alone in flexible CG; needs learned setup) | "amg" |
    # "learned_mg" (the network as the multigrid cycle's post-smoother; needs learned setup)
    preconditioner: str = "jacobi"
    fcg_depth: int = 0  # flexible CG: earlier directions each new one is A-orthogonalised against (0: auto)

    def native(self) -> native.SolverOptions:
        o = native.default_options()
        o.rtol = self.rtol
        o.max_iter = self.max_iter
        o.record_history = int(self.record_history)
        o.precision = {"fp64": native.PRECISION_FP64, "mixed": native.PRECISION_MIXED}[self.precision]
        o.true_residual_stop = int(self.true_residual_stop)
        o.max_refinements = self.max_refinements
        o.check_interval = self.check_interval
        o.launch_mode = {"auto": native.LAUNCH_AUTO, "persistent": native.LAUNCH_PERSISTENT,
                         "graph": native.LAUNCH_GRAPH, "instrumented": native.LAUNCH_INSTRUMENTED}[self.launch]
        o.preconditioner = {"jacobi": native.PRECOND_JACOBI, "learned": native.PRECOND_LEARNED,
                            "amg": native.PRECOND_AMG,
                            "learned_mg": native.PRECOND_LEARNED_MG}[self.preconditioner]
        o.fcg_depth = self.fcg_depth
        return o


@dataclasses.dataclass
class SolverStats:
    """solver.hpp:99-107 plus the B200 counters."""
    iterations: int = 0
    rel_residual: float = 0.0
    true_rel_residual: float = 0.0
    converged: bool = False
    message: str = ""
    warning: str = ""
    residual_history: list = dataclasses.field(default_factory=list)
    status: int = 0
    refinements: int = 0
    solve_seconds: float = 0.0
    spmv_calls: int = 0


class CgJacobiSolver:
    """Jacobi-preconditioned CG on the GPU (solver.hpp:131-146)."""

    def __init__(self, options: SolverOptions | None = None):
        self.options = options or SolverOptions()
        self.A = None
        self._stats = SolverStats()

    def setup(self, A: GpuCsrMatrix) -> None:
        """inv_diag = 1 / A_ii; raises CstgError on a non-positive diagonal (solver.cpp:133-148)."""
        A.ctx.check(A.ctx.L.cstg_pcg_setup(A.ctx.h))
        self.A = A

    def solve(self, b, x=None) -> SolverStats:
        """Solves A x = b from x = 0 (pcg_jacobi, solver.cpp:109-131). x: output array of
        n doubles (numpy, or a torch CUDA tensor when b is one); the solution is also kept in
        self.x. Check the returned stats: converged may be false."""
        if self.A is None:
            raise LogicError(native.ERR_STATE, "cg_jacobi: solve() called before setup()")
        ctx = self.A.ctx
        o = self.options.native()
        st = native.Stats()
        b = _f64(b)
        dev = _is_device(b)
        if dev:
            import torch
            n = b.numel()
            x = torch.empty_like(b) if x is None else x
            hist = torch.zeros(o.max_iter + 1, dtype=torch.float64, device=b.device) \
                if self.options.record_history else None
            with ctx.ordered(b.device):
                ctx.check(ctx.L.cstg_pcg_solve_device(ctx.h, _ptr(b), _ptr(x), C.byref(o), C.byref(st),
                                                      _ptr(hist)))
        else:
            n = b.size
            x = np.zeros(n) if x is None else x
            hist = np.zeros(o.max_iter + 1) if self.options.record_history else None
            ctx.check(ctx.L.cstg_pcg_solve(ctx.h, _ptr(b), _ptr(x), C.byref(o), C.byref(st), _ptr(hist)))
        s = SolverStats(iterations=st.iterations, rel_residual=st.rel_residual,
                        true_rel_residual=st.true_rel_residual, converged=bool(st.converged),
                        message=st.message.decode(), warning=st.warning.decode(), status=st.status,
                        refinements=st.refinements, solve_seconds=st.solve_seconds,
                        spmv_calls=st.spmv_calls)
        if hist is not None:
            cnt = 1 if st.status == native.SOLVE_ZERO_RHS else st.iterations + 1
            h = hist[:cnt]
            s.residual_history = (h.cpu().numpy() if dev else h).tolist()
        self.x = x
        self._stats = s
        return s

    def stats(self) -> SolverStats:
        return self._stats

    def breakdown(self) -> dict:
        """The reference's SolveBreakdown fields (solver.hpp:17-56) of the last solve run with
        launch="instrumented": device seconds of each phase (CUDA events) and the counts."""
        bd = native.Breakdown()
        self.A.ctx.check(self.A.ctx.L.cstg_solve_breakdown(self.A.ctx.h, C.byref(bd)))
        return {"setup": bd.setup, "spmv_local": bd.spmv_local, "dot_local": bd.dot_local,
                "vector_ops": bd.vector_ops, "total": bd.total, "spmv_calls": bd.spmv_calls,
                "reductions": bd.reductions}


def pcg_jacobi(A: GpuCsrMatrix, b, x=None, options: SolverOptions | None = None) -> SolverStats:
    """pcg_jacobi on the GPU with the Jacobi preconditioner of A (solver.hpp:115-118)."""
    s = CgJacobiSolver(options)
    s.setup(A)
    return s.solve(b, x)


def compute_element_stresses(ctx_or_K, u, E: float, nu: float, plane: int = PlaneCondition.Stress) -> dict:
    """Constant stress of every element plus centroid and area (postprocess.cpp:35-60)."""
    ctx = ctx_or_K.ctx if isinstance(ctx_or_K, GpuCsrMatrix) else ctx_or_K
    u = np.ascontiguousarray(u, dtype=np.float64)
    ne = ctx.mesh.num_triangles
    out = np.zeros(8 * ne)
    ctx.check(ctx.L.cstg_element_stresses(ctx.h, _ptr(u), float(E), float(nu), int(plane), _ptr(out)))
    names = ["sxx", "syy", "txy", "von_mises", "szz", "cx", "cy", "area"]
    return {k: out[i * ne:(i + 1) * ne] for i, k in enumerate(names)}


def scf_at_hole(stresses: dict, a: float, sigma_inf: float = 1.0):
    """SCF = sigma_xx / sigma_inf at the element whose centroid is closest to (0, a), the
    first such element on ties (postprocess.cpp:101-105,134-140). Returns (scf, element)."""
    d = np.hypot(stresses["cx"], stresses["cy"] - a)
    e = int(np.argmin(d))
    return stresses["sxx"][e] / sigma_inf, e


def amg_setup(K: GpuCsrMatrix) -> dict:
    """Builds the multigrid hierarchy of K (after CgJacobiSolver.setup) and describes it."""
    info = native.AmgInfo()
    K.ctx.check(K.ctx.L.cstg_amg_setup(K.ctx.h, C.byref(info)))
    return {"levels": info.levels, "dofs": list(info.dofs[:info.levels]), "nnz": list(info.nnz[:info.levels]),
            "setup_seconds": info.setup_seconds, "tail_level": info.tail_level, "tail_cluster": info.tail_cluster}


def amg_set_smoother(K: GpuCsrMatrix, kind: str) -> None:
    """The cycle's smoother: "chebyshev" (degree 2, the default) or "jacobi" (damped)."""
    code = {"chebyshev": 0, "jacobi": 1}[kind]
    K.ctx.check(K.ctx.L.cstg_amg_set_smoother(K.ctx.h, code))


def amg_set_strength(K: GpuCsrMatrix, theta_fine: float = 0.0, theta_coarse: float = 0.03) -> None:
    """Strength-of-connection thresholds of the aggregation (finest level, coarser levels); the
    hierarchy is rebuilt on next use when they change."""
    K.ctx.check(K.ctx.L.cstg_amg_set_strength(K.ctx.h, float(theta_fine), float(theta_coarse)))


def amg_set_tail(K: GpuCsrMatrix, enable: bool) -> None:
    """Runs the small coarse levels as one cluster launch (True, the default) or level by level."""
    K.ctx.check(K.ctx.L.cstg_amg_set_tail(K.ctx.h, int(bool(enable))))


def amg_apply(K: GpuCsrMatrix, r, z=None):
    """z = M r (one V-cycle) on CUDA float64 tensors."""
    import torch
    z = torch.empty_like(r) if z is None else z
    with K.ctx.ordered(r.device):
        K.ctx.check(K.ctx.L.cstg_amg_apply_device(K.ctx.h, _ptr(r), _ptr(z)))
    return z


def amg_time(K: GpuCsrMatrix, reps: int = 20) -> dict:
    """Seconds per finest-level smoothing sweep and per V-cycle (CUDA events, back to back)."""
    out = (C.c_double * 2)()
    K.ctx.check(K.ctx.L.cstg_amg_time(K.ctx.h, int(reps), out))
    return {"sweep_s": out[0], "vcycle_s": out[1]}

