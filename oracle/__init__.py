"""CPU oracle for the CST assembly -> Dirichlet elimination -> Jacobi-PCG path.

TEST INFRASTRUCTURE ONLY. Two checkers live here, both CPU code:

* `cst_oracle.c` (loaded through `Oracle`) restates the reference's serial core
  (FreddyJuka/mpi-cst-fem-solver: src/element.cpp, src/assembly.cpp, src/csr.cpp, src/bc.cpp,
  src/solver.cpp) operation for operation, so its results are bit-identical to the reference;
* `RefCore` loads `_ref/libcstfem_ref.so`, the reference's own serial core compiled from its
  sources by `Makefile` (`make ref`), when that build exists.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs import this
package, as the thing results are checked or timed against; the GPU library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcst_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcstfem_ref.so")
# Reference checkout whose sources `make ref` compiles (the Makefile's REF): the directory
# `reference` beside this repository unless CSTFEM_REF names another.
REF_DIR = os.environ.get("CSTFEM_REF", os.path.abspath(os.path.join(HERE, "..", "..", "reference")))


def ref_sources_present() -> bool:
    return os.path.isfile(os.path.join(REF_DIR, "src", "solver.cpp"))

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OracleError(RuntimeError):
    pass


def build(ref: bool = False) -> None:
    """Compile the restatement (and the reference core when `ref` and its sources exist)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_DIR}"] + targets, check=True)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("breakdown", C.c_int),
                ("rel_residual", C.c_double), ("true_rel_residual", C.c_double)]


class Oracle:
    """ctypes front of oracle/cst_oracle.c; names follow the reference's functions."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.or_last_message.restype = C.c_char_p
        L.or_constitutive.argtypes = [C.c_double, C.c_double, C.c_int, _dp]
        L.or_signed_area.argtypes = [_dp]
        L.or_signed_area.restype = C.c_double
        L.or_cst_stiffness.argtypes = [_dp, _dp, C.c_double, _dp]
        L.or_element_stress.argtypes = [_dp, _dp, _dp, C.c_double, C.c_int, _dp]
        L.or_build_pattern.argtypes = [C.c_int, C.c_int, _ip, C.c_void_p, C.c_void_p]
        L.or_build_pattern.restype = C.c_longlong
        L.or_assemble.argtypes = [C.c_int, _dp, C.c_int, _ip, _dp, C.c_double, _ip, _ip, _dp]
        L.or_spmv.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
        L.or_apply_dirichlet.argtypes = [C.c_int, _ip, _ip, _dp, C.c_int, _ip, _dp, _dp]
        L.or_add_traction.argtypes = [C.c_int, _dp, C.c_int, _ip, C.c_int, _ip, C.c_double,
                                      C.c_double, C.c_double, _dp]
        L.or_pcg_jacobi.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_int,
                                    C.c_void_p, C.POINTER(_Stats)]
        L.mp_param_count.restype = C.c_long
        L.mp_round_bf16.argtypes = [C.c_double]
        L.mp_round_bf16.restype = C.c_double
        L.mp_features.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.mp_forward.argtypes = [C.c_int, _ip, _ip, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
        L.mp_apply.argtypes = [C.c_int, _dp, _dp, C.c_double, _dp, _dp]
        L.mp_loss.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, C.c_double, _dp, C.c_void_p]
        L.mp_loss.restype = C.c_double
        L.mp_loss_cycle.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp,
                                    C.c_void_p]
        L.mp_loss_cycle.restype = C.c_double
        L.mp_backward.argtypes = [C.c_int, _ip, _ip, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        self.L = L

    def _err(self, what):
        raise OracleError(f"{what}: {self.L.or_last_message().decode()}")

    # element.cpp
    def constitutive_matrix(self, E, nu, plane_strain=False):
        D = np.zeros(9)
        self.L.or_constitutive(E, nu, int(plane_strain), D)
        return D

    def cst_signed_area(self, xy6):
        return self.L.or_signed_area(_f64(xy6))

    def cst_stiffness(self, xy6, D, t):
        K = np.zeros(36)
        self.L.or_cst_stiffness(_f64(xy6), _f64(D), t, K)
        return K

    def element_stress(self, xy6, ue, D, nu, plane_strain=False):
        out = np.zeros(5)
        self.L.or_element_stress(_f64(xy6), _f64(ue), _f64(D), nu, int(plane_strain), out)
        return out

    # assembly.cpp / csr.cpp
    def build_stiffness_pattern(self, n_nodes, triangles):
        tri = _i32(triangles)
        row_ptr = np.zeros(2 * n_nodes + 1, dtype=np.int32)
        nnz = self.L.or_build_pattern(n_nodes, tri.size // 3, tri, row_ptr.ctypes.data, None)
        if nnz < 0:
            self._err("build_stiffness_pattern")
        cols = np.zeros(max(nnz, 1), dtype=np.int32)[:nnz]
        self.L.or_build_pattern(n_nodes, tri.size // 3, tri, row_ptr.ctypes.data, cols.ctypes.data)
        return row_ptr, cols

    def assemble_stiffness(self, xy, triangles, D, t, row_ptr, cols):
        xy, tri = _f64(xy), _i32(triangles)
        vals = np.zeros(cols.size)
        if self.L.or_assemble(xy.size // 2, xy, tri.size // 3, tri, _f64(D), t, _i32(row_ptr),
                              _i32(cols), vals):
            self._err("assemble_stiffness")
        return vals

    def multiply(self, row_ptr, cols, vals, x):
        y = np.zeros(row_ptr.size - 1)
        self.L.or_spmv(row_ptr.size - 1, _i32(row_ptr), _i32(cols), _f64(vals), _f64(x), y)
        return y

    # bc.cpp
    def apply_dirichlet(self, row_ptr, cols, vals, dofs, values, b):
        """In place on vals and b (both float64 C-contiguous), like the reference."""
        assert vals.dtype == np.float64 and b.dtype == np.float64
        d, v = _i32(dofs), _f64(values)
        if self.L.or_apply_dirichlet(row_ptr.size - 1, _i32(row_ptr), _i32(cols), vals, d.size, d,
                                     v, b):
            self._err("apply_dirichlet")

    def add_traction(self, xy, triangles, edges, thickness, tx, ty, f):
        xy, tri, e = _f64(xy), _i32(triangles), _i32(edges).reshape(-1)
        if self.L.or_add_traction(xy.size // 2, xy, tri.size // 3, tri, e.size // 2, e, thickness,
                                  tx, ty, f):
            self._err("add_traction")

    # solver.cpp
    def pcg_jacobi(self, row_ptr, cols, vals, b, rtol=1e-10, max_iter=20000, record_history=False):
        n = row_ptr.size - 1
        x = np.zeros(n)
        hist = np.zeros(max_iter + 1) if record_history else None
        st = _Stats()
        rc = self.L.or_pcg_jacobi(n, _i32(row_ptr), _i32(cols), _f64(vals), _f64(b), x, rtol, max_iter,
                                  hist.ctypes.data if hist is not None else None, C.byref(st))
        if rc:
            self._err("pcg_jacobi")
        stats = dict(iterations=st.iterations, converged=bool(st.converged),
                     breakdown=bool(st.breakdown), rel_residual=st.rel_residual,
                     true_rel_residual=st.true_rel_residual,
                     message=self.L.or_last_message().decode())
        if hist is not None:
            stats["residual_history"] = hist[: (st.iterations + 1 if st.iterations or st.converged else 1)]
        return x, stats


    # ---- the learned preconditioner's network (mpnn_oracle.c; no reference counterpart) ----
    MP_F, MP_L = 64, 3

    def mp_param_count(self):
        return int(self.L.mp_param_count())

    def mp_round_bf16(self, a):
        return np.array([self.L.mp_round_bf16(float(v)) for v in np.ravel(a)]).reshape(np.shape(a))

    def mp_features(self, r, invd, xy, mat, coord_scale=10.0):
        """Network inputs (N x 8) and the residual scale s = RMS(r)."""
        r, invd = _f64(r), _f64(invd)
        N = r.size // 2
        s = float(np.sqrt(np.dot(r, r) / r.size))
        d_mean = float(np.mean(1.0 / invd))
        X = np.zeros(N * 8)
        self.L.mp_features(N, r, invd, _f64(xy), _f64(mat), s, d_mean, float(coord_scale), X)
        return X, s

    def mp_forward(self, node_ptr, nbr, X, P, q=True):
        N = node_ptr.size - 1
        F, L = self.MP_F, self.MP_L
        H = np.zeros((L + 1) * N * F)
        G = np.zeros(L * N * F)
        A = np.zeros(L * N * F)
        Y = np.zeros(N * 2)
        self.L.mp_forward(N, _i32(node_ptr), _i32(nbr), _f64(X), _f64(P), int(q), H, G, A, Y)
        return Y, (H, G, A)

    def mp_apply(self, r, invd, s, Y):
        z = np.zeros(_f64(r).size)
        self.L.mp_apply(z.size // 2, _f64(r), _f64(invd), float(s), _f64(Y), z)
        return z

    def mp_loss(self, rp, cols, vals, r, e, invd, s, Y, grad=True):
        dY = np.zeros(_f64(r).size) if grad else None
        L = self.L.mp_loss(_f64(r).size // 2, _i32(rp), _i32(cols), _f64(vals), _f64(r), _f64(e), _f64(invd),
                           float(s), _f64(Y), dY.ctypes.data if grad else None)
        return L, dY

    def mp_loss_cycle(self, rp, cols, vals, r, e, xfix, r2, winvd, s, Y, grad=True):
        """Loss of the learned multigrid cycle's output z = xfix + winvd (r2 + s Y) and dL/dY."""
        dY = np.zeros(_f64(r).size) if grad else None
        L = self.L.mp_loss_cycle(_f64(r).size // 2, _i32(rp), _i32(cols), _f64(vals), _f64(r), _f64(e), _f64(xfix),
                                 _f64(r2), _f64(winvd), float(s), _f64(Y), dY.ctypes.data if grad else None)
        return L, dY

    def mp_backward(self, node_ptr, nbr, X, P, cache, dY, q=True):
        N = node_ptr.size - 1
        H, G, A = cache
        dP = np.zeros(self.mp_param_count())
        w = [np.zeros(N * self.MP_F) for _ in range(3)]
        self.L.mp_backward(N, _i32(node_ptr), _i32(nbr), _f64(X), _f64(P), int(q), H, G, A, _f64(dY), dP, *w)
        return dP


class _RefStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rel_residual", C.c_double),
                ("true_rel_residual", C.c_double), ("t_setup", C.c_double), ("t_solve", C.c_double),
                ("t_spmv", C.c_double), ("t_dot", C.c_double), ("t_vec", C.c_double)]


class RefCore:
    """The reference's own serial core (oracle/_ref/libcstfem_ref.so via oracle/ref_shim.cpp)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise OracleError(f"{REF_SO} missing: run `make -C oracle ref` where the reference "
                              "sources are present")
        L = C.CDLL(REF_SO)
        L.ref_last_message.restype = C.c_char_p
        L.ref_mesh_create.restype = C.c_void_p
        L.ref_mesh_create.argtypes = [C.c_int, _dp, C.c_int, _ip]
        L.ref_mesh_add_group.argtypes = [C.c_void_p, C.c_char_p, C.c_int, _ip]
        L.ref_mesh_read.restype = C.c_void_p
        L.ref_mesh_read.argtypes = [C.c_char_p]
        L.ref_mesh_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3
        L.ref_mesh_get.argtypes = [C.c_void_p, _dp, _ip]
        L.ref_mesh_group.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.ref_mesh_destroy.argtypes = [C.c_void_p]
        L.ref_constitutive.argtypes = [C.c_double, C.c_double, C.c_int, _dp]
        L.ref_cst_stiffness.argtypes = [_dp, _dp, C.c_double, _dp]
        L.ref_pattern.restype = C.c_void_p
        L.ref_pattern.argtypes = [C.c_void_p]
        L.ref_csr_create.restype = C.c_void_p
        L.ref_csr_create.argtypes = [C.c_int, _ip, _ip, _dp]
        L.ref_csr_nnz.restype = C.c_longlong
        L.ref_csr_nnz.argtypes = [C.c_void_p]
        L.ref_csr_rows.argtypes = [C.c_void_p]
        L.ref_csr_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_csr_destroy.argtypes = [C.c_void_p]
        L.ref_assemble.argtypes = [C.c_void_p, _dp, C.c_double, C.c_void_p]
        L.ref_spmv.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_add_traction.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double, _dp]
        L.ref_dirichlet_dofs.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_char_p),
                                         C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p,
                                         C.c_void_p]
        L.ref_apply_dirichlet.argtypes = [C.c_void_p, C.c_int, _ip, _dp, _dp]
        L.ref_pcg.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int, C.c_void_p,
                              C.POINTER(_RefStats), C.c_char_p, C.c_char_p]
        L.ref_element_stresses.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double, C.c_int, _dp]
        self.L = L

    def _err(self, what):
        raise OracleError(f"{what}: {self.L.ref_last_message().decode()}")

    # mesh
    def mesh_from_arrays(self, xy, triangles, groups=None):
        xy, tri = _f64(xy), _i32(triangles)
        m = self.L.ref_mesh_create(xy.size // 2, xy, tri.size // 3, tri)
        for name, e in (groups or {}).items():
            e = _i32(e).reshape(-1)
            self.L.ref_mesh_add_group(m, name.encode(), e.size // 2, e)
        return m

    def read_gmsh(self, path):
        m = self.L.ref_mesh_read(path.encode())
        if not m:
            self._err("read_gmsh")
        return m

    def mesh_arrays(self, m, group_names=()):
        nn, nt, fl = C.c_int(), C.c_int(), C.c_int()
        self.L.ref_mesh_info(m, C.byref(nn), C.byref(nt), C.byref(fl))
        xy = np.zeros(2 * nn.value)
        tri = np.zeros(3 * nt.value, dtype=np.int32)
        self.L.ref_mesh_get(m, xy, tri)
        groups = {}
        for g in group_names:
            k = self.L.ref_mesh_group(m, g.encode(), None)
            if k >= 0:
                e = np.zeros(2 * k, dtype=np.int32)
                self.L.ref_mesh_group(m, g.encode(), e.ctypes.data)
                groups[g] = e.reshape(-1, 2)
        return xy, tri, groups, fl.value

    def free_mesh(self, m):
        self.L.ref_mesh_destroy(m)

    # element
    def constitutive_matrix(self, E, nu, plane_strain=False):
        D = np.zeros(9)
        self.L.ref_constitutive(E, nu, int(plane_strain), D)
        return D

    def cst_stiffness(self, xy6, D, t):
        K = np.zeros(36)
        self.L.ref_cst_stiffness(_f64(xy6), _f64(D), t, K)
        return K

    # CSR
    def pattern(self, m):
        return self.L.ref_pattern(m)

    def csr(self, n, row_ptr, cols, vals):
        return self.L.ref_csr_create(n, _i32(row_ptr), _i32(cols), _f64(vals))

    def csr_arrays(self, K):
        n = self.L.ref_csr_rows(K)
        nnz = self.L.ref_csr_nnz(K)
        rp = np.zeros(n + 1, dtype=np.int32)
        cols = np.zeros(nnz, dtype=np.int32)
        vals = np.zeros(nnz)
        self.L.ref_csr_get(K, rp.ctypes.data, cols.ctypes.data, vals.ctypes.data)
        return rp, cols, vals

    def free_csr(self, K):
        self.L.ref_csr_destroy(K)

    def assemble(self, m, D, t, K):
        if self.L.ref_assemble(m, _f64(D), t, K):
            self._err("assemble_stiffness")

    def multiply(self, K, x):
        y = np.zeros(self.L.ref_csr_rows(K))
        self.L.ref_spmv(K, _f64(x), y)
        return y

    def add_traction(self, m, group, t, tx, ty, f):
        if self.L.ref_add_traction(m, group.encode(), t, tx, ty, f):
            self._err("add_traction")

    def dirichlet_dofs(self, m, specs):
        """specs: [(group, component, value)] -> sorted (dofs, values) (DirichletDofs order)."""
        k = len(specs)
        g = (C.c_char_p * k)(*[s[0].encode() for s in specs])
        c = (C.c_int * k)(*[s[1] for s in specs])
        v = (C.c_double * k)(*[s[2] for s in specs])
        cnt = self.L.ref_dirichlet_dofs(m, k, g, c, v, None, None)
        if cnt < 0:
            self._err("add_dirichlet")
        d = np.zeros(cnt, dtype=np.int32)
        vals = np.zeros(cnt)
        self.L.ref_dirichlet_dofs(m, k, g, c, v, d.ctypes.data, vals.ctypes.data)
        return d, vals

    def apply_dirichlet(self, K, dofs, values, b):
        if self.L.ref_apply_dirichlet(K, _i32(dofs).size, _i32(dofs), _f64(values), b):
            self._err("apply_dirichlet")

    def pcg(self, K, b, rtol=1e-10, max_iter=20000, record_history=False):
        n = self.L.ref_csr_rows(K)
        x = np.zeros(n)
        hist = np.zeros(max_iter + 1) if record_history else None
        st = _RefStats()
        msg, warn = C.create_string_buffer(256), C.create_string_buffer(256)
        if self.L.ref_pcg(K, _f64(b), x, rtol, max_iter,
                          hist.ctypes.data if hist is not None else None, C.byref(st), msg, warn):
            self._err("pcg_jacobi")
        stats = dict(iterations=st.iterations, converged=bool(st.converged),
                     rel_residual=st.rel_residual, true_rel_residual=st.true_rel_residual,
                     message=msg.value.decode(), warning=warn.value.decode(),
                     t_setup=st.t_setup, t_solve=st.t_solve, t_spmv=st.t_spmv, t_dot=st.t_dot,
                     t_vec=st.t_vec)
        if hist is not None:
            stats["residual_history"] = hist[: st.iterations + 1]
        return x, stats

    def element_stresses(self, m, u, E, nu, plane_strain=False):
        nn, nt, fl = C.c_int(), C.c_int(), C.c_int()
        self.L.ref_mesh_info(m, C.byref(nn), C.byref(nt), C.byref(fl))
        out = np.zeros(8 * nt.value)
        if self.L.ref_element_stresses(m, _f64(u), E, nu, int(plane_strain), out):
            self._err("compute_element_stresses")
        names = ["sxx", "syy", "txy", "von_mises", "szz", "cx", "cy", "area"]
        return {k: out[i * nt.value:(i + 1) * nt.value].copy() for i, k in enumerate(names)}
