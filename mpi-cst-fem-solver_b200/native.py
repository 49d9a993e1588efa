"""ctypes binding of the C ABI (include/cstfem_b200.h).

The library is the in-tree libcstfem_b200.so built by build.py. There is no fallback: if the
library is missing or a CUDA device is absent, the calls fail with an error.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

# status codes (cstfem_b200.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_NONPOSITIVE_DIAGONAL = 3
ERR_PATTERN = 4
ERR_DIRICHLET_CONFLICT = 5
ERR_STATE = 6
ERR_MESH = 7
ERR_TIMEOUT = 8
ERR_UNSUPPORTED = 9

SOLVE_CONVERGED = 0
SOLVE_ZERO_RHS = 1
SOLVE_BREAKDOWN = 2
SOLVE_MAX_ITER = 3
SOLVE_TIMEOUT = 4

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class CstgError(RuntimeError):
    """A call of the C ABI failed (the reference throws std::runtime_error there)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class LogicError(CstgError):
    """Call-order / pattern errors (the reference throws std::logic_error there)."""


class SolverOptions(C.Structure):
    _fields_ = [("rtol", C.c_double), ("max_iter", C.c_int), ("record_history", C.c_int),
                ("precision", C.c_int), ("true_residual_stop", C.c_int),
                ("max_refinements", C.c_int), ("check_interval", C.c_int),
                ("launch_mode", C.c_int), ("preconditioner", C.c_int), ("fcg_depth", C.c_int),
                ("reserved", C.c_int * 1)]


TRACTION_CONSTANT = 0
TRACTION_KIRSCH = 1
TRACTION_STRESS = 2

PRECOND_JACOBI = 0
PRECOND_LEARNED = 1
PRECOND_AMG = 2
PRECOND_LEARNED_MG = 3
AMG_CHEBYSHEV, AMG_JACOBI = 0, 1  # cstg_amg_set_smoother

LAUNCH_AUTO = 0
LAUNCH_PERSISTENT = 1
LAUNCH_GRAPH = 2
LAUNCH_INSTRUMENTED = 3


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
                ("refinements", C.c_int), ("rel_residual", C.c_double),
                ("true_rel_residual", C.c_double), ("solve_seconds", C.c_double),
                ("spmv_calls", C.c_longlong), ("message", C.c_char * 256),
                ("warning", C.c_char * 256)]


class Breakdown(C.Structure):
    """cstg_breakdown: the reference's SolveBreakdown fields of an instrumented solve."""
    _fields_ = [("setup", C.c_double), ("spmv_local", C.c_double), ("dot_local", C.c_double),
                ("vector_ops", C.c_double), ("total", C.c_double), ("spmv_calls", C.c_longlong),
                ("reductions", C.c_longlong), ("valid", C.c_int), ("reserved", C.c_int * 3)]


class AmgInfo(C.Structure):
    """cstg_amg_info: the multigrid hierarchy."""
    _fields_ = [("levels", C.c_int), ("dofs", C.c_int * 16), ("nnz", C.c_longlong * 16),
                ("setup_seconds", C.c_double), ("tail_level", C.c_int), ("tail_cluster", C.c_int)]


class BatchConfig(C.Structure):
    """cstg_batch_config: CTAs per cluster (one cluster per plate) and threads per CTA."""
    _fields_ = [("cluster_ctas", C.c_int), ("threads", C.c_int), ("reserved", C.c_int * 2)]


class BatchResult(C.Structure):
    """cstg_batch_result: one per (system, load case)."""
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("refinements", C.c_int),
                ("fp64", C.c_int), ("rel_residual", C.c_double), ("true_rel_residual", C.c_double)]


_vp = C.c_void_p
_SIGS = {
    "cstg_version": (C.c_int, []),
    "cstg_kernel_launches": (C.c_longlong, []),
    "cstg_create": (_vp, [C.c_int, C.POINTER(C.c_int)]),
    "cstg_destroy": (None, [_vp]),
    "cstg_last_error": (C.c_char_p, [_vp]),
    "cstg_set_stream": (C.c_int, [_vp, _vp]),
    "cstg_get_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "cstg_binary_version": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "cstg_solve_breakdown": (C.c_int, [_vp, C.POINTER(Breakdown)]),
    "cstg_default_options": (None, [C.POINTER(SolverOptions)]),
    "cstg_set_mesh": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp]),
    "cstg_set_mesh_device": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp]),
    "cstg_build_pattern": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "cstg_assemble": (C.c_int, [_vp, _vp, C.c_double]),
    "cstg_matrix_size": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "cstg_get_csr": (C.c_int, [_vp, _vp, _vp, _vp]),
    "cstg_set_csr": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "cstg_apply_dirichlet": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "cstg_apply_dirichlet_device": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "cstg_multiply": (C.c_int, [_vp, _vp, _vp]),
    "cstg_multiply_device": (C.c_int, [_vp, _vp, _vp]),
    "cstg_multiply_mixed_device": (C.c_int, [_vp, _vp, _vp]),
    "cstg_pcg_setup": (C.c_int, [_vp]),
    "cstg_pcg_solve": (C.c_int, [_vp, _vp, _vp, C.POINTER(SolverOptions), C.POINTER(Stats), _vp]),
    "cstg_pcg_solve_device": (C.c_int, [_vp, _vp, _vp, C.POINTER(SolverOptions), C.POINTER(Stats),
                                        _vp]),
    "cstg_element_stresses": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_int, _vp]),
    "cstg_add_traction": (C.c_int, [_vp, C.c_int, _vp, C.c_double, C.c_double, C.c_double, _vp]),
    "cstg_add_traction_device": (C.c_int, [_vp, C.c_int, _vp, C.c_double, C.c_int, C.c_double, C.c_double, _vp]),
    "cstg_pcg_solve_static": (C.c_int, [C.c_int, _vp, _vp, _vp, _vp, _vp, C.POINTER(SolverOptions),
                                        C.POINTER(Stats), _vp]),
    "cstg_assemble_materials": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "cstg_apply_dirichlet_multi": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, _vp]),
    "cstg_apply_dirichlet_multi_device": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, _vp]),
    "cstg_batch_solve": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.POINTER(SolverOptions),
                                   C.POINTER(BatchConfig), _vp, C.POINTER(C.c_double)]),
    "cstg_batch_solve_device": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.POINTER(SolverOptions),
                                          C.POINTER(BatchConfig), _vp, C.POINTER(C.c_double)]),
    "cstg_batch_autotune": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.POINTER(SolverOptions),
                                      C.POINTER(BatchConfig), C.POINTER(C.c_double)]),
    "cstg_pcg_iterates_device": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp, C.POINTER(C.c_int),
                                           C.POINTER(SolverOptions), C.POINTER(Stats)]),
    "cstg_read_gmsh": (C.c_int, [C.c_char_p, C.POINTER(_vp), C.c_char_p, C.c_int]),
    "cstg_mesh_destroy": (None, [_vp]),
    "cstg_mesh_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]),
    "cstg_mesh_arrays": (C.c_int, [_vp, _vp, _vp, _vp]),
    "cstg_mesh_group": (C.c_int, [_vp, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_int), _vp]),
    "cstg_amg_setup": (C.c_int, [_vp, C.POINTER(AmgInfo)]),
    "cstg_amg_apply_device": (C.c_int, [_vp, _vp, _vp]),
    "cstg_amg_time": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double)]),
    "cstg_amg_set_tail": (C.c_int, [_vp, C.c_int]),
    "cstg_amg_set_smoother": (C.c_int, [_vp, C.c_int]),
    "cstg_amg_set_strength": (C.c_int, [_vp, C.c_double, C.c_double]),
    "cstg_mpnn_param_count": (C.c_longlong, []),
    "cstg_learned_setup": (C.c_int, [_vp, _vp, _vp]),
    "cstg_learned_set_params": (C.c_int, [_vp, _vp]),
    "cstg_learned_apply_device": (C.c_int, [_vp, _vp, _vp]),
    "cstg_trainer_create": (_vp, [C.c_int, _vp, C.POINTER(C.c_int)]),
    "cstg_trainer_destroy": (None, [_vp]),
    "cstg_trainer_last_error": (C.c_char_p, [_vp]),
    "cstg_trainer_accumulate": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp, _vp]),
    "cstg_trainer_accumulate_cycle": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp, _vp]),
    "cstg_learned_cycle_parts_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "cstg_set_wait_limits": (C.c_int, [_vp, C.c_longlong, C.c_longlong]),
    "cstg_learned_time": (C.c_int, [_vp, C.c_int, _vp]),
    "cstg_trainer_step": (C.c_int, [_vp, C.c_float, C.c_float]),
    "cstg_trainer_params": (C.c_int, [_vp, _vp, _vp]),
    "cstg_trainer_zero_grad": (C.c_int, [_vp]),
}

STATIC_MAX_ROWS = 65536  # CSTG_STATIC_MAX_ROWS

_lock = threading.Lock()
_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True) -> C.CDLL:
    """Loads libcstfem_b200.so (building it first when missing and nvcc is available)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(_build.LIB):
            if not build_if_missing:
                raise CstgError(ERR_STATE, f"{_build.LIB} is missing (run build.py)")
            _build.build_library()
        L = C.CDLL(_build.LIB)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        return L


def check(L, ctx, rc: int, what: str = ""):
    if rc == OK:
        return
    msg = L.cstg_last_error(ctx).decode() if ctx else ""
    cls = LogicError if rc in (ERR_STATE, ERR_PATTERN) else CstgError
    raise cls(rc, msg or f"{what}: status {rc}")


def default_options() -> SolverOptions:
    o = SolverOptions()
    load().cstg_default_options(C.byref(o))
    return o
