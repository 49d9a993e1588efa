"""B200 (sm_100a) CST assembly -> Dirichlet elimination -> Jacobi-PCG path.

A drop-in for the serial core of FreddyJuka/mpi-cst-fem-solver: the kernels live in
libcstfem_b200.so behind the C ABI of include/cstfem_b200.h; `solver` mirrors the reference's
C++ interface on top of it, `plate` generates the synthetic O-grid plates.

The directory name is not a Python identifier; import it with
``importlib.import_module("mpi-cst-fem-solver_b200")``.
"""
from . import batch, build, learned, mesh_io, native, plate  # noqa: F401
from .mesh_io import read_gmsh, write_gmsh  # noqa: F401
from .native import CstgError, LogicError  # noqa: F401
from .batch import BatchSolution, BatchSolver, PlateBatch, build_batch  # noqa: F401
from .solver import amg_apply, amg_set_smoother, amg_set_strength, amg_set_tail, amg_setup, amg_time  # noqa: F401
from .solver import (CgJacobiSolver, Context, DirichletDofs, GpuCsrMatrix,  # noqa: F401
                     PlaneCondition, SolverOptions, SolverStats, add_dirichlet_group,
                     add_kirsch_traction, add_stress_traction, add_traction, apply_dirichlet, assemble_stiffness, build_stiffness_pattern,
                     compute_element_stresses, constitutive_matrix, pcg_jacobi, scf_at_hole)

__version__ = "0.1.0"
