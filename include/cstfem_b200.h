/*
 * cstfem_b200.h -- C ABI of the B200 (sm_100a) CST assembly / Dirichlet / Jacobi-PCG path.
 *
 * Drop-in for the serial core of FreddyJuka/mpi-cst-fem-solver (cstfem_core). The call shapes
 * are the reference's: build_stiffness_pattern -> assemble_stiffness -> apply_dirichlet ->
 * CgJacobiSolver::setup / solve (pcg_jacobi), on the reference's row-owner CSR layout
 * (row_ptr int32[n+1], cols int32[nnz] sorted per row, vals double[nnz]; DOF 2*node+component;
 * one 2x2 block per pair of nodes sharing a triangle). Only plain pointers and sizes cross
 * the boundary.
 *
 * Conventions
 *  - Every call returns a status code (CSTG_OK = 0). Where the reference throws an exception
 *    the call returns the matching CSTG_ERR_* code and cstg_last_error() gives the message.
 *    Solver non-convergence is not an error (the reference reports it in SolverStats):
 *    cstg_pcg_solve returns CSTG_OK with stats.converged = 0 and stats.status set.
 *  - Functions without a suffix take HOST pointers and copy through pinned staging buffers;
 *    the *_device variants take device pointers on the context's device (no copies).
 *    Device vectors of doubles must be 16-byte aligned (cudaMalloc / torch allocations are);
 *    misaligned ones are rejected with CSTG_ERR_INVALID_ARGUMENT.
 *  - A context owns all the device memory it uses; buffers grow and are reused, so repeated
 *    calls of the same size allocate nothing. A context is used by one host thread at a
 *    time; work is ordered on the context's stream (cstg_set_stream).
 *  - The context keeps the mesh, the pattern and the matrix between calls, like the
 *    reference's Mesh / CsrMatrix objects live between the driver's phases.
 */
#ifndef CSTFEM_B200_H
#define CSTFEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define CSTG_OK 0
#define CSTG_ERR_INVALID_ARGUMENT 1   /* bad sizes / pointers / DOF out of range            */
#define CSTG_ERR_CUDA 2               /* a CUDA runtime call failed                           */
#define CSTG_ERR_NONPOSITIVE_DIAGONAL 3 /* solver.cpp:139-140, bc.cpp:151-153                  */
#define CSTG_ERR_PATTERN 4            /* entry missing from the pattern, assembly.cpp:67-69   */
#define CSTG_ERR_DIRICHLET_CONFLICT 5 /* same DOF with two values, bc.cpp:107-116             */
#define CSTG_ERR_STATE 6              /* call order (e.g. solve before setup, solver.cpp:151) */
#define CSTG_ERR_MESH 7               /* node index out of range, node neighbourhood too big  */
#define CSTG_ERR_TIMEOUT 8            /* a bounded device wait gave up                        */
#define CSTG_ERR_UNSUPPORTED 9        /* option not available for this matrix kind            */

/* stats.status values (how the iteration ended) */
#define CSTG_SOLVE_CONVERGED 0        /* recursive residual < rtol (solver.cpp:80-87)         */
#define CSTG_SOLVE_ZERO_RHS 1         /* ||b|| = 0, x = 0 (solver.cpp:44-49)                  */
#define CSTG_SOLVE_BREAKDOWN 2        /* p'Ap <= 0 (solver.cpp:65-71)                          */
#define CSTG_SOLVE_MAX_ITER 3         /* max_iter reached (solver.cpp:100-104)                */
#define CSTG_SOLVE_TIMEOUT 4          /* a device barrier gave up; result not usable          */

/* precision / method of cstg_pcg_solve */
#define CSTG_PRECISION_FP64 0         /* plain FP64 Jacobi-PCG, the reference's arithmetic     */
#define CSTG_PRECISION_MIXED 1        /* FP32 SpMV matrix (difference form) with FP64
                                         accumulation, FP64 vectors and scalars, FP64
                                         true-residual replacement (reliable updates); the
                                         solve stops on the FP64 true residual. Mesh pattern
                                         matrices only. */

typedef struct cstg_ctx cstg_ctx;

/* ≙ cstfem::SolverOptions (include/cstfem/solver.hpp:93-97) plus the B200 additions. */
typedef struct {
  double rtol;              /* default 1e-10                                               */
  int max_iter;             /* default 20000                                               */
  int record_history;       /* fill `history` (max_iter + 1 doubles) with ||r_k||/||b||     */
  int precision;            /* CSTG_PRECISION_*                                            */
  int true_residual_stop;   /* 1: converge only when the FP64 true residual ||b-Ax||/||b||
                               < rtol (residual replacement + restart when the recursive
                               residual converged first); 0: the reference's rule
                               (recursive residual, solver.cpp:80-82)                      */
  int max_refinements;      /* cap on replacements/restarts when true_residual_stop (16)   */
  int check_interval;       /* iterations per device graph between host checks (0: auto)  */
  int launch_mode;          /* CSTG_LAUNCH_*                                               */
  int preconditioner;       /* CSTG_PRECOND_*                                              */
  int fcg_depth;            /* flexible CG with a nonlinear (learned) preconditioner: each new
                               direction is A-orthogonalised against this many earlier ones
                               (1: the one-term flexible CG; at most 5); 0: automatic (3 for
                               the learned preconditioners, 1 otherwise)                     */
  int reserved[1];
} cstg_solver_options;

/* preconditioner of cstg_pcg_solve */
#define CSTG_PRECOND_JACOBI 0   /* Jacobi (the reference's CgJacobiSolver)                      */
#define CSTG_PRECOND_LEARNED 1  /* the learned network inside flexible CG, Jacobi as fallback;
                                   needs cstg_learned_setup after cstg_pcg_setup                */
#define CSTG_PRECOND_AMG 2      /* smoothed-aggregation multigrid V(2,2) cycle (no reference
                                   counterpart); hierarchy built on the first solve after
                                   cstg_pcg_setup (or by cstg_amg_setup)                         */
#define CSTG_PRECOND_LEARNED_MG 3 /* the learned network as the finest-level post-smoother of the
                                   multigrid cycle (global reach through the hierarchy), inside
                                   flexible CG with Jacobi-PCG as the stagnation fallback; needs
                                   cstg_learned_setup (with the smoother's weights) after
                                   cstg_pcg_setup                                                */

/* launch_mode of cstg_pcg_solve */
#define CSTG_LAUNCH_AUTO 0        /* persistent kernel for mesh-pattern matrices, else graph  */
#define CSTG_LAUNCH_PERSISTENT 1  /* one cooperative kernel runs all iterations (mesh pattern) */
#define CSTG_LAUNCH_GRAPH 2       /* 3-4 kernels per iteration, chunks replayed as CUDA graphs */
#define CSTG_LAUNCH_INSTRUMENTED 3 /* FP64 Jacobi-PCG with its kernels launched one by one and CUDA
                                      events between the phases (cstg_solve_breakdown); slower  */

/* ≙ cstfem::SolverStats (include/cstfem/solver.hpp:99-107) plus counters. */
typedef struct {
  int iterations;           /* CG iterations (all restarts together)                        */
  int converged;            /* 1 when the stopping rule was met                             */
  int status;               /* CSTG_SOLVE_*                                                 */
  int refinements;          /* FP64 residual replacements / restarts performed             */
  double rel_residual;      /* recursive ||r_k|| / ||b|| at exit                            */
  double true_rel_residual; /* ||b - A x|| / ||b|| recomputed in FP64 at exit               */
  double solve_seconds;     /* device time of the solve (CUDA events)                       */
  long long spmv_calls;     /* SpMV launches (iterations + true residuals)                  */
  char message[256];        /* SolverStats::message                                         */
  char warning[256];        /* SolverStats::warning (true residual > 10 rtol)               */
} cstg_stats;

/* ≙ cstfem::SolveBreakdown (include/cstfem/solver.hpp:17-56): device seconds of the phases of the
 * last solve run with launch_mode CSTG_LAUNCH_INSTRUMENTED (CUDA events between the phases of every
 * iteration). setup: the Jacobi diagonal (cstg_pcg_setup); spmv_local: q = A p with its fused p'Ap
 * partial sums, and A x of the true residual; dot_local: 0 (every dot product is fused into the
 * SpMV or vector kernels and counted there); vector_ops: the x, r, p updates with their fused dots
 * and b - A x; total: setup + the whole solve. The distributed fields of the reference (halo,
 * allreduce) have no counterpart on one device. */
typedef struct {
  double setup, spmv_local, dot_local, vector_ops, total;
  long long spmv_calls, reductions;
  int valid;
  int reserved[3];
} cstg_breakdown;

/* ---- batched solves: launch shape and per-system results -------------------------------- */
/* No reference counterpart. Launch shape of the batched persistent solve: each plate is solved
 * by one thread-block cluster of `cluster_ctas` CTAs (1, 2, 4, 8 or 16) of `threads` threads
 * (256 or 512). cluster_ctas == 0 means "not chosen" (the tuned or default shape is used). */
typedef struct {
  int cluster_ctas;
  int threads;
  int reserved[2];
} cstg_batch_config;

/* One per (system, load case), system-major: results[s * n_rhs + q]. */
typedef struct {
  int iterations;           /* CG iterations of this load case                          */
  int status;               /* CSTG_SOLVE_*                                             */
  int refinements;          /* FP64 residual replacements (reliable updates + checks)   */
  int fp64;                 /* 1 when the system finished on the FP64 operator          */
  double rel_residual;      /* recursive ||r|| / ||b|| at exit                          */
  double true_rel_residual; /* FP64 ||b - A x|| / ||b|| at exit                         */
} cstg_batch_result;

/* ---- context --------------------------------------------------------------------------- */
/* No reference counterpart (the reference keeps its state in caller objects). */
cstg_ctx* cstg_create(int device, int* status);
void cstg_destroy(cstg_ctx* ctx);
const char* cstg_last_error(const cstg_ctx* ctx);
int cstg_set_stream(cstg_ctx* ctx, void* cuda_stream); /* NULL: the context's own stream */
/* The stream the context's work is ordered on (its own or the one given to cstg_set_stream), so
 * a caller can order its own streams against it with events. Asynchronous entry points (the
 * *_device calls that only enqueue: cstg_multiply_device, cstg_multiply_mixed_device,
 * cstg_add_traction_device) return before their kernels have run; every other entry point
 * returns after its work on this stream has finished. No entry point waits for work the caller
 * issued on other streams: inputs written there must be finished (or the context's stream made
 * to wait for them) before the call. */
int cstg_get_stream(cstg_ctx* ctx, void** cuda_stream);
/* The phase times of the last instrumented solve (CSTG_LAUNCH_INSTRUMENTED) since cstg_pcg_setup. */
int cstg_solve_breakdown(cstg_ctx* ctx, cstg_breakdown* out);
void cstg_default_options(cstg_solver_options* opt);
int cstg_version(void);
/* The compute architecture of the library's kernels as the CUDA runtime reports it for `device`
 * (cudaFuncGetAttributes binaryVersion: 100 for sm_100a). */
int cstg_binary_version(int device, int* version);
/* Bounded device waits (no reference counterpart). Every device-side wait of the library gives
 * up after a number of polls and reports CSTG_ERR_TIMEOUT (stats->status CSTG_SOLVE_TIMEOUT where
 * a solve was running) with the context still usable: the persistent solve's grid barriers
 * (default 50,000,000 polls, about 2 s) and the learned network's tensor-core waits (default
 * 4,194,304 polls). 0 makes a wait give up at once (failure-detection tests); -1 restores the
 * default. A tensor-core wait that gives up still lets its matrix multiply finish (bounded)
 * before the kernel releases its memory. */
int cstg_set_wait_limits(cstg_ctx* ctx, long long barrier_polls, long long mma_polls);
/* Kernel launches issued by this library in this process so far (every kernel node of a
 * replayed CUDA graph counts). Benchmarks read it around a timed region. */
long long cstg_kernel_launches(void);

/* ---- mesh -------------------------------------------------------------------------------
 * ≙ cstfem::Mesh (include/cstfem/mesh.hpp:19-30): xy = 2 doubles per node, tri = 3 int32 per
 * triangle, counter-clockwise, 0-based (read_gmsh reorients, mesh_io.cpp:281-289).        */
int cstg_set_mesh(cstg_ctx* ctx, int n_nodes, const double* xy, int n_tri, const int32_t* tri);
int cstg_set_mesh_device(cstg_ctx* ctx, int n_nodes, const double* d_xy, int n_tri,
                         const int32_t* d_tri);

/* ---- build_stiffness_pattern (include/cstfem/assembly.hpp:15, src/assembly.cpp:9-42) -----
 * Builds the CSR pattern and the element slot map on the device. nnz_out may be NULL. */
int cstg_build_pattern(cstg_ctx* ctx, int64_t* nnz_out);

/* ---- assemble_stiffness (include/cstfem/assembly.hpp:22, src/assembly.cpp:54-74) ---------
 * Zeroes the values and adds every triangle's Ke = t |A| B^T D B (element.cpp:37-55),
 * bit-identical to the reference (same FP64 operations, same per-entry summation order).
 * D is the 3x3 row-major constitutive matrix (constitutive_matrix, element.cpp:7-15). */
int cstg_assemble(cstg_ctx* ctx, const double D[9], double thickness);
/* assemble_stiffness for a mesh made of several disjoint parts with different materials
 * (e.g. many plates concatenated for a batched solve): element e uses D[9 m .. 9 m + 8] and
 * thickness[m], m = material_of_element[e] (host arrays). Each part's entries are bit-identical
 * to assemble_stiffness (src/assembly.cpp:54-74) on that part alone. */
int cstg_assemble_materials(cstg_ctx* ctx, int n_materials, const double* D, const double* thickness,
                            const int32_t* material_of_element);

/* ---- CSR access ----------------------------------------------------------------------------
 * cstg_get_csr copies the current matrix (pattern + values) to host arrays sized by
 * cstg_matrix_size; any pointer may be NULL. cstg_set_csr replaces the matrix by a caller's
 * CSR (≙ passing any CsrMatrix to CgJacobiSolver::setup, solver.hpp:134); such a matrix has no
 * mesh pattern and uses the scalar-CSR SpMV. */
int cstg_matrix_size(cstg_ctx* ctx, int* n_rows, int64_t* nnz);
int cstg_get_csr(cstg_ctx* ctx, int32_t* row_ptr, int32_t* cols, double* vals);
int cstg_set_csr(cstg_ctx* ctx, int n_rows, const int32_t* row_ptr, const int32_t* cols,
                 const double* vals);

/* ---- apply_dirichlet (include/cstfem/bc.hpp:53, src/bc.cpp:137-166) -----------------------
 * dofs/values: prescribed DOFs (any order; a DOF repeated with the same value is allowed,
 * with different values -> CSTG_ERR_DIRICHLET_CONFLICT, DirichletDofs::add bc.cpp:107-116).
 * Symmetric elimination in place on the context's matrix and on b (n_rows doubles).    */
int cstg_apply_dirichlet(cstg_ctx* ctx, int n_fixed, const int32_t* dofs, const double* values,
                         double* b_inout);
int cstg_apply_dirichlet_device(cstg_ctx* ctx, int n_fixed, const int32_t* d_dofs,
                                const double* d_values, double* d_b_inout);
/* apply_dirichlet for n_rhs load vectors sharing K (b: n_rhs vectors of n_rows doubles, one
 * after another): each vector gets exactly what a separate apply_dirichlet (bc.cpp:137-166)
 * would give it; K is eliminated once. */
int cstg_apply_dirichlet_multi(cstg_ctx* ctx, int n_fixed, const int32_t* dofs, const double* values,
                               int n_rhs, double* b);
int cstg_apply_dirichlet_multi_device(cstg_ctx* ctx, int n_fixed, const int32_t* d_dofs,
                                      const double* d_values, int n_rhs, double* d_b);

/* ---- LinearOperator::apply / CsrMatrix::multiply (solver.hpp:60-64, csr.cpp:19-26) ------
 * cstg_multiply returns when y is on the host; cstg_multiply_device only enqueues the SpMV on
 * the context's stream (the caller orders / synchronises). */
int cstg_multiply(cstg_ctx* ctx, const double* x, double* y);
int cstg_multiply_device(cstg_ctx* ctx, const double* d_x, double* d_y);
/* The SpMV of the mixed-precision solver (no reference counterpart): y = K x with K's
 * off-diagonal 2x2 blocks stored in FP32 in difference form, (K x)_n = sum_{m != n} K_nm (x_m -
 * x_n) + S_n x_n, S_n the FP64 row-block sum; FP64 x and y, FP64 accumulation. Needs the mesh
 * pattern and cstg_pcg_setup; enqueued on the context's stream. */
int cstg_multiply_mixed_device(cstg_ctx* ctx, const double* d_x, double* d_y);

/* ---- CgJacobiSolver::setup (solver.hpp:134, solver.cpp:133-148) ----------------------------
 * inv_diag = 1 / K_ii; CSTG_ERR_NONPOSITIVE_DIAGONAL names the first such row. */
int cstg_pcg_setup(cstg_ctx* ctx);

/* ---- CgJacobiSolver::solve / pcg_jacobi (solver.hpp:115-118,135; solver.cpp:35-131) ------
 * Jacobi-PCG from x = 0 on the current matrix. opt NULL = defaults. history: NULL or
 * max_iter + 1 doubles (host for cstg_pcg_solve, device for the _device variant). */
int cstg_pcg_solve(cstg_ctx* ctx, const double* b, double* x, const cstg_solver_options* opt,
                   cstg_stats* stats, double* history);
int cstg_pcg_solve_device(cstg_ctx* ctx, const double* d_b, double* d_x,
                          const cstg_solver_options* opt, cstg_stats* stats, double* d_history);

/* ---- compute_element_stresses (postprocess.cpp:35-60, element.cpp:57-81) ------------------
 * u: 2 doubles per node. out: 8 arrays of n_tri doubles, in this order:
 * sxx, syy, txy, von_mises, szz, cx, cy, area. */
int cstg_element_stresses(cstg_ctx* ctx, const double* u, double E, double nu, int plane_strain,
                          double* out);

/* ---- add_traction (bc.hpp:74-75, bc.cpp:190-253) -----------------------------------------
 * Consistent nodal forces of a constant traction (tx, ty) on line edges (n_edges x 2 node
 * pairs), 2-point Gauss, times thickness, added to the host array f (2 per node). After
 * cstg_build_pattern the loads are computed on the GPU (the loaded nodes' entries of f copied up
 * and back, the pattern's node incidence: cstg_add_traction_device); before it, on the host from the mesh of cstg_set_mesh.
 * Bit-identical to the reference either way. Every edge is checked first: an edge not adjacent
 * to exactly one triangle returns CSTG_ERR_MESH with the reference's message (the triangle
 * count) and f is left as it was. */
int cstg_add_traction(cstg_ctx* ctx, int n_edges, const int32_t* edges, double thickness,
                      double tx, double ty, double* f);

/* add_traction on the GPU (src/bc.cpp:190-253; kind CSTG_TRACTION_KIRSCH: the traction of the
 * analytical Kirsch field, src/kirsch.cpp:40-45, with a = p0, sigma_inf = p1; CONSTANT: t = (p0,
 * p1)). Edges (2 x n_edges node indices) and f (n_rows doubles, accumulated into) are device
 * pointers; the node -> triangle incidence of cstg_build_pattern is used. A constant traction
 * gives loads bit-identical to the reference; the Kirsch traction agrees to rounding (GPU sin,
 * cos, atan2). An edge not adjacent to exactly one triangle leaves f untouched and returns
 * CSTG_ERR_MESH with the reference's message. */
#define CSTG_TRACTION_CONSTANT 0
#define CSTG_TRACTION_KIRSCH 1
/* the traction sigma . n of the uniform stress sigma = diag(p0, p1) (outward normal n of each
 * edge): the loads of the reference's Neumann patch tests, tests/test_patch.cpp:86-112 */
#define CSTG_TRACTION_STRESS 2
int cstg_add_traction_device(cstg_ctx* ctx, int n_edges, const int32_t* d_edges, double thickness, int kind,
                             double p0, double p1, double* d_f);

/* ---- Jacobi-PCG without allocating ----------------------------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device memory where they
 * solve: applications with a fixed device-memory budget whose pool allocator forbids foreign
 * cudaMalloc calls after start-up, plugin hosts calling from a callback where cudaMalloc /
 * cudaFree would synchronise the device and stall other work, real-time loops that must not
 * block in the driver's allocator. CgJacobiSolver setup + solve (FP64, the same kernels and
 * arithmetic as cstg_pcg_solve on a caller CSR) on the caller's device CSR (d_row_ptr[n+1],
 * d_cols, d_vals), right-hand side d_b and solution d_x, on the calling thread's current
 * device and `stream` (NULL: the legacy default stream); returns when the solve has ended.
 * Every work vector lives in one static device array of the library sized for at most
 * CSTG_STATIC_MAX_ROWS rows (2.06 MiB on every GPU that loads the library, held until the
 * process exits); larger systems are rejected with CSTG_ERR_INVALID_ARGUMENT. Every call looks
 * up the array's device address in the current device context (cudaGetSymbolAddress); the
 * first call on a device also loads the library's device code there, so make that first call
 * before any stream capture. All calls share the array and it keeps the last call's
 * contents (each call resets the state it needs): calls that overlap on a GPU race, so
 * serialise them. Needs precision CSTG_PRECISION_FP64 and record_history 0. Errors return a
 * status code with the text in stats->message. */
#define CSTG_STATIC_MAX_ROWS 65536
int cstg_pcg_solve_static(int n_rows, const int32_t* d_row_ptr, const int32_t* d_cols,
                          const double* d_vals, const double* d_b, double* d_x,
                          const cstg_solver_options* opt, cstg_stats* stats, void* stream);

/* ---- batched Jacobi-PCG ------------------------------------------------------------------
 * No counterpart in the reference (its driver solves one system per run, src/driver.cpp:164-188;
 * a batch is what a caller gets by running that path once per plate and load case). The
 * context's matrix must be block diagonal over the node ranges node_offsets[s] ..
 * node_offsets[s+1] (0 = node_offsets[0] <= ... <= node_offsets[n_systems] = node count; no
 * matrix entry couples two ranges, which is checked), set up with cstg_pcg_setup. All systems
 * and all n_rhs load vectors (b: n_rhs vectors of n_rows doubles, one after another; x the
 * same) are solved in one persistent launch: one thread-block cluster per system at a time,
 * largest systems first, load cases in groups of up to four sharing each matrix read.
 * opt->precision MIXED: FP32 difference-form SpMV with FP64 vectors and scalars; FP64: FP64
 * SpMV. Every load case stops on the FP64 true residual ||b - A x|| <= rtol ||b|| (reliable
 * updates replace the recursive residual by the FP64 one once per decade of reduction; a
 * system switches to the FP64 operator when the FP32 one stops improving the true residual).
 * max_iter and max_refinements apply per load case. `config` NULL: the shape from the last
 * cstg_batch_autotune on this context, else 8 CTAs x 512 threads. The launches are captured
 * once into a CUDA graph and replayed while the matrix, the vectors and the arguments are
 * unchanged. `seconds` (optional): device time of the solve. Results in `results`
 * (n_systems * n_rhs, system-major). */
int cstg_batch_solve(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs,
                     const double* b, double* x, const cstg_solver_options* opt,
                     const cstg_batch_config* config, cstg_batch_result* results, double* seconds);
int cstg_batch_solve_device(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs,
                            const double* d_b, double* d_x, const cstg_solver_options* opt,
                            const cstg_batch_config* config, cstg_batch_result* results,
                            double* seconds);
/* Times every feasible launch shape (cluster 1/2/4/8/16 CTAs x 256/512 threads) on this batch
 * (device vectors; the solve runs with `opt`, e.g. a reduced max_iter to bound the tuning
 * time), keeps the fastest for later cstg_batch_solve calls on this context and returns it. */
int cstg_batch_autotune(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs,
                        const double* d_b, double* d_x, const cstg_solver_options* opt,
                        cstg_batch_config* best, double* best_seconds);

/* ---- learned preconditioner -----------------------------------------------------------------
 * No counterpart in the reference. A message-passing network over the node graph of the
 * stiffness pattern (3 layers of width 64, BF16 weights with FP32 accumulation, the layers on
 * the tensor cores) maps a residual r to z = D^-1 (r + s Y(r / s)), s = RMS(r); with all weights
 * zero it is the Jacobi step. Parameters: cstg_mpnn_param_count() floats, packed as
 * W_in[64][8], b_in[64], (W_l[64][128], b_l[64]) for l = 1..3, W_out[2][64], b_out[2], every W
 * row-major [out][in]. Inputs per node: r / s (2), diagonal / its mean (2), coordinates / 10 (2)
 * and two material values (the caller's: log(D00) and D01/D00 of the node's constitutive matrix).
 * cstg_learned_setup: after cstg_pcg_setup (host arrays; node_material has 2 floats per node).
 * Then cstg_pcg_solve with opt->preconditioner = CSTG_PRECOND_LEARNED runs flexible CG
 * (Polak-Ribiere) with the network; Jacobi takes over when the network's direction is not a
 * descent direction (one step) or when ||r|| has not halved over 1000 iterations (for the rest
 * of the solve). Mesh-pattern matrices only. */
/* Training data: plain FP64 Jacobi-PCG (the reference's recurrence) on d_b, copying the iterate
 * x_k to d_X + j * n_rows after every `every` iterations (k = every, 2 every, ...), at most
 * max_snapshots of them; *n_snapshots receives the count. The solve itself ends as
 * cstg_pcg_solve_device does. */
int cstg_pcg_iterates_device(cstg_ctx* ctx, const double* d_b, int every, int max_snapshots, double* d_X,
                             int* n_snapshots, const cstg_solver_options* opt, cstg_stats* stats);
long long cstg_mpnn_param_count(void);
int cstg_learned_setup(cstg_ctx* ctx, const float* params, const float* node_material);
int cstg_learned_set_params(cstg_ctx* ctx, const float* params);
/* z = M(r) on device vectors (2 x node count doubles each). */
int cstg_learned_apply_device(cstg_ctx* ctx, const double* d_r, double* d_z);
/* Timing of the network's inference launches on the context's stream (CUDA events, `reps`
 * back-to-back launches of each after a warm-up): out[0] seconds per encoder launch, out[1 .. 3]
 * per launch of message-passing layer 1 .. 3 (the third with the decoder). */
int cstg_learned_time(cstg_ctx* ctx, int reps, double* out);

/* Training on the GPU with the library's forward and backward kernels. A sample is a residual
 * r and the error e = A^-1 r of the context's matrix (device, n_rows doubles each, samples one
 * after another); its loss is 1 - (z'r)^2 / ((z'Az)(e'r)), z = M(r). accumulate adds the
 * gradients of n_samples losses (the context must have cstg_learned_setup done; its weights are
 * not used, the trainer's are); step applies Adam (beta 0.9 / 0.999) with the accumulated
 * gradient times grad_scale and clears it. */
typedef struct cstg_trainer cstg_trainer;
cstg_trainer* cstg_trainer_create(int device, const float* params, int* status);
void cstg_trainer_destroy(cstg_trainer* tr);
const char* cstg_trainer_last_error(const cstg_trainer* tr);
int cstg_trainer_accumulate(cstg_trainer* tr, cstg_ctx* ctx, int n_samples, const double* d_R, const double* d_E,
                            double* losses);
int cstg_trainer_step(cstg_trainer* tr, float lr, float grad_scale);
/* The same for the network as the post-smoother of the learned multigrid cycle
 * (CSTG_PRECOND_LEARNED_MG): per sample, x_fix = pre-smoothing + coarse correction of r (fixed),
 * r2 = r - A x_fix, z = x_fix + omega D^-1 (r2 + s2 Y(r2 / s2)), s2 = RMS(r2), omega =
 * 4 / (3 lambda_max(D^-1 A)), and the loss 1 - (z'r)^2 / ((z'Az)(e'r)) of the whole cycle's
 * output; the gradient flows through the network's one application. Needs cstg_learned_setup
 * on the context (its multigrid hierarchy is built when missing). */
int cstg_trainer_accumulate_cycle(cstg_trainer* tr, cstg_ctx* ctx, int n_samples, const double* d_R,
                                  const double* d_E, double* losses);
/* The learned cycle's parts for one residual (device vectors of n_rows doubles; any output may be
 * NULL): x_fix (pre-smoothing + coarse correction), r2 = r - A x_fix (FP32 finest operator),
 * winvd = omega D^-1, and z = the whole cycle's output. For checks against the CPU oracle. */
int cstg_learned_cycle_parts_device(cstg_ctx* ctx, const double* d_r, double* d_xfix, double* d_r2,
                                    double* d_winvd, double* d_z);
int cstg_trainer_params(cstg_trainer* tr, float* params, float* grads);
int cstg_trainer_zero_grad(cstg_trainer* tr);

/* ---- Gmsh .msh 4.1 reader (host) --------------------------------------------------------------
 * ≙ read_gmsh (include/cstfem/mesh.hpp, src/mesh_io.cpp): ASCII 4.1 only; triangles turned
 * counter-clockwise (counted in `flipped`); line elements filed by physical-group name (groups in
 * name order). On error returns CSTG_ERR_MESH with "path:line: message" in err. No GPU needed. */
typedef struct cstg_mesh cstg_mesh;
int cstg_read_gmsh(const char* path, cstg_mesh** mesh, char* err, int err_len);
void cstg_mesh_destroy(cstg_mesh* mesh);
int cstg_mesh_info(const cstg_mesh* mesh, int* n_nodes, int* n_tri, int* n_groups, int* flipped);
/* xy: 2 per node, tri: 3 per triangle (0-based), node_tags: the file's tags (any may be NULL) */
int cstg_mesh_arrays(const cstg_mesh* mesh, double* xy, int32_t* tri, long long* node_tags);
/* group `index` (0 .. n_groups-1): its name and edges (2 node indices each; NULL to query) */
int cstg_mesh_group(const cstg_mesh* mesh, int index, char* name, int name_len, int* n_edges, int32_t* edges);

/* ---- multigrid preconditioner -------------------------------------------------------------------
 * No counterpart in the reference. Smoothed aggregation on the GPU: distance-2 MIS aggregates of
 * the node graph (on coarse levels, of its strong connections: cstg_amg_set_strength), tentative prolongator from the 2D rigid-body modes (per-aggregate QR), one
 * damped-Jacobi prolongator smoothing step, Galerkin coarse operators (3 x 3 blocks), dense
 * inverse of the coarsest level; the preconditioner is one V(2,2) cycle with Chebyshev smoothing
 * (or damped Jacobi, cstg_amg_set_smoother; lambda_max(D^-1 A) by power iteration). Deterministic. Used by
 * cstg_pcg_solve with opt->preconditioner = CSTG_PRECOND_AMG (flexible CG driver, FP64 true-
 * residual check as for the other preconditioners). Mesh-pattern matrices only. */
typedef struct {
  int levels;
  int dofs[16];
  long long nnz[16];
  double setup_seconds;
  int tail_level;    /* first level run by the one-cluster tail launch (0: none) */
  int tail_cluster;  /* CTAs in that cluster */
} cstg_amg_info;
int cstg_amg_setup(cstg_ctx* ctx, cstg_amg_info* info);
/* z = M r (device vectors) with the context's hierarchy (built if missing). */
int cstg_amg_apply_device(cstg_ctx* ctx, const double* d_r, double* d_z);
/* Timing on the context's stream (CUDA events, `reps` back-to-back launches after a warm-up):
 * out[0] = seconds per finest-level smoothing sweep, out[1] = seconds per V-cycle. */
int cstg_amg_time(cstg_ctx* ctx, int reps, double* out);
/* The small coarse levels and the coarsest solve run as one thread-block-cluster launch with
 * cluster barriers between phases (default), or as one launch per level and phase (enable = 0).
 * Both give the same bits. */
int cstg_amg_set_tail(cstg_ctx* ctx, int enable);
/* Smoother of the cycle: Chebyshev polynomial of degree 2 on [1.1 lambda / 20, 1.1 lambda] of
 * D^-1 A (default) or damped Jacobi with weight 4 / (3 lambda); two pre- and two post-smoothing
 * steps either way (the same number of operator applications). */
#define CSTG_AMG_CHEBYSHEV 0
#define CSTG_AMG_JACOBI 1
int cstg_amg_set_smoother(cstg_ctx* ctx, int kind);
/* Strength-of-connection thresholds of the aggregation, on the finest level and on the coarser
 * levels (each in [0, 1); default 0 and 0.03): block (i, j) joins the aggregation graph when
 * ||A_ij||_F >= theta sqrt(||A_ii||_F ||A_jj||_F). A change rebuilds the hierarchy on next use. */
int cstg_amg_set_strength(cstg_ctx* ctx, double theta_fine, double theta_coarse);

#ifdef __cplusplus
}
#endif
#endif /* CSTFEM_B200_H */
