// Jacobi-PCG on a caller's device CSR matrix without allocating any memory.
//
// Some callers cannot allocate device memory on the path that calls the solver: a host
// application that owns a fixed device-memory budget and forbids allocations after start-up
// (pool allocators that fail or fragment on foreign cudaMalloc calls), plugin hosts that run
// the solve from a callback where cudaMalloc / cudaFree would synchronise the whole device
// and stall other work, and real-time loops that must not block in the driver's allocator.
// For them, cstg_pcg_solve_static keeps every work vector of the solve (inverse diagonal,
// r, p, A p, the block partial sums and the solver state) in one file-scope static
// __device__ array whose size is fixed when the library is loaded; the caller passes only
// its matrix, right-hand side and solution.
//
// The array holds at most CSTG_STATIC_MAX_ROWS rows (65,536: 4 vectors of 512 KiB plus
// about 65 KiB of partial sums and state, 2.06 MiB in all). Every GPU that loads the library
// holds it until the process exits. All calls in the process share it, so two calls whose
// work overlaps on a GPU (other threads, other streams) race and corrupt each other's
// results; callers serialise them.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/cstfem_b200.h"
#include "common.cuh"
#include "kernels.h"

using namespace cstg;

namespace {

constexpr size_t kStateBytes = 256;                                // PcgState
constexpr size_t kErrBytes = 256;                                  // error word (int[8])
constexpr size_t kPartialBytes = sizeof(double) * 4 * kMaxGrid;  // 64 KiB
constexpr size_t kVecBytes = sizeof(double) * (size_t)CSTG_STATIC_MAX_ROWS;
constexpr size_t kScratchBytes = kStateBytes + kErrBytes + kPartialBytes + 4 * kVecBytes;
static_assert(sizeof(PcgState) <= kStateBytes, "state slot too small");
static_assert(kPartialBytes % 256 == 0, "partials must keep 256-byte alignment");

// The scratch of every cstg_pcg_solve_static call (see the file comment).
static __device__ __align__(256) double g_pcg_scratch[kScratchBytes / sizeof(double)];

// Device address of g_pcg_scratch in the current device's context. Looked up on every call:
// a cached address would go stale when the context is torn down and re-created
// (cudaDeviceReset), while the lookup itself is a host-side table read once the module is
// loaded (the first call on a device loads it, so that call comes before any stream capture).
cudaError_t scratch_address(char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<char*>(p);
  return cudaSuccess;
}

// Sets stats->message (the reference's exception text) and returns `code`.
int fail_msg(cstg_stats* stats, int code, const char* fmt, ...) {
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(stats->message, sizeof stats->message, fmt, ap);
    va_end(ap);
  }
  return code;
}

#define SCK(call)                                                                             \
  do {                                                                                        \
    const cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                                    \
      return fail_msg(stats, CSTG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));         \
  } while (0)

}  // namespace

extern "C" int cstg_pcg_solve_static(int n_rows, const int32_t* d_row_ptr, const int32_t* d_cols,
                                     const double* d_vals, const double* d_b, double* d_x,
                                     const cstg_solver_options* opt, cstg_stats* stats,
                                     void* stream) {
  cstg_solver_options o;
  if (opt)
    o = *opt;
  else
    cstg_default_options(&o);
  if (n_rows < 0 || n_rows > CSTG_STATIC_MAX_ROWS)
    return fail_msg(stats, CSTG_ERR_INVALID_ARGUMENT,
                    "pcg_solve_static: %d rows outside the static scratch (0 to %d rows)", n_rows,
                    CSTG_STATIC_MAX_ROWS);
  if (n_rows > 0 && (!d_row_ptr || !d_cols || !d_vals || !d_b || !d_x))
    return fail_msg(stats, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve_static: null array");
  if (((reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_x)) & 15u) != 0)
    return fail_msg(stats, CSTG_ERR_INVALID_ARGUMENT,
                    "pcg_solve_static: b and x must be 16-byte aligned device vectors");
  if (o.precision != CSTG_PRECISION_FP64 || o.record_history || !(o.rtol >= 0.0) || o.max_iter < 0 ||
      o.max_refinements < 0 || o.check_interval < 0)
    return fail_msg(stats, CSTG_ERR_UNSUPPORTED,
                    "pcg_solve_static: needs FP64 precision, no history and valid options");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = nullptr;
  SCK(scratch_address(&base));
  PcgState* st = reinterpret_cast<PcgState*>(base);
  int* err = reinterpret_cast<int*>(base + kStateBytes);
  double* partials = reinterpret_cast<double*>(base + kStateBytes + kErrBytes);
  double* vec = reinterpret_cast<double*>(base + kStateBytes + kErrBytes + kPartialBytes);
  double* inv_diag = vec;
  double* r = vec + CSTG_STATIC_MAX_ROWS;
  double* p = vec + 2 * (size_t)CSTG_STATIC_MAX_ROWS;
  double* Ap = vec + 3 * (size_t)CSTG_STATIC_MAX_ROWS;

  // State (tickets, done flag) and error word start from known values on every call.
  SCK(cudaMemsetAsync(st, 0, kStateBytes, s));
  SCK(cudaMemsetAsync(err, 0x7f, kErrBytes, s));
  int nnz = 0;
  if (n_rows) SCK(cudaMemcpyAsync(&nnz, d_row_ptr + n_rows, sizeof(int), cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));

  CsrMatrixDev A;
  A.n_rows = n_rows;
  A.row_ptr = d_row_ptr;
  A.cols = d_cols;
  A.vals = d_vals;
  const double avg = n_rows ? (double)nnz / n_rows : 1.0;
  int sub = 1;
  while (sub < 32 && sub < avg) sub <<= 1;
  A.sub = sub;

  // CgJacobiSolver::setup
  int h_err[kErrSlots];
  if (n_rows) SCK(launch_inv_diag(n_rows, d_row_ptr, d_cols, d_vals, inv_diag, err, s));
  SCK(cudaMemcpyAsync(h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, s));
  SCK(cudaStreamSynchronize(s));
  if (h_err[kErrDiag] != 0x7f7f7f7f)
    return fail_msg(stats, CSTG_ERR_NONPOSITIVE_DIAGONAL, "cg_jacobi: non-positive diagonal at row %d",
                    h_err[kErrDiag]);

  PcgBuffers w;
  w.n = n_rows;
  w.x = d_x;
  w.r = r;
  w.p = p;
  w.Ap = Ap;
  w.inv_diag = inv_diag;
  w.b = d_b;
  w.partials = partials;
  w.history = nullptr;
  w.st = st;
  w.err = err;

  const int chunk = o.check_interval > 0 ? o.check_interval : 50;
  const long long max_chunks = (long long)o.max_iter / chunk + 2 + (long long)o.max_refinements * 4;
  PcgState h;
  auto snap = [&]() -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  };
  const auto t0 = std::chrono::steady_clock::now();
  SCK(launch_pcg_init(w, o.rtol, o.max_iter, false, s));
  SCK(snap());
  long long chunks = 0, spmv_calls = 0;
  bool true_done = false;
  while (h.done != CSTG_SOLVE_ZERO_RHS + 1) {
    while (h.done == 0) {
      if (++chunks > max_chunks)
        return fail_msg(stats, CSTG_ERR_TIMEOUT, "pcg_solve_static: no end after %lld chunks", chunks);
      const int it0 = h.iter;
      for (int k = 0; k < chunk; ++k) SCK(launch_pcg_iteration(w, nullptr, &A, s));
      SCK(snap());
      spmv_calls += h.iter - it0 + (h.done == CSTG_SOLVE_BREAKDOWN + 1);
    }
    SCK(launch_spmv(nullptr, &A, w.x, w.Ap, s));
    ++spmv_calls;
    SCK(launch_true_residual(w, o.true_residual_stop != 0, o.max_refinements, s));
    SCK(snap());
    true_done = true;
    if (h.done != 0) break;
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->iterations = h.iter;
    stats->status = h.done - 1;
    stats->converged = (h.done == CSTG_SOLVE_CONVERGED + 1 || h.done == CSTG_SOLVE_ZERO_RHS + 1);
    stats->refinements = h.replace_count;
    stats->rel_residual = h.rel;
    stats->true_rel_residual = true_done ? h.true_rel : 0.0;
    stats->solve_seconds = secs;
    stats->spmv_calls = spmv_calls;
    char* m = stats->message;
    const size_t L = sizeof stats->message;
    switch (h.done - 1) {
      case CSTG_SOLVE_ZERO_RHS: std::snprintf(m, L, "zero right-hand side, x = 0"); break;
      case CSTG_SOLVE_CONVERGED:
        std::snprintf(m, L, "converged in %d iterations, relative residual %g", h.iter, h.rel);
        break;
      case CSTG_SOLVE_BREAKDOWN:
        std::snprintf(m, L, "CG breakdown at iteration %d: p'Ap = %g (matrix not SPD?)", h.iter + 1, h.pAp);
        break;
      default:
        std::snprintf(m, L, "NOT converged: reached max_iter = %d, relative residual %g (rtol %g)",
                      o.max_iter, h.rel, o.rtol);
        break;
    }
    if (stats->converged && h.done != CSTG_SOLVE_ZERO_RHS + 1 && stats->true_rel_residual > 10.0 * o.rtol)
      std::snprintf(stats->warning, sizeof stats->warning,
                    "WARNING: CG recursive residual converged (%g) but the true residual ||b - Ax|| / "
                    "||b|| = %g exceeds 10 * rtol = %g",
                    h.rel, stats->true_rel_residual, 10.0 * o.rtol);
  }
  return CSTG_OK;
}
