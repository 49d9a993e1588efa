// Host-side context of the C ABI and the helpers every C-ABI file shares (device buffers,
// error reporting with the reference's messages, error-word handling).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cstfem_b200.h"
#include "common.cuh"
#include "kernels.h"

using namespace cstg;

namespace cstg_host {

constexpr int kErrNone = 0x7f7f7f7f;  // memset(0x7f) sentinel of the device error word
// Mixed precision: a reliable update replaces the FP32 recursive residual by the FP64 one when
// it has dropped by this factor since the last update (~one replacement per decade).
constexpr double kReliableDelta = 0.1;
// Iterations per batch of the instrumented solve (events between every phase, read per batch).
constexpr int kBdChunk = 50;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace cstg_host

using cstg_host::DevBuf;
struct AmgData;  // amg_api.cu: the multigrid hierarchy of a context

struct cstg_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  unsigned long long generation = 0;  // bumped whenever a device buffer moves

  // pinned host staging: error word + state snapshot
  int* h_err = nullptr;
  PcgState* h_state = nullptr;

  // mesh
  int n_nodes = 0, n_tri = 0;
  bool has_mesh = false, host_mesh = false;
  std::vector<double> h_xy;
  std::vector<int32_t> h_tri;
  std::vector<int> h_ne_ptr, h_ne;  // host incidence for add_traction (built lazily)
  DevBuf xy, tri;

  // incidence + pattern
  DevBuf cnt, cursor, ne_ptr, ne, scan_tmp, deg, node_ptr, bnbr, slot;
  DevBuf row_ptr, cols, vals;
  int kind = 0;  // 0 none, 1 mesh block pattern, 2 caller CSR
  int n_rows = 0;
  long long nnz = 0;
  int csr_sub = 8;
  bool has_values = false, setup_done = false;

  // Dirichlet
  DevBuf fixed, ubar, dofs, dvals;

  // solver
  DevBuf b_in, x, r, p, Ap, inv_diag, partials, state, err_word, hist, vec_in, vec_out, stress;
  // mixed precision: FP32 difference-form operator and FP32 work vectors
  DevBuf val32, nbr32, S32;
  bool mixed_ready = false;
  cudaGraphExec_t graph = nullptr;
  unsigned long long graph_gen = ~0ull;
  int graph_chunk = 0, graph_hist = -1, graph_kind = -1, graph_n = -1, graph_prec = -1, graph_refs = -1;
  const double* graph_b = nullptr;

  // GPU traction: per-edge contributions and per-node records
  DevBuf tr_con, tr_cnt, tr_ptr, tr_cur, tr_rec;
  DevBuf tr_edges, tr_f;  // host-pointer traction calls routed through the device path

  // multi-material assembly
  DevBuf mat, mat_tab;

  // batched solves: plate table, LPT order, interleaved load-case vectors, per-system results
  DevBuf bat_sys, bat_order, bat_queue, bat_b, bat_x, bat_r, bat_p, bat_Ap, bat_stats, bat_in, bat_out;
  std::vector<int32_t> bat_offsets;  // host copy of the last validated plate table
  unsigned long long bat_checked_gen = ~0ull;
  cstg_batch_config bat_cfg{};       // tuned launch shape (cluster_ctas == 0: not tuned)
  cudaGraphExec_t bat_graph = nullptr;
  unsigned long long bat_graph_key = 0;
  long long bat_graph_launches = 0;  // kernel nodes per replay of bat_graph

  // learned preconditioner: packed weights (FP32 master, BF16 + FP32 copies), per-node static
  // inputs, inference activations, network scalars, z; the flexible-CG chunk graph
  unsigned long long setup_count = 0;  // bumped by every cstg_pcg_setup
  DevBuf lp_p32, lp_pb, lp_pf, lp_sf, lp_h0, lp_h1, lp_sc, lp_z, lp_mat;
  bool learned_ready = false;
  unsigned long long learned_setup = ~0ull;  // setup_count the static inputs were built for
  cudaGraphExec_t fcg_graph = nullptr;
  unsigned long long fcg_key = 0;
  long long fcg_graph_launches = 0;
  int fcg_graph_precond = -1;

  // smoothed-aggregation multigrid hierarchy (built on demand)
  AmgData* amg = nullptr;

  // learned multigrid cycle: the post-smoother's weights omega D^-1 (omega = 4 / (3 lambda_max)),
  // built for the hierarchy of setup `lm_winvd_for`
  DevBuf lm_winvd;
  unsigned long long lm_winvd_for = ~0ull;
  // the network layers' gather plan for the node pattern of `lp_plan_for` (the pattern count)
  DevBuf lp_plan_hdr, lp_plan_runs, lp_plan_local;
  unsigned long long pattern_count = 0;  // bumped by every cstg_build_pattern
  unsigned long long lp_plan_for = ~0ull;
  bool lp_plan_on = true;  // CSTG_MP_GATHER=rows turns the plan off (every tile gathers row by row)
  bool lp_plan_use = false;  // the plan covers at least a quarter of the tiles
  // truncated flexible CG: ring of earlier directions and their A-products, ring state
  DevBuf fcg_ph[kFcgMaxHist], fcg_qh[kFcgMaxHist], fcg_ring;

  // the last instrumented solve's phase times (CSTG_LAUNCH_INSTRUMENTED) and its event pool
  cstg_breakdown bd{};
  std::vector<cudaEvent_t> bd_ev;

  // bounded device waits (polls before a wait gives up; cstg_set_wait_limits)
  long long barrier_spin = kBarrierSpinDefault;
  long long mbar_spin = kMpMbarSpinDefault;
};

namespace cstg_host {

inline int fail(cstg_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    const cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                                 \
      return fail(ctx, CSTG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));            \
  } while (0)

template <class T>
inline T* buf_ptr(DevBuf& b) {
  return static_cast<T*>(b.p);
}

// Grow-only device buffer. Returns 0 or an error code.
inline int ensure(cstg_ctx* ctx, DevBuf& b, size_t bytes) {
  bytes = std::max<size_t>(bytes, 256);
  if (b.bytes >= bytes) return CSTG_OK;
  if (b.p) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
  }
  CK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  ctx->generation++;
  return CSTG_OK;
}

#define ENSURE(buf, bytes)                          \
  do {                                              \
    const int rc_ = ensure(ctx, (buf), (bytes));    \
    if (rc_) return rc_;                            \
  } while (0)

inline void free_buf(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

inline int begin(cstg_ctx* ctx) {
  if (!ctx) return CSTG_ERR_INVALID_ARGUMENT;
  ctx->err.clear();
  CK(cudaSetDevice(ctx->device));
  return CSTG_OK;
}

#define BEGIN(ctx)                 \
  do {                             \
    const int rb_ = begin(ctx);    \
    if (rb_) return rb_;           \
  } while (0)

inline int reset_err(cstg_ctx* ctx) {
  CK(cudaMemsetAsync(ctx->err_word.p, 0x7f, sizeof(int) * kErrSlots, ctx->stream));
  return CSTG_OK;
}

// Copies the error word to the host and waits for the stream.
inline int read_err(cstg_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->h_err, ctx->err_word.p, sizeof(int) * kErrSlots, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

#define RESET_ERR()                     \
  do {                                  \
    const int r_ = reset_err(ctx);      \
    if (r_) return r_;                  \
  } while (0)
#define READ_ERR()                      \
  do {                                  \
    const int r_ = read_err(ctx);       \
    if (r_) return r_;                  \
  } while (0)

// constitutive_matrix (element.cpp:7-15), host side, same operations.
inline void constitutive(double E, double nu, int plane_strain, double D[9]) {
  if (!plane_strain) {
    const double c = E / (1.0 - nu * nu);
    const double v[9] = {c, c * nu, 0.0, c * nu, c, 0.0, 0.0, 0.0, c * (1.0 - nu) / 2.0};
    std::memcpy(D, v, sizeof v);
  } else {
    const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double v[9] = {c * (1.0 - nu), c * nu, 0.0, c * nu, c * (1.0 - nu), 0.0,
                         0.0, 0.0, c * (1.0 - 2.0 * nu) / 2.0};
    std::memcpy(D, v, sizeof v);
  }
}

inline BlockMatrix block_view(cstg_ctx* ctx) {
  BlockMatrix m;
  m.n_nodes = ctx->n_nodes;
  m.node_ptr = buf_ptr<int>(ctx->node_ptr);
  m.bnbr = buf_ptr<int>(ctx->bnbr);
  m.vals = buf_ptr<double>(ctx->vals);
  return m;
}

inline CsrMatrixDev csr_view(cstg_ctx* ctx) {
  CsrMatrixDev m;
  m.n_rows = ctx->n_rows;
  m.row_ptr = buf_ptr<int>(ctx->row_ptr);
  m.cols = buf_ptr<int>(ctx->cols);
  m.vals = buf_ptr<double>(ctx->vals);
  m.sub = ctx->csr_sub;
  return m;
}

inline int spmv(cstg_ctx* ctx, const double* x, double* y) {
  if (ctx->kind == 1) {
    const BlockMatrix bm = block_view(ctx);
    CK(launch_spmv(&bm, nullptr, x, y, ctx->stream));
  } else {
    const CsrMatrixDev cm = csr_view(ctx);
    CK(launch_spmv(nullptr, &cm, x, y, ctx->stream));
  }
  return CSTG_OK;
}

// The vector kernels load 16-byte pairs; caller device vectors must allow that.
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

inline void g_fmt(char* out, size_t n, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(out, n, fmt, ap);
  va_end(ap);
}

// Defined in amg_api.cu: the multigrid hierarchy (built when missing or stale) and z = M r.
int amg_ready(cstg_ctx* ctx);
// skip: see amg_sweep_f32; dots (may be null): take the flexible-CG scalars in the cycle's last
// sweep (only with two or more levels: a one-level hierarchy is the dense solve alone)
int amg_apply(cstg_ctx* ctx, const double* r, double* z, const int* skip, const FcgDotSink* dots = nullptr);
void amg_free(cstg_ctx* ctx);
int amg_levels(const cstg_ctx* ctx);
int amg_chebyshev(const cstg_ctx* ctx);  // 1: Chebyshev smoothing, 0: damped Jacobi
unsigned long long amg_signature(const cstg_ctx* ctx);  // level shapes of the current hierarchy
// The learned cycle's pieces (the hierarchy must be ready): x = pre-smoothing + coarse correction
// of b (no post-smoothing); out = b - A x with the finest level's FP32 operator; the finest
// level's residual scratch (free outside a cycle); lambda_max(D^-1 A) of the finest level (device).
int amg_apply_pre(cstg_ctx* ctx, const double* b, double* x, const int* skip);
int amg_residual_fine(cstg_ctx* ctx, const double* b, const double* x, double* out, const int* skip);
double* amg_fine_scratch(cstg_ctx* ctx);
const double* amg_fine_lambda(cstg_ctx* ctx);
unsigned long long amg_built_for(const cstg_ctx* ctx);  // setup_count of the hierarchy (~0: none)

// Defined in learned_api.cu: flexible CG with the learned preconditioner.
int run_fcg(cstg_ctx* ctx, const double* d_b, double* d_x, const cstg_solver_options& o, cstg_stats* stats);

// Defined in api.cu: the FP32 difference-form operator of the current matrix.
int ensure_mixed(cstg_ctx* ctx);
MixedMatrix mixed_view(cstg_ctx* ctx);

}  // namespace cstg_host

using namespace cstg_host;
