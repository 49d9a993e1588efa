// C ABI of the learned preconditioner: network set-up on a context (weights, per-node static
// inputs), z = M(r), the flexible-CG solve (cstg_pcg_solve with CSTG_PRECOND_LEARNED), and the
// trainer that fits the network on the GPU with the project's forward and backward kernels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ctx.h"

namespace {

// Depth of the truncated flexible CG with a learned preconditioner (each new direction is
// A-orthogonalised against this many earlier ones): the network's output varies nonlinearly with
// r, and the one-term recurrence then loses the conjugacy that a linear preconditioner keeps.
constexpr int kFcgDepthLearned = 3;
// Stagnation rule of the flexible CG: the network is switched off when ||r|| has not halved
// over this many iterations.
constexpr int kFcgWindow = 1000;
constexpr double kFcgRatio2 = 0.25;
constexpr double kCoordScale = 10.0;

MpnnParams params_view(cstg_ctx* ctx) {
  MpnnParams P;
  P.pb = buf_ptr<__nv_bfloat16>(ctx->lp_pb);
  P.pf = buf_ptr<float>(ctx->lp_pf);
  return P;
}

// The layers' gather plan for the current node pattern (built once per pattern): per tile of 128
// nodes the runs of consecutive rows its nodes read, and per node the slots of its own and its
// neighbours' rows in that union.
int plan_ready(cstg_ctx* ctx) {
  if (!ctx->lp_plan_on || ctx->lp_plan_for == ctx->pattern_count) return CSTG_OK;
  const int N = ctx->n_nodes;
  const int tiles = std::max((N + kMpTile - 1) / kMpTile, 1);
  ENSURE(ctx->lp_plan_hdr, sizeof(int4) * (size_t)tiles);
  ENSURE(ctx->lp_plan_runs, sizeof(int2) * (size_t)tiles * kPlanMaxRuns);
  ENSURE(ctx->lp_plan_local, sizeof(uint4) * (size_t)std::max(N, 1));
  int planned = 0;
  if (N) {
    CK(launch_mp_tile_plan(N, buf_ptr<int>(ctx->node_ptr), buf_ptr<int>(ctx->bnbr), buf_ptr<int4>(ctx->lp_plan_hdr),
                           buf_ptr<int2>(ctx->lp_plan_runs), buf_ptr<uint4>(ctx->lp_plan_local), ctx->stream));
    std::vector<int4> hdr((size_t)tiles);
    CK(cudaMemcpyAsync(hdr.data(), ctx->lp_plan_hdr.p, sizeof(int4) * hdr.size(), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (const int4& h : hdr) planned += h.z == 0 ? 1 : 0;
  }
  // the plan kernel (2 CTAs per SM, bulk-copied unions) pays off when a good share of the tiles
  // is planned; patterns numbered without locality (most tiles rejected) keep the row kernel
  ctx->lp_plan_use = 4 * planned >= tiles;
  ctx->lp_plan_for = ctx->pattern_count;
  return CSTG_OK;
}

MpnnGraph graph_view(cstg_ctx* ctx) {
  MpnnGraph g;
  g.n_nodes = ctx->n_nodes;
  g.node_ptr = buf_ptr<int>(ctx->node_ptr);
  g.nbr = buf_ptr<int>(ctx->bnbr);
  if (ctx->lp_plan_on && ctx->lp_plan_use && ctx->lp_plan_for == ctx->pattern_count) {
    g.plan.hdr = buf_ptr<int4>(ctx->lp_plan_hdr);
    g.plan.runs = buf_ptr<int2>(ctx->lp_plan_runs);
    g.plan.local = buf_ptr<uint4>(ctx->lp_plan_local);
  }
  return g;
}

MpnnWork infer_work(cstg_ctx* ctx) {
  MpnnWork w;
  w.H[0] = buf_ptr<__nv_bfloat16>(ctx->lp_h0);
  w.H[1] = buf_ptr<__nv_bfloat16>(ctx->lp_h1);
  return w;
}

int upload_params(cstg_ctx* ctx, const float* params) {
  ENSURE(ctx->lp_p32, sizeof(float) * kMpParams);
  ENSURE(ctx->lp_pb, sizeof(__nv_bfloat16) * kMpParams);
  ENSURE(ctx->lp_pf, sizeof(float) * kMpParams);
  CK(cudaMemcpyAsync(ctx->lp_p32.p, params, sizeof(float) * kMpParams, cudaMemcpyHostToDevice, ctx->stream));
  CK(launch_mp_params(buf_ptr<float>(ctx->lp_p32), buf_ptr<__nv_bfloat16>(ctx->lp_pb), buf_ptr<float>(ctx->lp_pf),
                      ctx->stream));
  return CSTG_OK;
}

// The learned cycle's post-smoother weights omega D^-1 (omega = 4 / (3 lambda_max(D^-1 A))) for the
// current hierarchy, which is built when missing.
int cycle_ready(cstg_ctx* ctx) {
  const int rc = amg_ready(ctx);
  if (rc) return rc;
  if (ctx->lm_winvd_for == amg_built_for(ctx)) return CSTG_OK;
  const int n = ctx->n_rows;
  ENSURE(ctx->lm_winvd, sizeof(double) * (size_t)std::max(n, 1));
  CK(launch_mp_smoother_weights(n, buf_ptr<double>(ctx->inv_diag), amg_fine_lambda(ctx), 4.0 / 3.0,
                                buf_ptr<double>(ctx->lm_winvd), ctx->stream));
  ctx->lm_winvd_for = amg_built_for(ctx);
  return CSTG_OK;
}

// z = learned cycle of r on stream s (the context's): z = x_fix (pre-smoothing + coarse
// correction), r2 = r - A z in the finest level's scratch, z += omega D^-1 (r2 + s2 Y(r2 / s2)).
// train: the network keeps its activations in mw (the trainer's buffers).
int cycle_apply(cstg_ctx* ctx, const MpnnGraph& g, const MpnnParams& P, MpnnWork& mw, MpScratch* msc,
                const double* winvd, const double* r, double* z, const int* skip, bool train, cudaStream_t s) {
  int rc = amg_apply_pre(ctx, r, z, skip);
  if (rc) return rc;
  double* r2 = amg_fine_scratch(ctx);
  rc = amg_residual_fine(ctx, r, z, r2, skip);
  if (rc) return rc;
  CK(launch_mp_rr(ctx->n_rows, r2, msc, s, skip));
  CK(launch_mp_forward(g, P, r2, winvd, &msc->rr, buf_ptr<float>(ctx->lp_sf), skip, mw, train, z, z, ctx->mbar_spin,
                       buf_ptr<int>(ctx->err_word), s));
  return CSTG_OK;
}

}  // namespace

// ---- flexible CG ------------------------------------------------------------------------------

int cstg_host::run_fcg(cstg_ctx* ctx, const double* d_b, double* d_x, const cstg_solver_options& o,
                       cstg_stats* stats) {
  const int n = ctx->n_rows, N = ctx->n_nodes;
  // the learned cycle: multigrid pre-smoothing and coarse correction, the network as the
  // finest level's post-smoother
  const bool cycle_net = o.preconditioner == CSTG_PRECOND_LEARNED_MG;
  const bool use_amg = o.preconditioner == CSTG_PRECOND_AMG || cycle_net;
  const bool use_net = o.preconditioner == CSTG_PRECOND_LEARNED || cycle_net;
  if (use_amg) {
    const int rc = amg_ready(ctx);  // the multigrid hierarchy of this matrix (built once per setup)
    if (rc) return rc;
  }
  if (cycle_net) {
    const int rc = cycle_ready(ctx);
    if (rc) return rc;
  }
  ENSURE(ctx->x, sizeof(double) * (size_t)n);
  ENSURE(ctx->r, sizeof(double) * (size_t)n);
  ENSURE(ctx->p, sizeof(double) * (size_t)n);
  ENSURE(ctx->Ap, sizeof(double) * (size_t)n);
  ENSURE(ctx->lp_z, sizeof(double) * (size_t)n);
  if (use_net) {
    ENSURE(ctx->lp_h0, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
    ENSURE(ctx->lp_h1, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  }
  const bool mixed = o.precision == CSTG_PRECISION_MIXED;
  if (mixed) {
    const int rc = ensure_mixed(ctx);
    if (rc) return rc;
  }
  FcgBuffers w;
  w.n = n;
  w.x = buf_ptr<double>(ctx->x);
  w.r = buf_ptr<double>(ctx->r);
  w.p = buf_ptr<double>(ctx->p);
  w.q = buf_ptr<double>(ctx->Ap);
  w.z = buf_ptr<double>(ctx->lp_z);
  w.b = d_b;
  w.inv_diag = buf_ptr<double>(ctx->inv_diag);
  w.partials = buf_ptr<double>(ctx->partials);
  w.st = buf_ptr<PcgState>(ctx->state);
  const BlockMatrix bm = block_view(ctx);
  const auto set_ring = [&](int h) {
    w.hist = h;
    for (int j = 0; j < h; ++j) {
      w.ph[j] = buf_ptr<double>(ctx->fcg_ph[j]);
      w.qh[j] = buf_ptr<double>(ctx->fcg_qh[j]);
    }
    w.ring = h > 0 ? buf_ptr<FcgRing>(ctx->fcg_ring) : nullptr;
  };
  const MixedMatrix mm = mixed ? mixed_view(ctx) : MixedMatrix{};
  const MpnnGraph g = graph_view(ctx);
  const MpnnParams P = params_view(ctx);
  MpnnWork mw = infer_work(ctx);
  int* err = buf_ptr<int>(ctx->err_word);
  const float* sf = buf_ptr<float>(ctx->lp_sf);
  const int* skip = &w.st->mp_skip;
  const double* rr = &w.st->rr;

  // With the multigrid cycle the scalars z'r, z'q and beta are taken inside the cycle's last
  // finest-level sweep (no separate dots pass), and there is no stagnation fallback (the cycle is
  // a fixed symmetric positive operator).
  const bool fused_dots = o.preconditioner == CSTG_PRECOND_AMG && amg_levels(ctx) > 1;
  // truncated flexible CG for the nonlinear (learned) preconditioners: the ring of earlier directions
  const int depth = o.fcg_depth > 0 ? o.fcg_depth : (use_net ? kFcgDepthLearned : 1);
  const int hist = fused_dots ? 0 : std::min(depth - 1, kFcgMaxHist);
  if (hist > 0) {
    for (int j = 0; j < hist; ++j) {
      ENSURE(ctx->fcg_ph[j], sizeof(double) * (size_t)std::max(n, 1));
      ENSURE(ctx->fcg_qh[j], sizeof(double) * (size_t)std::max(n, 1));
    }
    ENSURE(ctx->fcg_ring, sizeof(FcgRing));
  }
  set_ring(hist);
  MpScratch* msc = buf_ptr<MpScratch>(ctx->lp_sc);
  const double* winvd = cycle_net ? buf_ptr<double>(ctx->lm_winvd) : nullptr;
  FcgDotSink sink;
  sink.q = w.q;
  sink.partials = w.partials;
  sink.st = w.st;
  auto precondition = [&]() -> int {
    if (cycle_net) {
      const int rc = cycle_apply(ctx, g, P, mw, msc, winvd, w.r, w.z, skip, false, ctx->stream);
      if (rc) return rc;
    } else if (use_amg) {
      const int rc = amg_apply(ctx, w.r, w.z, &w.st->done, fused_dots ? &sink : nullptr);  // (cycles after
      if (rc) return rc;                                                                   // convergence return at once)
    } else {
      CK(launch_mp_forward(g, P, w.r, w.inv_diag, rr, sf, skip, mw, false, nullptr, w.z, ctx->mbar_spin, err,
                           ctx->stream));
    }
    if (fused_dots)
      CK(launch_fcg_pupdate(w, ctx->stream));
    else if (w.hist > 0)
      CK(launch_fcg_dots_ring(w, ctx->stream));
    else
      CK(launch_fcg_dots(w, ctx->stream));
    return CSTG_OK;
  };
  auto iteration = [&]() -> int {
    if (mixed)
      CK(launch_spmv_mixed_pcg(mm, bm, w.p, w.q, w.partials, w.st, ctx->stream));
    else
      CK(launch_spmv_pcg(bm, w.p, w.q, w.partials, w.st, ctx->stream));
    CK(launch_fcg_update(w, o.preconditioner == CSTG_PRECOND_AMG ? 0 : kFcgWindow, kFcgRatio2, ctx->stream,
                         mixed ? kReliableDelta : 0.0));
    // mixed precision: the FP32 operator's rounding accumulates in the recursive residual, which
    // is replaced by the FP64 b - A x once per decade of reduction (no restart)
    if (mixed) CK(launch_fcg_reliable(w, bm, ctx->stream));
    return precondition();
  };
  const int chunk = o.check_interval > 0 ? o.check_interval : 25;
  // the captured chunk depends on the buffers (generation), the shapes and the method
  unsigned long long key = 1469598103934665603ull;
  for (unsigned long long v : {ctx->generation, (unsigned long long)chunk, (unsigned long long)o.precision,
                               (unsigned long long)(uintptr_t)d_b, (unsigned long long)n,
                               (unsigned long long)ctx->n_nodes, use_amg ? amg_signature(ctx) : 0ull,
                               (unsigned long long)hist})
    key = (key ^ v) * 1099511628211ull;
  if (!ctx->fcg_graph || ctx->fcg_key != key || ctx->fcg_graph_precond != o.preconditioner) {
    if (ctx->fcg_graph) {
      cudaGraphExecDestroy(ctx->fcg_graph);
      ctx->fcg_graph = nullptr;
    }
    const long long l0 = launches_total();
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = CSTG_OK;
    for (int k = 0; k < chunk && rc == CSTG_OK; ++k) rc = iteration();
    const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &gr);
    const long long captured = launches_total() - l0;
    count_launches(-captured);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    CK(ee);
    const cudaError_t ie = cudaGraphInstantiate(&ctx->fcg_graph, gr, 0);
    cudaGraphDestroy(gr);
    CK(ie);
    ctx->fcg_key = key;
    ctx->fcg_graph_launches = captured;
    ctx->fcg_graph_precond = o.preconditioner;
  }

  RESET_ERR();
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (n) CK(cudaMemsetAsync(w.q, 0, sizeof(double) * (size_t)n, ctx->stream));
  if (hist > 0) CK(cudaMemsetAsync(w.ring, 0, sizeof(FcgRing), ctx->stream));  // an empty ring
  int zero = 0;
  CK(cudaMemcpyAsync(&w.st->fp64_mode, &zero, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CK(launch_fcg_init(w, o.rtol, o.max_iter, kFcgWindow, ctx->stream));
  {
    const int rc = precondition();
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(ctx->h_state, ctx->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  PcgBuffers pw;  // the true-residual kernel's view
  pw.n = n;
  pw.x = w.x;
  pw.r = w.r;
  pw.p = w.p;
  pw.Ap = w.q;
  pw.inv_diag = w.inv_diag;
  pw.b = d_b;
  pw.partials = w.partials;
  pw.st = w.st;
  long long chunks = 0, spmv_calls = 0;
  const long long max_chunks = (long long)o.max_iter / chunk + 4 + 4LL * o.max_refinements;
  bool true_done = false, switched = false;
  int fallback_iter = -1;
  while (ctx->h_state->done != CSTG_SOLVE_ZERO_RHS + 1) {
    while (ctx->h_state->done == 0) {
      if (++chunks > max_chunks)
        return fail(ctx, CSTG_ERR_TIMEOUT, "pcg_solve: the device state did not finish after %lld chunks",
                    chunks);
      const int it0 = ctx->h_state->iter;
      CK(cudaGraphLaunch(ctx->fcg_graph, ctx->stream));
      count_launches(ctx->fcg_graph_launches);
      CK(cudaMemcpyAsync(ctx->h_state, ctx->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      spmv_calls += ctx->h_state->iter - it0;
      if (fallback_iter < 0 && ctx->h_state->fallback) fallback_iter = ctx->h_state->fb_it0;
    }
    // FP64 true residual; a miss re-opens the solve from the replaced residual (Jacobi step)
    CK(launch_spmv(&bm, nullptr, w.x, w.q, ctx->stream));
    ++spmv_calls;
    CK(launch_true_residual(pw, o.true_residual_stop != 0, o.max_refinements, ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_state, ctx->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    true_done = true;
    if (ctx->h_state->done != 0) break;
    if (mixed && !switched) {  // the FP32 operator's accuracy floor: FP64 SpMV from here
      const int one = 1;
      CK(cudaMemcpyAsync(&w.st->fp64_mode, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
      switched = true;
    }
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  if (n) CK(cudaMemcpyAsync(d_x, w.x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
  const PcgState s = *ctx->h_state;
  READ_ERR();
  if (ctx->h_err[kErrTimeout] != kErrNone)
    return fail(ctx, CSTG_ERR_TIMEOUT, "pcg_solve: a tensor-core wait of the learned preconditioner timed out");
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->iterations = s.iter;
    stats->status = s.done - 1;
    stats->converged = (s.done == CSTG_SOLVE_CONVERGED + 1 || s.done == CSTG_SOLVE_ZERO_RHS + 1);
    stats->refinements = s.replace_count;
    stats->rel_residual = s.rel;
    stats->true_rel_residual = true_done ? s.true_rel : 0.0;
    stats->solve_seconds = ms * 1e-3;
    stats->spmv_calls = spmv_calls;
    char pre[160];
    if (cycle_net && fallback_iter >= 0)
      g_fmt(pre, sizeof pre, "learned multigrid cycle, switched to Jacobi at iteration %d (stagnation)",
            fallback_iter);
    else if (cycle_net)
      g_fmt(pre, sizeof pre, "learned multigrid cycle: %s pre-smoothing, network post-smoothing, %d levels",
            amg_chebyshev(ctx) ? "Chebyshev" : "damped-Jacobi", amg_levels(ctx));
    else if (use_amg)
      g_fmt(pre, sizeof pre, "smoothed-aggregation multigrid V(2,2), %s smoothing, %d levels",
            amg_chebyshev(ctx) ? "Chebyshev" : "damped-Jacobi", amg_levels(ctx));
    else if (fallback_iter >= 0)
      g_fmt(pre, sizeof pre, "learned preconditioner, switched to Jacobi at iteration %d (stagnation)",
            fallback_iter);
    else
      g_fmt(pre, sizeof pre, "learned preconditioner throughout");
    switch (s.done - 1) {
      case CSTG_SOLVE_ZERO_RHS:
        g_fmt(stats->message, sizeof stats->message, "zero right-hand side, x = 0");
        break;
      case CSTG_SOLVE_CONVERGED:
        g_fmt(stats->message, sizeof stats->message,
              "converged in %d iterations, relative residual %g (flexible CG, %s; %d FP64 residual "
              "replacements%s)",
              s.iter, s.rel, pre, s.replace_count, switched ? "; FP64 SpMV after the first" : "");
        break;
      case CSTG_SOLVE_BREAKDOWN:
        g_fmt(stats->message, sizeof stats->message, "CG breakdown at iteration %d: p'Ap = %g (matrix not SPD?)",
              s.iter + 1, s.pAp);
        break;
      default:
        g_fmt(stats->message, sizeof stats->message,
              "NOT converged: reached max_iter = %d, relative residual %g (rtol %g; %s)", o.max_iter, s.rel,
              o.rtol, pre);
        break;
    }
    if (stats->converged && s.done != CSTG_SOLVE_ZERO_RHS + 1 && stats->true_rel_residual > 10.0 * o.rtol)
      g_fmt(stats->warning, sizeof stats->warning,
            "WARNING: CG recursive residual converged (%g) but the true residual ||b - Ax|| / ||b|| = %g "
            "exceeds 10 * rtol = %g",
            s.rel, stats->true_rel_residual, 10.0 * o.rtol);
  }
  return CSTG_OK;
}

// ---- trainer ----------------------------------------------------------------------------------

struct cstg_trainer {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  DevBuf p32, m, v, grad, pb, pf, sc, az, z;
  DevBuf H[kMpL + 1], G[kMpL], A[kMpL], X, Y, dY, dH, dH2, dU, dAs, part;
  int step = 0;
  int cap_nodes = 0;
};

namespace {

int tfail(cstg_trainer* t, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (t) t->err = buf;
  return code;
}

#define TK(call)                                                                          \
  do {                                                                                    \
    const cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return tfail(tr, CSTG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int tensure(cstg_trainer* tr, DevBuf& b, size_t bytes) {
  bytes = std::max<size_t>(bytes, 256);
  if (b.bytes >= bytes) return CSTG_OK;
  if (b.p) {
    TK(cudaStreamSynchronize(tr->stream));
    TK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
  }
  TK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  return CSTG_OK;
}

#define TENSURE(buf, bytes)                        \
  do {                                             \
    const int rc_ = tensure(tr, (buf), (bytes));   \
    if (rc_) return rc_;                           \
  } while (0)

int trainer_work(cstg_trainer* tr, int N, MpnnWork& w) {
  const size_t nf = (size_t)N * kMpF;
  for (int l = 0; l <= kMpL; ++l) TENSURE(tr->H[l], sizeof(__nv_bfloat16) * nf);
  for (int l = 0; l < kMpL; ++l) {
    TENSURE(tr->G[l], sizeof(__nv_bfloat16) * nf);
    TENSURE(tr->A[l], sizeof(__nv_bfloat16) * nf);
  }
  TENSURE(tr->X, sizeof(__nv_bfloat16) * (size_t)N * kMpIn);
  TENSURE(tr->Y, sizeof(float) * 2 * (size_t)N);
  TENSURE(tr->dY, sizeof(float) * 2 * (size_t)N);
  TENSURE(tr->dH, sizeof(float) * nf);
  TENSURE(tr->dH2, sizeof(float) * nf);
  TENSURE(tr->dU, sizeof(float) * nf);
  TENSURE(tr->dAs, sizeof(float) * nf);
  TENSURE(tr->part, sizeof(float) * (size_t)kMpPartBlocks * kMpPartStride);
  TENSURE(tr->az, sizeof(double) * 2 * (size_t)N);
  TENSURE(tr->z, sizeof(double) * 2 * (size_t)N);
  for (int l = 0; l <= kMpL; ++l) w.H[l] = static_cast<__nv_bfloat16*>(tr->H[l].p);
  for (int l = 0; l < kMpL; ++l) {
    w.G[l] = static_cast<__nv_bfloat16*>(tr->G[l].p);
    w.A[l] = static_cast<__nv_bfloat16*>(tr->A[l].p);
  }
  w.X = static_cast<__nv_bfloat16*>(tr->X.p);
  w.Y = static_cast<float*>(tr->Y.p);
  w.dY = static_cast<float*>(tr->dY.p);
  w.dH = static_cast<float*>(tr->dH.p);
  w.dH2 = static_cast<float*>(tr->dH2.p);
  w.dU = static_cast<float*>(tr->dU.p);
  w.dAs = static_cast<float*>(tr->dAs.p);
  w.part = static_cast<float*>(tr->part.p);
  return CSTG_OK;
}

}  // namespace

extern "C" {

int cstg_learned_setup(cstg_ctx* ctx, const float* params, const float* node_material) {
  BEGIN(ctx);
  if (!params || (ctx->n_nodes > 0 && !node_material))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_setup: null parameters or material");
  if (ctx->kind != 1 || !ctx->setup_done)
    return fail(ctx, CSTG_ERR_STATE, "learned_setup: needs a mesh-pattern matrix after cstg_pcg_setup");
  CK(mpnn_prepare_device());
  const int N = ctx->n_nodes;
  int rc = upload_params(ctx, params);
  if (rc) return rc;
  // per-node static inputs on the GPU: diagonal / its mean, coordinates / plate size, material
  ENSURE(ctx->lp_sf, sizeof(float) * (size_t)std::max(N, 1) * 6 + 16);  // + the encoder's copy rounding
  ENSURE(ctx->lp_mat, sizeof(float) * (size_t)std::max(N, 1) * 2);
  ENSURE(ctx->lp_sc, sizeof(MpScratch));
  // the reductions' tickets must start at zero (a fresh allocation may hold old contents)
  CK(cudaMemsetAsync(ctx->lp_sc.p, 0, sizeof(MpScratch), ctx->stream));
  rc = plan_ready(ctx);
  if (rc) return rc;
  if (N) {
    CK(cudaMemcpyAsync(ctx->lp_mat.p, node_material, sizeof(float) * 2 * (size_t)N, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(launch_mp_static(N, buf_ptr<double>(ctx->inv_diag), buf_ptr<double>(ctx->xy), buf_ptr<float>(ctx->lp_mat),
                        kCoordScale, buf_ptr<MpScratch>(ctx->lp_sc), buf_ptr<float>(ctx->lp_sf), ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->learned_ready = true;
  ctx->learned_setup = ctx->setup_count;
  return CSTG_OK;
}

int cstg_learned_set_params(cstg_ctx* ctx, const float* params) {
  BEGIN(ctx);
  if (!params) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_set_params: null parameters");
  if (!ctx->learned_ready) return fail(ctx, CSTG_ERR_STATE, "learned_set_params: call cstg_learned_setup first");
  const int rc = upload_params(ctx, params);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

int cstg_learned_apply_device(cstg_ctx* ctx, const double* d_r, double* d_z) {
  BEGIN(ctx);
  if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
    return fail(ctx, CSTG_ERR_STATE, "learned_apply: call cstg_learned_setup after cstg_pcg_setup");
  if (ctx->n_rows && (!d_r || !d_z)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_apply: null vector");
  if (!aligned16(d_r) || !aligned16(d_z))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_apply: device vectors must be 16-byte aligned");
  const int N = ctx->n_nodes;
  ENSURE(ctx->lp_h0, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  ENSURE(ctx->lp_h1, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  MpScratch* sc = buf_ptr<MpScratch>(ctx->lp_sc);
  MpnnWork mw = infer_work(ctx);
  RESET_ERR();
  CK(launch_mp_rr(ctx->n_rows, d_r, sc, ctx->stream));
  CK(launch_mp_forward(graph_view(ctx), params_view(ctx), d_r, buf_ptr<double>(ctx->inv_diag), &sc->rr,
                       buf_ptr<float>(ctx->lp_sf), nullptr, mw, false, nullptr, d_z, ctx->mbar_spin,
                       buf_ptr<int>(ctx->err_word), ctx->stream));
  READ_ERR();
  if (ctx->h_err[kErrTimeout] != kErrNone)
    return fail(ctx, CSTG_ERR_TIMEOUT, "learned_apply: a tensor-core wait timed out");
  return CSTG_OK;
}

long long cstg_mpnn_param_count(void) { return kMpParams; }

cstg_trainer* cstg_trainer_create(int device, const float* params, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  if (!params) {
    set(CSTG_ERR_INVALID_ARGUMENT);
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    set(CSTG_ERR_CUDA);
    return nullptr;
  }
  cstg_trainer* tr = new cstg_trainer();
  tr->device = device;
  int rc = CSTG_OK;
  if (cudaStreamCreateWithFlags(&tr->stream, cudaStreamNonBlocking) != cudaSuccess) rc = CSTG_ERR_CUDA;
  if (!rc) rc = tensure(tr, tr->p32, sizeof(float) * kMpParams);
  if (!rc) rc = tensure(tr, tr->m, sizeof(float) * kMpParams);
  if (!rc) rc = tensure(tr, tr->v, sizeof(float) * kMpParams);
  if (!rc) rc = tensure(tr, tr->grad, sizeof(float) * kMpParams);
  if (!rc) rc = tensure(tr, tr->pb, sizeof(__nv_bfloat16) * kMpParams);
  if (!rc) rc = tensure(tr, tr->pf, sizeof(float) * kMpParams);
  if (!rc) rc = tensure(tr, tr->sc, sizeof(MpScratch));
  if (!rc && mpnn_prepare_device() != cudaSuccess) rc = CSTG_ERR_CUDA;
  if (!rc && (cudaMemcpyAsync(tr->p32.p, params, sizeof(float) * kMpParams, cudaMemcpyHostToDevice, tr->stream) ||
              cudaMemsetAsync(tr->m.p, 0, sizeof(float) * kMpParams, tr->stream) ||
              cudaMemsetAsync(tr->v.p, 0, sizeof(float) * kMpParams, tr->stream) ||
              cudaMemsetAsync(tr->grad.p, 0, sizeof(float) * kMpParams, tr->stream) ||
              cudaMemsetAsync(tr->sc.p, 0, sizeof(MpScratch), tr->stream) ||
              launch_mp_params(static_cast<float*>(tr->p32.p), static_cast<__nv_bfloat16*>(tr->pb.p),
                               static_cast<float*>(tr->pf.p), tr->stream) ||
              cudaStreamSynchronize(tr->stream)))
    rc = CSTG_ERR_CUDA;
  if (rc) {
    cstg_trainer_destroy(tr);
    set(rc);
    return nullptr;
  }
  set(CSTG_OK);
  return tr;
}

void cstg_trainer_destroy(cstg_trainer* tr) {
  if (!tr) return;
  cudaSetDevice(tr->device);
  if (tr->stream) cudaStreamSynchronize(tr->stream);
  DevBuf* all[] = {&tr->p32, &tr->m, &tr->v, &tr->grad, &tr->pb, &tr->pf, &tr->sc, &tr->az, &tr->z,
                   &tr->X,   &tr->Y, &tr->dY, &tr->dH,  &tr->dH2, &tr->dU, &tr->dAs, &tr->part};
  for (DevBuf* b : all) free_buf(*b);
  for (auto& b : tr->H) free_buf(b);
  for (auto& b : tr->G) free_buf(b);
  for (auto& b : tr->A) free_buf(b);
  if (tr->stream) cudaStreamDestroy(tr->stream);
  delete tr;
}

const char* cstg_trainer_last_error(const cstg_trainer* tr) { return tr ? tr->err.c_str() : "null trainer"; }

int cstg_trainer_accumulate(cstg_trainer* tr, cstg_ctx* ctx, int n_samples, const double* d_R, const double* d_E,
                            double* losses) {
  if (!tr) return CSTG_ERR_INVALID_ARGUMENT;
  tr->err.clear();
  TK(cudaSetDevice(tr->device));
  if (!ctx || ctx->device != tr->device)
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: the context must be on the trainer's device");
  if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
    return tfail(tr, CSTG_ERR_STATE, "trainer_accumulate: call cstg_learned_setup on the context first");
  if (n_samples < 0 || (n_samples > 0 && (!d_R || !d_E)))
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: bad samples");
  if (!aligned16(d_R) || !aligned16(d_E))
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: samples must be 16-byte aligned");
  const int N = ctx->n_nodes, n = ctx->n_rows;
  MpnnWork w;
  int rc = trainer_work(tr, N, w);
  if (rc) return rc;
  TK(cudaStreamSynchronize(ctx->stream));  // the context's matrix and inputs are ready
  const MpnnGraph g = graph_view(ctx);
  MpnnParams P;
  P.pb = static_cast<const __nv_bfloat16*>(tr->pb.p);
  P.pf = static_cast<const float*>(tr->pf.p);
  MpScratch* sc = static_cast<MpScratch*>(tr->sc.p);
  const BlockMatrix bm = block_view(ctx);
  const double* invd = buf_ptr<double>(ctx->inv_diag);
  double* z = static_cast<double*>(tr->z.p);
  double* az = static_cast<double*>(tr->az.p);
  float* grad = static_cast<float*>(tr->grad.p);
  int* err = buf_ptr<int>(ctx->err_word);
  TK(cudaMemsetAsync(err, 0x7f, sizeof(int) * kErrSlots, tr->stream));
  for (int i = 0; i < n_samples; ++i) {
    const double* r = d_R + (size_t)i * n;
    const double* e = d_E + (size_t)i * n;
    TK(launch_mp_rr(n, r, sc, tr->stream));
    TK(launch_mp_forward(g, P, r, invd, &sc->rr, buf_ptr<float>(ctx->lp_sf), nullptr, w, true, nullptr, z,
                         ctx->mbar_spin, err, tr->stream));
    TK(launch_spmv(&bm, nullptr, z, az, tr->stream));
    TK(launch_mp_loss(N, z, az, r, e, invd, sc, w, tr->stream));
    if (losses) TK(cudaMemcpyAsync(&losses[i], &sc->loss, sizeof(double), cudaMemcpyDeviceToHost, tr->stream));
    TK(launch_mp_backward(g, P, w, grad, ctx->mbar_spin, err, tr->stream));
  }
  int h_err[kErrSlots];
  TK(cudaMemcpyAsync(h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, tr->stream));
  TK(cudaStreamSynchronize(tr->stream));
  if (h_err[kErrTimeout] != kErrNone) return tfail(tr, CSTG_ERR_TIMEOUT, "trainer: a tensor-core wait timed out");
  return CSTG_OK;
}

int cstg_trainer_step(cstg_trainer* tr, float lr, float grad_scale) {
  if (!tr) return CSTG_ERR_INVALID_ARGUMENT;
  tr->err.clear();
  TK(cudaSetDevice(tr->device));
  if (!(lr > 0.f) || !(grad_scale > 0.f)) return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_step: bad lr/scale");
  tr->step += 1;
  TK(launch_mp_adam(static_cast<float*>(tr->p32.p), static_cast<float*>(tr->m.p), static_cast<float*>(tr->v.p),
                    static_cast<const float*>(tr->grad.p), lr, 0.9f, 0.999f, 1e-8f, tr->step, grad_scale,
                    static_cast<__nv_bfloat16*>(tr->pb.p), static_cast<float*>(tr->pf.p), tr->stream));
  TK(cudaMemsetAsync(tr->grad.p, 0, sizeof(float) * kMpParams, tr->stream));
  TK(cudaStreamSynchronize(tr->stream));
  return CSTG_OK;
}

int cstg_trainer_params(cstg_trainer* tr, float* params, float* grads) {
  if (!tr) return CSTG_ERR_INVALID_ARGUMENT;
  tr->err.clear();
  TK(cudaSetDevice(tr->device));
  if (params)
    TK(cudaMemcpyAsync(params, tr->p32.p, sizeof(float) * kMpParams, cudaMemcpyDeviceToHost, tr->stream));
  if (grads) TK(cudaMemcpyAsync(grads, tr->grad.p, sizeof(float) * kMpParams, cudaMemcpyDeviceToHost, tr->stream));
  TK(cudaStreamSynchronize(tr->stream));
  return CSTG_OK;
}

int cstg_trainer_zero_grad(cstg_trainer* tr) {
  if (!tr) return CSTG_ERR_INVALID_ARGUMENT;
  tr->err.clear();
  TK(cudaSetDevice(tr->device));
  TK(cudaMemsetAsync(tr->grad.p, 0, sizeof(float) * kMpParams, tr->stream));
  TK(cudaStreamSynchronize(tr->stream));
  return CSTG_OK;
}

}  // extern "C"

// ---- the learned multigrid cycle: training and parts ------------------------------------------

extern "C" {

int cstg_set_wait_limits(cstg_ctx* ctx, long long barrier_polls, long long mma_polls) {
  BEGIN(ctx);
  if (barrier_polls < -1 || mma_polls < -1)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_wait_limits: limits must be >= 0 (or -1 for the default)");
  ctx->barrier_spin = barrier_polls < 0 ? kBarrierSpinDefault : barrier_polls;
  ctx->mbar_spin = mma_polls < 0 ? kMpMbarSpinDefault : mma_polls;
  return CSTG_OK;
}

int cstg_learned_cycle_parts_device(cstg_ctx* ctx, const double* d_r, double* d_xfix, double* d_r2, double* d_winvd,
                                    double* d_z) {
  BEGIN(ctx);
  if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
    return fail(ctx, CSTG_ERR_STATE, "learned_cycle_parts: call cstg_learned_setup after cstg_pcg_setup");
  if (ctx->n_rows && !d_r) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_cycle_parts: null residual");
  if (!aligned16(d_r) || !aligned16(d_xfix) || !aligned16(d_r2) || !aligned16(d_winvd) || !aligned16(d_z))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_cycle_parts: device vectors must be 16-byte aligned");
  int rc = cycle_ready(ctx);
  if (rc) return rc;
  const int n = ctx->n_rows, N = ctx->n_nodes;
  const size_t bytes = sizeof(double) * (size_t)n;
  ENSURE(ctx->lp_z, bytes);
  ENSURE(ctx->lp_h0, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  ENSURE(ctx->lp_h1, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  double* z = buf_ptr<double>(ctx->lp_z);
  MpScratch* msc = buf_ptr<MpScratch>(ctx->lp_sc);
  MpnnWork mw = infer_work(ctx);
  RESET_ERR();
  rc = amg_apply_pre(ctx, d_r, z, nullptr);
  if (rc) return rc;
  if (d_xfix && n) CK(cudaMemcpyAsync(d_xfix, z, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  double* r2 = amg_fine_scratch(ctx);
  rc = amg_residual_fine(ctx, d_r, z, r2, nullptr);
  if (rc) return rc;
  if (d_r2 && n) CK(cudaMemcpyAsync(d_r2, r2, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_winvd && n) CK(cudaMemcpyAsync(d_winvd, ctx->lm_winvd.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(launch_mp_rr(n, r2, msc, ctx->stream));
  CK(launch_mp_forward(graph_view(ctx), params_view(ctx), r2, buf_ptr<double>(ctx->lm_winvd), &msc->rr,
                       buf_ptr<float>(ctx->lp_sf), nullptr, mw, false, z, z, ctx->mbar_spin,
                       buf_ptr<int>(ctx->err_word), ctx->stream));
  if (d_z && n) CK(cudaMemcpyAsync(d_z, z, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  READ_ERR();
  if (ctx->h_err[kErrTimeout] != kErrNone)
    return fail(ctx, CSTG_ERR_TIMEOUT, "learned_cycle_parts: a tensor-core wait timed out");
  return CSTG_OK;
}

int cstg_trainer_accumulate_cycle(cstg_trainer* tr, cstg_ctx* ctx, int n_samples, const double* d_R,
                                  const double* d_E, double* losses) {
  if (!tr) return CSTG_ERR_INVALID_ARGUMENT;
  tr->err.clear();
  TK(cudaSetDevice(tr->device));
  if (!ctx || ctx->device != tr->device)
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: the context must be on the trainer's device");
  if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
    return tfail(tr, CSTG_ERR_STATE, "trainer_accumulate: call cstg_learned_setup on the context first");
  if (n_samples < 0 || (n_samples > 0 && (!d_R || !d_E)))
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: bad samples");
  if (!aligned16(d_R) || !aligned16(d_E))
    return tfail(tr, CSTG_ERR_INVALID_ARGUMENT, "trainer_accumulate: samples must be 16-byte aligned");
  {
    const int rc = cycle_ready(ctx);  // (the context's own error text on failure)
    if (rc) return tfail(tr, rc, "trainer_accumulate: %s", ctx->err.c_str());
  }
  const int N = ctx->n_nodes, n = ctx->n_rows;
  MpnnWork w;
  int rc = trainer_work(tr, N, w);
  if (rc) return rc;
  // everything runs on the context's stream, where the hierarchy and the samples' producers are
  TK(cudaStreamSynchronize(tr->stream));
  cudaStream_t s = ctx->stream;
  const MpnnGraph g = graph_view(ctx);
  MpnnParams P;
  P.pb = static_cast<const __nv_bfloat16*>(tr->pb.p);
  P.pf = static_cast<const float*>(tr->pf.p);
  MpScratch* sc = static_cast<MpScratch*>(tr->sc.p);
  const BlockMatrix bm = block_view(ctx);
  const double* winvd = buf_ptr<double>(ctx->lm_winvd);
  double* z = static_cast<double*>(tr->z.p);
  double* az = static_cast<double*>(tr->az.p);
  float* grad = static_cast<float*>(tr->grad.p);
  int* err = buf_ptr<int>(ctx->err_word);
  TK(cudaMemsetAsync(err, 0x7f, sizeof(int) * kErrSlots, s));
  for (int i = 0; i < n_samples; ++i) {
    const double* r = d_R + (size_t)i * n;
    const double* e = d_E + (size_t)i * n;
    rc = cycle_apply(ctx, g, P, w, sc, winvd, r, z, nullptr, true, s);
    if (rc) return tfail(tr, rc, "trainer_accumulate: %s", ctx->err.c_str());
    TK(launch_spmv(&bm, nullptr, z, az, s));
    TK(launch_mp_loss(N, z, az, r, e, winvd, sc, w, s));
    if (losses) TK(cudaMemcpyAsync(&losses[i], &sc->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    TK(launch_mp_backward(g, P, w, grad, ctx->mbar_spin, err, s));
  }
  int h_err[kErrSlots];
  TK(cudaMemcpyAsync(h_err, err, sizeof h_err, cudaMemcpyDeviceToHost, s));
  TK(cudaStreamSynchronize(s));
  if (h_err[kErrTimeout] != kErrNone) return tfail(tr, CSTG_ERR_TIMEOUT, "trainer: a tensor-core wait timed out");
  return CSTG_OK;
}

}  // extern "C"

extern "C" int cstg_learned_time(cstg_ctx* ctx, int reps, double* out) {
  BEGIN(ctx);
  if (reps < 1 || !out) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "learned_time: bad arguments");
  if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
    return fail(ctx, CSTG_ERR_STATE, "learned_time: call cstg_learned_setup after cstg_pcg_setup");
  const int N = ctx->n_nodes, n = ctx->n_rows;
  ENSURE(ctx->lp_h0, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  ENSURE(ctx->lp_h1, sizeof(__nv_bfloat16) * (size_t)N * kMpF);
  ENSURE(ctx->lp_z, sizeof(double) * (size_t)std::max(n, 1));
  ENSURE(ctx->vec_in, sizeof(double) * (size_t)std::max(n, 1));
  double* r = buf_ptr<double>(ctx->vec_in);
  double* z = buf_ptr<double>(ctx->lp_z);
  CK(cudaMemsetAsync(r, 0, sizeof(double) * (size_t)n, ctx->stream));
  if (n) CK(launch_mp_smoother_weights(n, buf_ptr<double>(ctx->inv_diag), buf_ptr<double>(ctx->inv_diag), 1.0, r,
                                       ctx->stream));  // r_i = invd_i / invd_0: a nonzero residual
  MpScratch* sc = buf_ptr<MpScratch>(ctx->lp_sc);
  MpnnWork mw = infer_work(ctx);
  CK(launch_mp_rr(n, r, sc, ctx->stream));
  RESET_ERR();
  // whole applications, then each stage alone (the same launches launch_mp_forward issues)
  float ms = 0.f;
  for (int stage = 0; stage < 4; ++stage) {
    for (int w = 0; w < 2; ++w) {  // warm-up, then timed
      CK(cudaEventRecord(ctx->ev0, ctx->stream));
      for (int k = 0; k < reps; ++k)
        CK(launch_mp_stage(graph_view(ctx), params_view(ctx), stage, r, buf_ptr<double>(ctx->inv_diag), &sc->rr,
                           buf_ptr<float>(ctx->lp_sf), mw, z, ctx->mbar_spin, buf_ptr<int>(ctx->err_word),
                           ctx->stream));
      CK(cudaEventRecord(ctx->ev1, ctx->stream));
    }
    CK(cudaEventSynchronize(ctx->ev1));
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    out[stage] = ms * 1e-3 / reps;
  }
  READ_ERR();
  if (ctx->h_err[kErrTimeout] != kErrNone) return fail(ctx, CSTG_ERR_TIMEOUT, "learned_time: a tensor-core wait timed out");
  return CSTG_OK;
}
