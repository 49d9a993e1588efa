// C ABI of the batched solve (cstg_batch_solve / _device / cstg_batch_autotune): argument and
// plate-table checks, the largest-first work order, the interleaved load-case buffers, the
// CUDA graph that holds one batched solve, and the launch-shape autotuner.
#include <cuda_runtime.h>

#include <numeric>

#include "ctx.h"

static_assert(sizeof(cstg_batch_result) == sizeof(BatchResultDev), "result layouts differ");

namespace {

constexpr int kMaxGroup = 4;  // load cases solved together (one matrix read for all of them)

struct Shape {
  int cluster, threads;
};
constexpr Shape kShapes[] = {{1, 256}, {1, 512}, {2, 256}, {2, 512}, {4, 256},  {4, 512},
                             {8, 256}, {8, 512}, {16, 256}, {16, 512}};

unsigned long long mix(unsigned long long h, unsigned long long v) {
  h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
  return h;
}

int check_args(cstg_ctx* ctx, int n_sys, const int32_t* offs, int n_rhs, const cstg_solver_options* opt,
               cstg_solver_options& o) {
  if (ctx->kind != 1 || !ctx->has_values)
    return fail(ctx, CSTG_ERR_STATE, "batch_solve: no mesh-pattern matrix (cstg_build_pattern + assemble)");
  if (!ctx->setup_done) return fail(ctx, CSTG_ERR_STATE, "batch_solve: call cstg_pcg_setup first");
  if (n_sys < 1 || !offs || n_rhs < 1)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: bad arguments");
  if (offs[0] != 0 || offs[n_sys] != ctx->n_nodes)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT,
                "batch_solve: node_offsets must run from 0 to the node count (%d)", ctx->n_nodes);
  for (int s = 0; s < n_sys; ++s)
    if (offs[s + 1] < offs[s])
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: node_offsets decrease at system %d", s);
  if (opt)
    o = *opt;
  else
    cstg_default_options(&o);
  if (!(o.rtol > 0.0) || o.max_iter < 1 || o.max_refinements < 0)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: bad solver options");
  if (o.precision != CSTG_PRECISION_FP64 && o.precision != CSTG_PRECISION_MIXED)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: unknown precision %d", o.precision);
  if (o.record_history)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "batch_solve: no residual history in batched solves");
  return CSTG_OK;
}

// Plate table, work order (largest first) and the coupling check, redone when the table or a
// device buffer changed; the interleaved vectors; the FP32 operator.
int prepare(cstg_ctx* ctx, int n_sys, const int32_t* offs, int n_rhs, const cstg_solver_options& o) {
  const std::vector<int32_t> table(offs, offs + n_sys + 1);
  const size_t group = (size_t)std::min(n_rhs, kMaxGroup);
  const size_t vec = sizeof(double) * (size_t)ctx->n_rows * group;
  ENSURE(ctx->bat_sys, sizeof(int) * table.size());
  ENSURE(ctx->bat_order, sizeof(int) * (size_t)n_sys);
  ENSURE(ctx->bat_queue, 256);
  ENSURE(ctx->bat_b, vec);
  ENSURE(ctx->bat_x, vec);
  ENSURE(ctx->bat_r, vec);
  ENSURE(ctx->bat_p, vec);
  ENSURE(ctx->bat_Ap, vec);
  ENSURE(ctx->bat_stats, sizeof(BatchResultDev) * (size_t)n_sys * (size_t)n_rhs);
  if (o.precision == CSTG_PRECISION_MIXED) {
    const int rc = ensure_mixed(ctx);
    if (rc) return rc;
  }
  if (ctx->bat_offsets != table || ctx->bat_checked_gen != ctx->generation) {
    std::vector<int32_t> order(n_sys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return table[a + 1] - table[a] > table[b + 1] - table[b];
    });
    CK(cudaMemcpyAsync(ctx->bat_sys.p, table.data(), sizeof(int) * table.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemcpyAsync(ctx->bat_order.p, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice,
                       ctx->stream));
    RESET_ERR();
    CK(launch_batch_check(ctx->n_nodes, n_sys, buf_ptr<int>(ctx->bat_sys), buf_ptr<int>(ctx->node_ptr),
                          buf_ptr<int>(ctx->bnbr), buf_ptr<int>(ctx->err_word), ctx->stream));
    READ_ERR();  // also waits for the host tables' copies
    if (ctx->h_err[kErrBatch] != kErrNone) {
      ctx->bat_offsets.clear();
      const int n = ctx->h_err[kErrBatch];
      const int s = (int)(std::upper_bound(table.begin(), table.end(), n) - table.begin()) - 1;
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT,
                  "batch_solve: node %d of system %d is coupled to a node of another system", n, s);
    }
    ctx->bat_offsets = table;
    ctx->bat_checked_gen = ctx->generation;
  }
  return CSTG_OK;
}

// Enqueues one batched solve: per group of up to four load cases, pack, the persistent launch,
// unpack. `launched` receives the number of kernel launches enqueued.
int enqueue(cstg_ctx* ctx, int n_sys, int n_rhs, const double* d_b, double* d_x, const cstg_solver_options& o,
            Shape sh, int n_clusters, long long* launched) {
  const int N = ctx->n_nodes;
  const long long ld = ctx->n_rows;
  long long k = 0;
  for (int q0 = 0; q0 < n_rhs; q0 += kMaxGroup) {
    const int R = std::min(kMaxGroup, n_rhs - q0);
    CK(cudaMemsetAsync(ctx->bat_queue.p, 0, sizeof(int), ctx->stream));
    CK(launch_batch_pack(N, R, q0, ld, d_b, buf_ptr<double>(ctx->bat_b), ctx->stream));
    BatchArgs a;
    a.n_sys = n_sys;
    a.sys_node = buf_ptr<int>(ctx->bat_sys);
    a.order = buf_ptr<int>(ctx->bat_order);
    a.queue = buf_ptr<int>(ctx->bat_queue);
    if (o.precision == CSTG_PRECISION_MIXED) a.A32 = mixed_view(ctx);
    a.A64 = block_view(ctx);
    a.start_fp64 = o.precision == CSTG_PRECISION_FP64;
    a.inv_diag = buf_ptr<double>(ctx->inv_diag);
    a.b = buf_ptr<double>(ctx->bat_b);
    a.x = buf_ptr<double>(ctx->bat_x);
    a.r = buf_ptr<double>(ctx->bat_r);
    a.p = buf_ptr<double>(ctx->bat_p);
    a.Ap = buf_ptr<double>(ctx->bat_Ap);
    a.rtol = o.rtol;
    a.max_iter = o.max_iter;
    a.max_refine = o.max_refinements;
    a.res = buf_ptr<BatchResultDev>(ctx->bat_stats);
    a.res_stride = n_rhs;
    a.res_offset = q0;
    CK(launch_batch_pcg(a, R, sh.cluster, sh.threads, n_clusters, ctx->stream));
    CK(launch_batch_unpack(N, R, q0, ld, buf_ptr<double>(ctx->bat_x), d_x, ctx->stream));
    k += N > 0 ? 3 : 1;
  }
  *launched = k;
  return CSTG_OK;
}

int fit_shape(cstg_ctx* ctx, int n_rhs, Shape sh, int* max_clusters) {
  (void)ctx;
  int worst = INT_MAX;
  for (int q0 = 0; q0 < n_rhs; q0 += kMaxGroup) {
    int m = 0;
    const cudaError_t e = batch_max_clusters(std::min(kMaxGroup, n_rhs - q0), sh.cluster, sh.threads, &m);
    if (e != cudaSuccess) {
      cudaGetLastError();
      m = 0;
    }
    worst = std::min(worst, m);
  }
  *max_clusters = worst == INT_MAX ? 0 : worst;
  return CSTG_OK;
}

// One batched solve with shape `sh` (graph-captured when `graph`), timed with CUDA events.
int run(cstg_ctx* ctx, int n_sys, int n_rhs, const double* d_b, double* d_x, const cstg_solver_options& o,
        Shape sh, bool graph, double* seconds) {
  int maxc = 0;
  fit_shape(ctx, n_rhs, sh, &maxc);
  if (maxc < 1)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "batch_solve: launch shape %d CTAs x %d threads does not fit",
                sh.cluster, sh.threads);
  const int n_clusters = std::min(maxc, n_sys);
  long long launched = 0;
  if (graph) {
    unsigned long long key = 0x5eedull;
    for (unsigned long long v :
         {(unsigned long long)ctx->generation, (unsigned long long)n_sys, (unsigned long long)n_rhs,
          (unsigned long long)(uintptr_t)d_b, (unsigned long long)(uintptr_t)d_x, (unsigned long long)sh.cluster,
          (unsigned long long)sh.threads, (unsigned long long)n_clusters, (unsigned long long)o.max_iter,
          (unsigned long long)o.max_refinements, (unsigned long long)o.precision})
      key = mix(key, v);
    unsigned long long rt;
    std::memcpy(&rt, &o.rtol, sizeof rt);
    key = mix(key, rt);
    if (!ctx->bat_graph || ctx->bat_graph_key != key) {
      if (ctx->bat_graph) {
        cudaGraphExecDestroy(ctx->bat_graph);
        ctx->bat_graph = nullptr;
      }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue(ctx, n_sys, n_rhs, d_b, d_x, o, sh, n_clusters, &launched);
      const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
      count_launches(-launched);  // captured, not run: counted per graph launch below
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      CK(ee);
      const cudaError_t ie = cudaGraphInstantiate(&ctx->bat_graph, g, 0);
      cudaGraphDestroy(g);
      CK(ie);
      ctx->bat_graph_key = key;
      ctx->bat_graph_launches = launched;
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CK(cudaGraphLaunch(ctx->bat_graph, ctx->stream));
    count_launches(ctx->bat_graph_launches);
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
  } else {
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    const int rc = enqueue(ctx, n_sys, n_rhs, d_b, d_x, o, sh, n_clusters, &launched);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
  }
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (seconds) *seconds = ms * 1e-3;
  return CSTG_OK;
}

Shape pick(cstg_ctx* ctx, const cstg_batch_config* cfg) {
  if (cfg && cfg->cluster_ctas > 0) return {cfg->cluster_ctas, cfg->threads};
  if (ctx->bat_cfg.cluster_ctas > 0) return {ctx->bat_cfg.cluster_ctas, ctx->bat_cfg.threads};
  return {8, 512};
}

int results_out(cstg_ctx* ctx, int n_sys, int n_rhs, cstg_batch_result* results) {
  if (!results) return CSTG_OK;
  CK(cudaMemcpyAsync(results, ctx->bat_stats.p, sizeof(BatchResultDev) * (size_t)n_sys * (size_t)n_rhs,
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

int solve_device(cstg_ctx* ctx, int n_sys, const int32_t* offs, int n_rhs, const double* d_b, double* d_x,
                 const cstg_solver_options* opt, const cstg_batch_config* cfg, cstg_batch_result* results,
                 double* seconds) {
  cstg_solver_options o;
  int rc = check_args(ctx, n_sys, offs, n_rhs, opt, o);
  if (rc) return rc;
  if (ctx->n_rows && (!d_b || !d_x)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: null vector");
  if (!aligned16(d_b) || !aligned16(d_x))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: device vectors must be 16-byte aligned");
  const Shape sh = pick(ctx, cfg);
  bool known = false;
  for (const Shape& k : kShapes) known |= k.cluster == sh.cluster && k.threads == sh.threads;
  if (!known)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: unsupported launch shape %d CTAs x %d threads",
                sh.cluster, sh.threads);
  rc = prepare(ctx, n_sys, offs, n_rhs, o);
  if (rc) return rc;
  rc = run(ctx, n_sys, n_rhs, d_b, d_x, o, sh, true, seconds);
  if (rc) return rc;
  return results_out(ctx, n_sys, n_rhs, results);
}

}  // namespace

extern "C" {

int cstg_batch_solve_device(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs,
                            const double* d_b, double* d_x, const cstg_solver_options* opt,
                            const cstg_batch_config* config, cstg_batch_result* results, double* seconds) {
  BEGIN(ctx);
  return solve_device(ctx, n_systems, node_offsets, n_rhs, d_b, d_x, opt, config, results, seconds);
}

int cstg_batch_solve(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs, const double* b,
                     double* x, const cstg_solver_options* opt, const cstg_batch_config* config,
                     cstg_batch_result* results, double* seconds) {
  BEGIN(ctx);
  if (n_rhs < 1) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: bad arguments");
  const size_t n = (size_t)ctx->n_rows * (size_t)n_rhs;
  if (n && (!b || !x)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_solve: null vector");
  ENSURE(ctx->bat_in, sizeof(double) * n);
  ENSURE(ctx->bat_out, sizeof(double) * n);
  if (n) CK(cudaMemcpyAsync(ctx->bat_in.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  const int rc = solve_device(ctx, n_systems, node_offsets, n_rhs, buf_ptr<double>(ctx->bat_in),
                              buf_ptr<double>(ctx->bat_out), opt, config, results, seconds);
  if (rc) return rc;
  if (n) CK(cudaMemcpyAsync(x, ctx->bat_out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

int cstg_batch_autotune(cstg_ctx* ctx, int n_systems, const int32_t* node_offsets, int n_rhs, const double* d_b,
                        double* d_x, const cstg_solver_options* opt, cstg_batch_config* best,
                        double* best_seconds) {
  BEGIN(ctx);
  cstg_solver_options o;
  int rc = check_args(ctx, n_systems, node_offsets, n_rhs, opt, o);
  if (rc) return rc;
  if (ctx->n_rows && (!d_b || !d_x)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_autotune: null vector");
  if (!aligned16(d_b) || !aligned16(d_x))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "batch_autotune: device vectors must be 16-byte aligned");
  rc = prepare(ctx, n_systems, node_offsets, n_rhs, o);
  if (rc) return rc;
  Shape win{0, 0};
  double t_win = 0.0;
  for (const Shape& sh : kShapes) {
    int maxc = 0;
    fit_shape(ctx, n_rhs, sh, &maxc);
    if (maxc < 1) continue;
    double t0 = 0.0, t1 = 0.0;
    rc = run(ctx, n_systems, n_rhs, d_b, d_x, o, sh, false, &t0);  // warm-up (first-launch costs)
    if (rc) return rc;
    rc = run(ctx, n_systems, n_rhs, d_b, d_x, o, sh, false, &t1);
    if (rc) return rc;
    if (win.cluster == 0 || t1 < t_win) {
      win = sh;
      t_win = t1;
    }
  }
  if (win.cluster == 0) return fail(ctx, CSTG_ERR_UNSUPPORTED, "batch_autotune: no launch shape fits");
  ctx->bat_cfg.cluster_ctas = win.cluster;
  ctx->bat_cfg.threads = win.threads;
  if (best) *best = ctx->bat_cfg;
  if (best_seconds) *best_seconds = t_win;
  return CSTG_OK;
}

}  // extern "C"
