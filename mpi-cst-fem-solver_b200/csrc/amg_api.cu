// Host side of the smoothed-aggregation multigrid preconditioner: the level hierarchy on a
// context (built on the first CSTG_PRECOND_AMG solve after cstg_pcg_setup, or by cstg_amg_setup)
// and the V(2,2) cycle z = M r used inside the flexible-CG driver of learned_api.cu.
#include <cuda_runtime.h>

#include <chrono>
#include <vector>

#include "ctx.h"

namespace {

// dense inverse at or below this many coarse DOFs (one-CTA Gauss-Jordan: its time grows as n^3 on
// one SM, 31 ms at 453 DOFs, so the hierarchy coarsens once more rather than invert a level that size)
constexpr int kCoarsestDofs = 200;
constexpr int kMaxLevels = 10;
constexpr int kPowerIters = 20;
constexpr int kMaxMisRounds = 200;
// coarse levels at or below this many DOFs run in the tail kernel: one cluster of at most 16 SMs
// beats separate full-GPU launches only where a level's work is a few microseconds of latency
constexpr int kTailMaxDofs = 5000;
// Aggregation follows every connection on the finest level but only the strong ones below it
// (||A_ij|| >= theta sqrt(||A_ii|| ||A_jj||)): the Galerkin operators' wider stencils otherwise
// give aggregates of 20+ nodes, and the cycle converges markedly slower (111 -> 76 iterations on
// the 2M-DOF plate with this threshold, 2-4x larger levels below the first; on the finest level
// the same filter shrinks the first coarsening from 7x to 3x and costs more per cycle than it
// saves). Thresholds of 0.02-0.05 gave the same step time within 2 %; 0.12 and above can make a
// coarse row exceed its bound, and the level then aggregates over every connection.
constexpr double kThetaCoarse = 0.03;

}  // namespace

struct AmgLevel {
  int B = 2, n = 0, nc = 0;
  DevBuf ptr, col, val;          // A (finest level: ptr/col are the context's node pattern)
  const int* a_ptr = nullptr;
  const int* a_col = nullptr;
  DevBuf dinv, lam;
  DevBuf p_ptr, p_col, p_val, p_row, pt_ptr, pt_idx;  // transfer to the next level
  DevBuf xa, xb, r, bc;          // cycle vectors (bc: this level's right-hand side, levels >= 1)
  // the cycle's FP32 operators: this level's matrix (levels >= 1) and the transfer to the next
  // level, by fine row (p32) and by coarse row (pt32 with the fine row of each block in pt_row)
  DevBuf val32, p32, pt32, pt_row;
  int nnz_p = 0;
  int nnzb = 0;  // blocks of this level's matrix
  AmgBsr A() const {
    AmgBsr m;
    m.n = n;
    m.ptr = a_ptr;
    m.col = a_col;
    m.val = static_cast<const double*>(val.p);
    return m;
  }
  AmgBsr32 A32() const {
    AmgBsr32 m;
    m.n = n;
    m.nnzb = nnzb;
    m.ptr = a_ptr;
    m.col = a_col;
    m.val = static_cast<const float*>(val32.p);
    return m;
  }
  AmgBsr P() const {
    AmgBsr m;
    m.n = n;
    m.ptr = static_cast<const int*>(p_ptr.p);
    m.col = static_cast<const int*>(p_col.p);
    m.val = static_cast<const double*>(p_val.p);
    return m;
  }
};

struct AmgData {
  std::vector<AmgLevel> L;    // level storage: only grows, so rebuilds reuse the buffers
  int nl = 0;                 // levels of the current hierarchy (L[0 .. nl-1])
  DevBuf Minv, piv;
  int n_coarse = 0;           // DOFs of the dense coarsest level
  unsigned long long built_for = ~0ull;  // setup_count of the matrix it was built from
  double setup_seconds = 0.0;
  // the bottom of the cycle in one cluster launch (tail_level 0: every level launches its own kernels)
  bool tail_enabled = true;
  int cheb = 1;  // smoother: Chebyshev (1) or damped Jacobi (0)
  // strength-of-connection thresholds of the aggregation on the finest / the coarser levels
  double theta_fine = 0.0, theta_coarse = kThetaCoarse;
  int tail_cluster = -1;  // CTAs of the tail cluster on this device (-1 not yet queried, 0 none fits)
  int tail_level = 0;
  AmgTail tail;
  // scratch of the setup
  DevBuf state, m1, newroot, near, und, root_id, flags, agg1, agg2, agg_ptr, members, cnt, cur, P0, Bf, Bc, cnt2,
      ap_ptr, ap_col, ap_val, part, vx, vy, strong, dn, pt_tmp;
};

void cstg_host::amg_free(cstg_ctx* ctx) {
  if (!ctx->amg) return;
  AmgData* d = ctx->amg;
  for (AmgLevel& l : d->L) {
    DevBuf* all[] = {&l.ptr, &l.col, &l.val, &l.dinv, &l.lam, &l.p_ptr, &l.p_col, &l.p_val, &l.p_row, &l.pt_ptr,
                     &l.pt_idx, &l.xa, &l.xb, &l.r, &l.bc, &l.val32, &l.p32, &l.pt32, &l.pt_row};
    for (DevBuf* b : all) free_buf(*b);
  }
  DevBuf* all[] = {&d->Minv, &d->piv, &d->state, &d->m1, &d->newroot, &d->near, &d->und, &d->root_id, &d->flags,
                   &d->agg1, &d->agg2, &d->agg_ptr, &d->members, &d->cnt, &d->cur, &d->P0, &d->Bf, &d->Bc,
                   &d->cnt2, &d->ap_ptr, &d->ap_col, &d->ap_val, &d->part, &d->vx, &d->vy, &d->strong, &d->dn, &d->pt_tmp};
  for (DevBuf* b : all) free_buf(*b);
  delete d;
  ctx->amg = nullptr;
}

namespace {

int read_int(cstg_ctx* ctx, const int* d, int* h) {
  CK(cudaMemcpyAsync(h, d, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

// exclusive scan of n ints into out[0..n] and the total
int scan_total(cstg_ctx* ctx, const int* in, int n, int* out, int* total) {
  ENSURE(ctx->scan_tmp, sizeof(int) * (size_t)scan_tmp_ints(std::max(n, 1)));
  CK(scan_exclusive(in, n, out, buf_ptr<int>(ctx->scan_tmp), ctx->stream));
  return read_int(ctx, out + n, total);
}

// One coarsening step from level l (matrix and nullspace Bf set) to level l + 1.
// theta: strength-of-connection threshold of the aggregation (0: every connection)
int coarsen(cstg_ctx* ctx, AmgData* d, int l, double theta, bool* stop) {
  AmgLevel& lv = d->L[l];
  const int B = lv.B, n = lv.n;
  const AmgBsr A = lv.A();
  int* err = buf_ptr<int>(ctx->err_word);
  ENSURE(d->state, sizeof(int) * (size_t)n);
  ENSURE(d->m1, sizeof(unsigned long long) * (size_t)n);
  ENSURE(d->newroot, sizeof(int) * (size_t)n);
  ENSURE(d->near, sizeof(int) * (size_t)n);
  ENSURE(d->und, 256);
  ENSURE(d->root_id, sizeof(int) * ((size_t)n + 1));
  ENSURE(d->flags, sizeof(int) * (size_t)n);
  ENSURE(d->agg1, sizeof(int) * (size_t)n);
  ENSURE(d->agg2, sizeof(int) * (size_t)n);
  ENSURE(d->members, sizeof(int) * (size_t)n);
  // lambda_max(D^-1 A)
  ENSURE(lv.lam, sizeof(double));
  ENSURE(d->part, amg_lambda_scratch());
  ENSURE(d->vx, sizeof(double) * (size_t)n * B);
  ENSURE(d->vy, sizeof(double) * (size_t)n * B);
  // (on the FP32 operators the smoother applies: the finest level's difference form, else this
  // level's entry-major copy, built with the Galerkin product of the level above)
  if (l == 0) {
    const MixedMatrix mm = mixed_view(ctx);
    CK(amg_lambda_f32(&mm, nullptr, buf_ptr<double>(lv.dinv), buf_ptr<double>(d->vx), buf_ptr<double>(d->vy),
                      buf_ptr<double>(d->part), buf_ptr<double>(lv.lam), kPowerIters, ctx->stream));
  } else {
    const AmgBsr32 a32 = lv.A32();
    CK(amg_lambda_f32(nullptr, &a32, buf_ptr<double>(lv.dinv), buf_ptr<double>(d->vx), buf_ptr<double>(d->vy),
                      buf_ptr<double>(d->part), buf_ptr<double>(lv.lam), kPowerIters, ctx->stream));
  }
  // the strong connections the aggregation follows (none dropped at theta 0)
  const unsigned char* strong = nullptr;
  if (theta > 0.0) {
    int nnzb = 0;
    const int rc = read_int(ctx, lv.a_ptr + n, &nnzb);
    if (rc) return rc;
    ENSURE(d->strong, (size_t)std::max(nnzb, 1));
    ENSURE(d->dn, sizeof(double) * (size_t)n);
    CK(amg_strength(B, A, theta, buf_ptr<double>(d->dn), buf_ptr<unsigned char>(d->strong), ctx->stream));
    strong = buf_ptr<unsigned char>(d->strong);
  }
  // distance-2 maximal independent set of the strong-connection graph
  CK(cudaMemsetAsync(d->state.p, 0, sizeof(int) * (size_t)n, ctx->stream));
  int und = n;
  for (int round = 0; und > 0; ++round) {
    if (round >= kMaxMisRounds) return fail(ctx, CSTG_ERR_UNSUPPORTED, "amg_setup: aggregation did not settle");
    CK(amg_mis_round(A, strong, buf_ptr<int>(d->state), buf_ptr<unsigned long long>(d->m1), buf_ptr<int>(d->newroot),
                     buf_ptr<int>(d->near), buf_ptr<int>(d->und), ctx->stream));
    const int rc = read_int(ctx, buf_ptr<int>(d->und), &und);
    if (rc) return rc;
  }
  int n_roots = 0, n_left = 0;
  CK(amg_flag_eq(n, buf_ptr<int>(d->state), 1, buf_ptr<int>(d->flags), ctx->stream));
  int rc = scan_total(ctx, buf_ptr<int>(d->flags), n, buf_ptr<int>(d->root_id), &n_roots);
  if (rc) return rc;
  CK(amg_aggregate(B, A, strong, buf_ptr<int>(d->state), buf_ptr<int>(d->root_id), buf_ptr<int>(d->agg1),
                   buf_ptr<int>(d->agg2), ctx->stream));
  CK(amg_flag_negative(n, buf_ptr<int>(d->agg2), buf_ptr<int>(d->flags), ctx->stream));
  ENSURE(d->cnt, sizeof(int) * ((size_t)n + 1));
  rc = scan_total(ctx, buf_ptr<int>(d->flags), n, buf_ptr<int>(d->cnt), &n_left);
  if (rc) return rc;
  CK(amg_phase3(n, n_roots, buf_ptr<int>(d->cnt), buf_ptr<int>(d->agg2), ctx->stream));
  const int nc = n_roots + n_left;
  if (nc <= 0 || nc > (n * 4) / 5) {  // coarsening stalled: this level becomes the coarsest
    *stop = true;
    return CSTG_OK;
  }
  const int* agg = buf_ptr<int>(d->agg2);
  // aggregate members, tentative prolongator, coarse nullspace
  ENSURE(d->agg_ptr, sizeof(int) * ((size_t)nc + 1));
  ENSURE(d->cnt, sizeof(int) * ((size_t)std::max(n, nc) + 1));
  ENSURE(d->cur, sizeof(int) * ((size_t)std::max(n, nc) + 1));
  ENSURE(ctx->scan_tmp, sizeof(int) * (size_t)scan_tmp_ints(std::max(std::max(n, nc), 1)));
  CK(amg_group(n, agg, nc, buf_ptr<int>(d->agg_ptr), buf_ptr<int>(d->cnt), buf_ptr<int>(d->cur),
               buf_ptr<int>(d->members), buf_ptr<int>(ctx->scan_tmp), ctx->stream));
  ENSURE(d->P0, sizeof(double) * (size_t)n * B * 3);
  ENSURE(d->Bc, sizeof(double) * (size_t)nc * 9);
  CK(amg_tentative(B, nc, buf_ptr<int>(d->agg_ptr), buf_ptr<int>(d->members), buf_ptr<double>(d->Bf),
                   buf_ptr<double>(d->P0), buf_ptr<double>(d->Bc), err, ctx->stream));
  // smoothed prolongator
  ENSURE(lv.p_ptr, sizeof(int) * ((size_t)n + 1));
  CK(amg_p_count(B, A, agg, buf_ptr<int>(d->cnt), err, ctx->stream));
  int nnz_p = 0;
  rc = scan_total(ctx, buf_ptr<int>(d->cnt), n, buf_ptr<int>(lv.p_ptr), &nnz_p);
  if (rc) return rc;
  READ_ERR();
  if (ctx->h_err[kErrAmg] != kErrNone)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "amg_setup: level %d: an aggregate or a prolongator row is too large", l);
  ENSURE(lv.p_col, sizeof(int) * (size_t)std::max(nnz_p, 1));
  ENSURE(lv.p_val, sizeof(double) * (size_t)std::max(nnz_p, 1) * B * 3);
  AmgBsr P = lv.P();
  CK(amg_p_fill(B, A, agg, buf_ptr<double>(d->P0), buf_ptr<double>(lv.dinv), buf_ptr<double>(lv.lam), P, ctx->stream));
  // AP
  ENSURE(d->ap_ptr, sizeof(int) * ((size_t)n + 1));
  CK(amg_ap_count(B, A, P, buf_ptr<int>(d->cnt), err, ctx->stream));
  int nnz_ap = 0;
  rc = scan_total(ctx, buf_ptr<int>(d->cnt), n, buf_ptr<int>(d->ap_ptr), &nnz_ap);
  if (rc) return rc;
  ENSURE(d->ap_col, sizeof(int) * (size_t)std::max(nnz_ap, 1));
  ENSURE(d->ap_val, sizeof(double) * (size_t)std::max(nnz_ap, 1) * B * 3);
  AmgBsr AP;
  AP.n = n;
  AP.ptr = buf_ptr<int>(d->ap_ptr);
  AP.col = buf_ptr<int>(d->ap_col);
  AP.val = buf_ptr<double>(d->ap_val);
  CK(amg_ap_fill(B, A, P, AP, ctx->stream));
  // P' lists
  ENSURE(lv.p_row, sizeof(int) * (size_t)std::max(nnz_p, 1));
  ENSURE(lv.pt_ptr, sizeof(int) * ((size_t)nc + 1));
  ENSURE(lv.pt_idx, sizeof(int) * (size_t)std::max(nnz_p, 1));
  ENSURE(d->pt_tmp, sizeof(int) * (size_t)std::max(nnz_p, 1));
  CK(amg_pt(n, nc, P, buf_ptr<int>(lv.p_row), buf_ptr<int>(lv.pt_ptr), buf_ptr<int>(d->cnt), buf_ptr<int>(d->cur),
            buf_ptr<int>(d->pt_tmp), buf_ptr<int>(lv.pt_idx), buf_ptr<int>(ctx->scan_tmp), ctx->stream));
  // the cycle's FP32 copies of P
  ENSURE(lv.p32, sizeof(float) * (size_t)std::max(nnz_p, 1) * B * 3);
  ENSURE(lv.pt32, sizeof(float) * (size_t)std::max(nnz_p, 1) * B * 3);
  ENSURE(lv.pt_row, sizeof(int) * (size_t)std::max(nnz_p, 1));
  lv.nnz_p = nnz_p;
  CK(amg_transfer_f32(B, P, nnz_p, buf_ptr<int>(lv.pt_idx), buf_ptr<int>(lv.p_row), buf_ptr<float>(lv.p32),
                      buf_ptr<int>(lv.pt_row), buf_ptr<float>(lv.pt32), ctx->stream));
  // coarse operator
  if ((int)d->L.size() < l + 2) d->L.emplace_back();
  d->nl = l + 2;
  AmgLevel& nx = d->L[l + 1];
  AmgLevel& cur = d->L[l];  // (re-fetched: emplace_back may move the vector)
  nx.B = 3;
  nx.n = nc;
  cur.nc = nc;
  ENSURE(nx.ptr, sizeof(int) * ((size_t)nc + 1));
  CK(amg_ac_count(B, nc, buf_ptr<int>(cur.pt_ptr), buf_ptr<int>(cur.pt_idx), buf_ptr<int>(cur.p_row), AP,
                  buf_ptr<int>(d->cnt), err, ctx->stream));
  int nnz_c = 0;
  rc = scan_total(ctx, buf_ptr<int>(d->cnt), nc, buf_ptr<int>(nx.ptr), &nnz_c);
  if (rc) return rc;
  READ_ERR();
  if (ctx->h_err[kErrAmg] != kErrNone)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "amg_setup: level %d: a coarse row has more than %d blocks", l + 1,
                kAmgMaxRow);
  ENSURE(nx.col, sizeof(int) * (size_t)std::max(nnz_c, 1));
  ENSURE(nx.val, sizeof(double) * (size_t)std::max(nnz_c, 1) * 9);
  nx.a_ptr = buf_ptr<int>(nx.ptr);
  nx.a_col = buf_ptr<int>(nx.col);
  AmgBsr Ac = nx.A();
  CK(amg_ac_fill(B, nc, buf_ptr<int>(cur.pt_ptr), buf_ptr<int>(cur.pt_idx), buf_ptr<int>(cur.p_row), cur.P(), AP, Ac,
                 ctx->stream));
  ENSURE(nx.val32, sizeof(float) * (size_t)std::max(nnz_c, 1) * 9);
  nx.nnzb = nnz_c;
  CK(amg_coarse_f32(Ac, buf_ptr<float>(nx.val32), ctx->stream));
  // the coarse nullspace becomes the next level's basis
  ENSURE(d->Bf, sizeof(double) * (size_t)std::max(n * B * 3, nc * 9));
  CK(cudaMemcpyAsync(d->Bf.p, d->Bc.p, sizeof(double) * (size_t)nc * 9, cudaMemcpyDeviceToDevice, ctx->stream));
  return CSTG_OK;
}

// Maps the levels from the first level >= 1 with at most kTailMaxDofs DOFs down to the coarsest
// onto one cluster launch (k_amg_tail), when a cluster of 16 (else 8) CTAs fits on the device.
int setup_tail(cstg_ctx* ctx, AmgData* d) {
  d->tail_level = 0;
  if (!d->tail_enabled || d->nl < 3) return CSTG_OK;
  if (d->tail_cluster < 0) {
    d->tail_cluster = 0;
    for (int c : {16, 8}) {
      int m = 0;
      const cudaError_t e = amg_tail(nullptr, d->tail, c, &m, ctx->stream);
      if (e == cudaSuccess && m >= 1) {
        d->tail_cluster = c;
        break;
      }
      cudaGetLastError();  // a shape that cannot launch is not an error of the setup
    }
  }
  if (!d->tail_cluster) return CSTG_OK;
  int lt = 1;
  while (lt < d->nl - 1 && d->L[lt].n * d->L[lt].B > kTailMaxDofs) ++lt;
  if (lt >= d->nl - 1 || d->nl - lt > kAmgTailMax) return CSTG_OK;
  AmgTail& T = d->tail;
  T = AmgTail{};
  T.cheb = d->cheb;
  T.nl = d->nl - lt;
  T.n_coarse = d->n_coarse;
  T.Minv = buf_ptr<double>(d->Minv);
  for (int t = 0; t < T.nl; ++t) {
    AmgLevel& lv = d->L[lt + t];
    AmgTailLevel& v = T.L[t];
    v.b = buf_ptr<double>(lv.bc);
    v.x = buf_ptr<double>(lv.xb);
    if (t + 1 == T.nl) break;
    v.A = lv.A32();
    v.dinv = buf_ptr<double>(lv.dinv);
    v.lam = buf_ptr<double>(lv.lam);
    v.xa = buf_ptr<double>(lv.xa);
    v.r = buf_ptr<double>(lv.r);
    v.nc = lv.nc;
    v.pt_ptr = buf_ptr<int>(lv.pt_ptr);
    v.pt_row = buf_ptr<int>(lv.pt_row);
    v.pt32 = buf_ptr<float>(lv.pt32);
    v.p_ptr = buf_ptr<int>(lv.p_ptr);
    v.p_col = buf_ptr<int>(lv.p_col);
    v.p32 = buf_ptr<float>(lv.p32);
  }
  d->tail_level = lt;
  return CSTG_OK;
}

int amg_build(cstg_ctx* ctx) {
  if (!ctx->amg) {
    ctx->amg = new AmgData();
    ctx->amg->L.reserve(kMaxLevels + 1);
  }
  AmgData* d = ctx->amg;
  const auto t0 = std::chrono::steady_clock::now();
  amg_prepare_launch_shapes();
  if (d->L.empty()) d->L.emplace_back();
  d->nl = 1;
  {
    AmgLevel& f = d->L[0];
    f.B = 2;
    f.n = ctx->n_nodes;
    f.a_ptr = buf_ptr<int>(ctx->node_ptr);
    f.a_col = buf_ptr<int>(ctx->bnbr);
    ENSURE(f.val, sizeof(double) * (size_t)ctx->nnz);
    CK(amg_fine_bsr(f.n, f.a_ptr, buf_ptr<double>(ctx->vals), buf_ptr<double>(f.val), ctx->stream));
    ENSURE(d->Bf, sizeof(double) * (size_t)f.n * 6);
    CK(amg_rigid_modes(f.n, buf_ptr<double>(ctx->xy), buf_ptr<double>(d->Bf), ctx->stream));
  }
  RESET_ERR();
  for (int l = 0;; ++l) {
    AmgLevel& lv = d->L[l];
    ENSURE(lv.dinv, sizeof(double) * (size_t)lv.n * lv.B);
    CK(amg_dinv(lv.B, lv.A(), buf_ptr<double>(lv.dinv), buf_ptr<int>(ctx->err_word), ctx->stream));
    bool stop = lv.n * lv.B <= kCoarsestDofs || l + 1 >= kMaxLevels;
    if (!stop) {
      const double theta = l == 0 ? d->theta_fine : d->theta_coarse;
      int rc = coarsen(ctx, d, l, theta, &stop);
      if (rc == CSTG_ERR_UNSUPPORTED && theta > 0.0 && ctx->h_err[kErrAmg] != kErrNone) {
        // aggregates of the strong connections alone made an aggregate or a coarse row too large
        // for its bound: this level aggregates over every connection instead
        CK(cudaMemsetAsync(buf_ptr<int>(ctx->err_word) + kErrAmg, 0x7f, sizeof(int), ctx->stream));
        rc = coarsen(ctx, d, l, 0.0, &stop);
      }
      if (rc) return rc;
    }
    if (stop) break;
  }
  READ_ERR();
  if (ctx->h_err[kErrDiag] != kErrNone)
    return fail(ctx, CSTG_ERR_NONPOSITIVE_DIAGONAL, "amg_setup: non-positive diagonal on a level");
  AmgLevel& last = d->L[d->nl - 1];
  d->n_coarse = last.n * last.B;
  if (d->n_coarse > 1536)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "amg_setup: coarsest level has %d DOFs (coarsening stalled)", d->n_coarse);
  ENSURE(d->Minv, sizeof(double) * (size_t)d->n_coarse * d->n_coarse);
  ENSURE(d->piv, sizeof(double) * 2 * (size_t)d->n_coarse);
  // (a matrix at or below the coarsest size is its own coarsest level: the cycle is a direct solve)
  CK(amg_coarsest(last.B, last.A(), buf_ptr<double>(d->Minv), buf_ptr<double>(d->piv), ctx->stream));
  // cycle vectors
  for (int l = 0; l < d->nl; ++l) {
    AmgLevel& lv = d->L[l];
    const size_t m = (size_t)lv.n * lv.B;
    ENSURE(lv.xa, sizeof(double) * m);
    ENSURE(lv.xb, sizeof(double) * m);
    ENSURE(lv.r, sizeof(double) * m);
    ENSURE(lv.bc, sizeof(double) * m);
  }
  const int rt = setup_tail(ctx, d);
  if (rt) return rt;
  CK(cudaStreamSynchronize(ctx->stream));
  d->built_for = ctx->setup_count;
  d->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return CSTG_OK;
}

// V(2,2): x = cycle(l, b)
// dots (finest level only, may be null): the flexible-CG scalars, taken in the last sweep
int vcycle(cstg_ctx* ctx, AmgData* d, size_t l, const double* b, double* x, const int* skip,
           const FcgDotSink* dots) {
  AmgLevel& lv = d->L[l];
  cudaStream_t s = ctx->stream;
  if ((int)l + 1 == d->nl) {
    CK(amg_gemv(skip, d->n_coarse, buf_ptr<double>(d->Minv), b, x, s));
    return CSTG_OK;
  }
  if (d->tail_level > 0 && (int)l == d->tail_level && b == d->tail.L[0].b && x == d->tail.L[0].x) {
    CK(amg_tail(skip, d->tail, d->tail_cluster, nullptr, s));
    return CSTG_OK;
  }
  const double* dinv = buf_ptr<double>(lv.dinv);
  const double* lam = buf_ptr<double>(lv.lam);
  double* xa = buf_ptr<double>(lv.xa);
  double* r = buf_ptr<double>(lv.r);
  AmgLevel& nx = d->L[l + 1];
  // every operator of the cycle is FP32 (vectors and accumulation FP64): the finest level smooths
  // with the difference-form operator of the mixed solve, coarse levels with their Galerkin
  // operators rounded symmetrically, and the transfers use FP32 copies of P
  const bool fine = l == 0;
  const MixedMatrix mm = fine ? mixed_view(ctx) : MixedMatrix{};
  const AmgBsr32 A32 = lv.A32();
  const int cheb = d->cheb;
  auto sweep = [&](int mode, const double* xin, const double* xp, double* xout,
                   const FcgDotSink* dk = nullptr) -> cudaError_t {
    return fine ? amg_sweep_f32(skip, mode, cheb, mm, dinv, lam, b, xin, xp, xout, s, dk)
                : amg_sweep3_f32(skip, mode, cheb, A32, dinv, lam, b, xin, xp, xout, s);
  };
  CK(sweep(kSweepFirst, nullptr, nullptr, x));  // two pre-smoothing steps from x = 0
  CK(sweep(kSweepResidual, x, nullptr, r));
  CK(amg_restrict_f32(skip, lv.B, lv.nc, buf_ptr<int>(lv.pt_ptr), buf_ptr<int>(lv.pt_row), buf_ptr<float>(lv.pt32), r,
                      buf_ptr<double>(nx.bc), s));
  const int rc = vcycle(ctx, d, l + 1, buf_ptr<double>(nx.bc), buf_ptr<double>(nx.xb), skip, nullptr);
  if (rc) return rc;
  CK(amg_prolong_f32(skip, lv.B, lv.n, buf_ptr<int>(lv.p_ptr), buf_ptr<int>(lv.p_col), buf_ptr<float>(lv.p32),
                     buf_ptr<double>(nx.xb), x, s));
  CK(sweep(kSweepSmooth, x, nullptr, xa));  // two post-smoothing steps
  const FcgDotSink* dk = fine ? dots : nullptr;
  if (cheb)
    CK(sweep(kSweepSecond, xa, x, x, dk));  // (the previous iterate x is read at each node before it is overwritten)
  else
    CK(sweep(kSweepSmooth, xa, nullptr, x, dk));
  return CSTG_OK;
}

// The learned cycle's fixed part on the finest level: x = two Chebyshev (or damped-Jacobi)
// pre-smoothing steps from x = 0, then the coarse correction x += P V(P'(b - A x)); the
// post-smoothing step is the network's (learned_api.cu). With a one-level hierarchy x is the
// dense solve.
int vcycle_pre(cstg_ctx* ctx, AmgData* d, const double* b, double* x, const int* skip) {
  if (d->nl == 1) return vcycle(ctx, d, 0, b, x, skip, nullptr);
  AmgLevel& lv = d->L[0];
  cudaStream_t s = ctx->stream;
  AmgLevel& nx = d->L[1];
  const MixedMatrix mm = mixed_view(ctx);
  const double* dinv = buf_ptr<double>(lv.dinv);
  const double* lam = buf_ptr<double>(lv.lam);
  double* r = buf_ptr<double>(lv.r);
  CK(amg_sweep_f32(skip, kSweepFirst, d->cheb, mm, dinv, lam, b, nullptr, nullptr, x, s));
  CK(amg_sweep_f32(skip, kSweepResidual, d->cheb, mm, dinv, lam, b, x, nullptr, r, s));
  CK(amg_restrict_f32(skip, lv.B, lv.nc, buf_ptr<int>(lv.pt_ptr), buf_ptr<int>(lv.pt_row), buf_ptr<float>(lv.pt32), r,
                      buf_ptr<double>(nx.bc), s));
  const int rc = vcycle(ctx, d, 1, buf_ptr<double>(nx.bc), buf_ptr<double>(nx.xb), skip, nullptr);
  if (rc) return rc;
  CK(amg_prolong_f32(skip, lv.B, lv.n, buf_ptr<int>(lv.p_ptr), buf_ptr<int>(lv.p_col), buf_ptr<float>(lv.p32),
                     buf_ptr<double>(nx.xb), x, s));
  return CSTG_OK;
}

}  // namespace

int cstg_host::amg_apply_pre(cstg_ctx* ctx, const double* b, double* x, const int* skip) {
  return vcycle_pre(ctx, ctx->amg, b, x, skip);
}

int cstg_host::amg_residual_fine(cstg_ctx* ctx, const double* b, const double* x, double* out, const int* skip) {
  AmgData* d = ctx->amg;
  AmgLevel& lv = d->L[0];
  const MixedMatrix mm = mixed_view(ctx);
  CK(amg_sweep_f32(skip, kSweepResidual, d->cheb, mm, buf_ptr<double>(lv.dinv), buf_ptr<double>(lv.lam), b, x, nullptr,
                   out, ctx->stream));
  return CSTG_OK;
}

double* cstg_host::amg_fine_scratch(cstg_ctx* ctx) { return buf_ptr<double>(ctx->amg->L[0].r); }

const double* cstg_host::amg_fine_lambda(cstg_ctx* ctx) { return buf_ptr<double>(ctx->amg->L[0].lam); }

unsigned long long cstg_host::amg_built_for(const cstg_ctx* ctx) { return ctx->amg ? ctx->amg->built_for : ~0ull; }

int cstg_host::amg_ready(cstg_ctx* ctx) {
  if (ctx->amg && ctx->amg->built_for == ctx->setup_count && ctx->mixed_ready) return CSTG_OK;
  if (ctx->kind != 1 || !ctx->setup_done)
    return fail(ctx, CSTG_ERR_STATE, "amg_setup: needs a mesh-pattern matrix after cstg_pcg_setup");
  const int rc = ensure_mixed(ctx);  // the finest-level smoother's FP32 operator
  if (rc) return rc;
  if (ctx->amg && ctx->amg->built_for == ctx->setup_count) return CSTG_OK;
  return amg_build(ctx);
}

int cstg_host::amg_levels(const cstg_ctx* ctx) { return ctx->amg ? ctx->amg->nl : 0; }

int cstg_host::amg_chebyshev(const cstg_ctx* ctx) { return ctx->amg ? ctx->amg->cheb : 1; }

unsigned long long cstg_host::amg_signature(const cstg_ctx* ctx) {
  // the launch shapes and scalar arguments a captured cycle depends on (buffer moves are
  // covered by the context's generation)
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&h](unsigned long long v) { h = (h ^ v) * 1099511628211ull; };
  const AmgData* d = ctx->amg;
  if (!d) return h;
  mix((unsigned long long)d->nl);
  mix((unsigned long long)d->n_coarse);
  mix((unsigned long long)d->tail_level);
  mix((unsigned long long)d->cheb);
  mix((unsigned long long)d->tail_cluster);
  for (int l = 0; l < d->nl; ++l) {
    mix((unsigned long long)d->L[l].B);
    mix((unsigned long long)d->L[l].n);
    mix((unsigned long long)d->L[l].nc);
  }
  return h;
}

int cstg_host::amg_apply(cstg_ctx* ctx, const double* r, double* z, const int* skip, const FcgDotSink* dots) {
  return vcycle(ctx, ctx->amg, 0, r, z, skip, ctx->amg->nl > 1 ? dots : nullptr);
}

extern "C" {

int cstg_amg_setup(cstg_ctx* ctx, cstg_amg_info* info) {
  BEGIN(ctx);
  if (ctx->amg) ctx->amg->built_for = ~0ull;  // rebuild
  const int rc = amg_ready(ctx);
  if (rc) return rc;
  if (info) {
    AmgData* d = ctx->amg;
    std::memset(info, 0, sizeof *info);
    info->levels = d->nl;
    for (int l = 0; l < info->levels && l < 16; ++l) info->dofs[l] = d->L[l].n * d->L[l].B;
    for (int l = 0; l < info->levels && l < 16; ++l) {
      const AmgLevel& lv = d->L[l];
      int nnzb = 0;
      CK(cudaMemcpy(&nnzb, lv.a_ptr + lv.n, sizeof(int), cudaMemcpyDeviceToHost));
      info->nnz[l] = (long long)nnzb * lv.B * lv.B;
    }
    info->setup_seconds = d->setup_seconds;
    info->tail_level = d->tail_level;
    info->tail_cluster = d->tail_level > 0 ? d->tail_cluster : 0;
  }
  return CSTG_OK;
}

int cstg_amg_set_smoother(cstg_ctx* ctx, int kind) {
  BEGIN(ctx);
  if (kind != CSTG_AMG_CHEBYSHEV && kind != CSTG_AMG_JACOBI)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "amg_set_smoother: unknown smoother %d", kind);
  if (!ctx->amg) {
    ctx->amg = new AmgData();
    ctx->amg->L.reserve(kMaxLevels + 1);
  }
  ctx->amg->cheb = kind == CSTG_AMG_CHEBYSHEV ? 1 : 0;
  if (ctx->amg->nl > 0) return setup_tail(ctx, ctx->amg);
  return CSTG_OK;
}

int cstg_amg_set_strength(cstg_ctx* ctx, double theta_fine, double theta_coarse) {
  BEGIN(ctx);
  if (!(theta_fine >= 0.0 && theta_fine < 1.0 && theta_coarse >= 0.0 && theta_coarse < 1.0))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "amg_set_strength: thresholds must lie in [0, 1), got %g, %g",
                theta_fine, theta_coarse);
  if (!ctx->amg) {
    ctx->amg = new AmgData();
    ctx->amg->L.reserve(kMaxLevels + 1);
  }
  AmgData* d = ctx->amg;
  if (d->theta_fine != theta_fine || d->theta_coarse != theta_coarse) d->built_for = ~0ull;  // rebuilt on next use
  d->theta_fine = theta_fine;
  d->theta_coarse = theta_coarse;
  return CSTG_OK;
}

int cstg_amg_set_tail(cstg_ctx* ctx, int enable) {
  BEGIN(ctx);
  if (!ctx->amg) {
    ctx->amg = new AmgData();
    ctx->amg->L.reserve(kMaxLevels + 1);
  }
  ctx->amg->tail_enabled = enable != 0;
  if (ctx->amg->nl > 0) return setup_tail(ctx, ctx->amg);
  return CSTG_OK;
}

int cstg_amg_time(cstg_ctx* ctx, int reps, double* out) {
  BEGIN(ctx);
  if (reps < 1 || !out) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "amg_time: bad arguments");
  const int rc = amg_ready(ctx);
  if (rc) return rc;
  AmgData* d = ctx->amg;
  AmgLevel& f = d->L[0];
  const size_t m = (size_t)f.n * f.B;
  double* b = buf_ptr<double>(f.bc);
  double* xa = buf_ptr<double>(f.xa);
  double* xb = buf_ptr<double>(f.xb);
  CK(cudaMemsetAsync(b, 0, sizeof(double) * m, ctx->stream));
  CK(cudaMemsetAsync(xa, 0, sizeof(double) * m, ctx->stream));
  const MixedMatrix mm = mixed_view(ctx);
  float ms = 0.f;
  for (int w = 0; w < 2; ++w) {  // warm-up, then timed
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int k = 0; k < reps; ++k)
      CK(amg_sweep_f32(nullptr, kSweepSmooth, d->cheb, mm, buf_ptr<double>(f.dinv), buf_ptr<double>(f.lam), b, k & 1 ? xb : xa, nullptr, k & 1 ? xa : xb,
                       ctx->stream));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
  }
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  out[0] = ms * 1e-3 / reps;
  // (the finest level's xa and r are the cycle's scratch; its xb and bc are free)
  for (int w = 0; w < 2; ++w) {
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int k = 0; k < reps; ++k) {
      const int rc2 = vcycle(ctx, d, 0, b, xb, nullptr, nullptr);
      if (rc2) return rc2;
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
  }
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  out[1] = ms * 1e-3 / reps;
  return CSTG_OK;
}

int cstg_amg_apply_device(cstg_ctx* ctx, const double* d_r, double* d_z) {
  BEGIN(ctx);
  const int rc = amg_ready(ctx);
  if (rc) return rc;
  const int rc2 = amg_apply(ctx, d_r, d_z, nullptr);
  if (rc2) return rc2;
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

}  // extern "C"
