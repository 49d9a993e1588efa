// Mixed-precision Jacobi-PCG: FP32 SpMV operator with FP64 accumulation, FP64 vectors and
// scalars, FP64 true-residual replacement (reliable updates).
//
// FP32 operator in difference form. With S_n = sum over node n's block row of the 2x2 blocks
// (an FP64 sum, kept in FP64), the eliminated stiffness matrix acts as
//     (K x)_n = sum_{m != n} K_nm (x_m - x_n) + S_n x_n .
// Only the off-diagonal blocks are stored in FP32 (float4 a00 a01 a10 a11, block-major, with
// their neighbour node). Rounding K_nm to FP32 then perturbs K x by ~eps32 |K_nm| |x_m - x_n|,
// i.e. in proportion to the local variation of x instead of |x|: rigid translations (zero row
// sums of the unconstrained K) stay exact and the smooth low-eigenvalue modes that govern CG's
// convergence are barely disturbed. S_n stays FP64 because next to Dirichlet DOFs it is of the
// size of K itself. Measured on these plates: an all-FP32 matrix costs ~30 % more
// iterations; the difference form with FP64 vectors costs < 1 %. The vectors stay FP64: an
// FP32 search direction rounds p_m and p_n separately, so p_m - p_n carries eps32 |p| noise and
// the difference form loses its advantage (the iteration diverged at 2M DOFs that way).
//
// Reliable updates (van der Vorst & Ye): when the recursive residual has dropped below delta
// times its largest value since the last update, or meets rtol, or a cycle exceeds
// kReplaceCycleLimit iterations, r is replaced by the FP64 residual b - A x computed with the
// FP64 matrix; the solve stops only when that FP64 true residual is below rtol. The search
// direction is kept across replacements.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {
constexpr unsigned kFull = 0xffffffffu;

// A reliable update is forced after this many iterations even if the recursive residual has
// not dropped by delta (one FP64 SpMV per 1000 iterations).
constexpr int kReplaceCycleLimit = 1000;

template <int NV>
__device__ __forceinline__ bool last_block_reduce_m(const double (&v)[NV], double* partials,
                                                    unsigned int* ticket, double (&tot)[NV]) {
  __shared__ double sm[kWarps];
  __shared__ bool am_last;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double s = block_sum<kThreads>(v[q], sm);
    if (threadIdx.x == 0) partials[q * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(&partials[q * gridDim.x + i]);
    tot[q] = block_sum<kThreads>(s, sm);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

template <auto KERNEL>
int wave_grid_m() {
  static int cache[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!cache[dev]) {
    int sms = kSMs, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, KERNEL, kThreads, 0);
    cache[dev] = std::min(kMaxGrid, std::max(1, sms * std::max(per, 1)));
  }
  return cache[dev];
}

__device__ __forceinline__ const double2& ld2(const double* a, int i) {
  return reinterpret_cast<const double2*>(a)[i];
}
__device__ __forceinline__ double2& st2(double* a, int i) { return reinterpret_cast<double2*>(a)[i]; }
}  // namespace

// ---- conversion: FP64 node runs -> FP32 off-diagonal blocks + FP64 S -------------------------
// One thread per node. Node n's off-diagonal blocks start at node_ptr[n] - n: every node has
// exactly one self block.
__global__ void k_make_mixed(int N, const int* __restrict__ node_ptr, const int* __restrict__ bnbr,
                             const double* __restrict__ vals, float4* __restrict__ val32,
                             int* __restrict__ nbr32, double2* __restrict__ S64) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int b0 = node_ptr[n], deg = node_ptr[n + 1] - b0;
  const double* ra = vals + 4L * b0;
  const double* rb = ra + 2 * deg;
  double s00 = 0.0, s01 = 0.0, s10 = 0.0, s11 = 0.0;
  int o = b0 - n;
  for (int k = 0; k < deg; ++k) {
    const double a00 = ra[2 * k], a01 = ra[2 * k + 1], a10 = rb[2 * k], a11 = rb[2 * k + 1];
    s00 += a00;
    s01 += a01;
    s10 += a10;
    s11 += a11;
    const int m = bnbr[b0 + k];
    if (m != n) {
      val32[o] = make_float4((float)a00, (float)a01, (float)a10, (float)a11);
      nbr32[o] = m;
      ++o;
    }
  }
  S64[2 * n] = make_double2(s00, s01);
  S64[2 * n + 1] = make_double2(s10, s11);
}

// ---- FP32-matrix difference-form SpMV on FP64 vectors (+ p'Ap) -------------------------------
// FP64 block SpMV of node groups (the FP64 path's loop) for the solve's last stretch after a
// precision switch; returns this thread's share of p'Ap.
__device__ __forceinline__ double spmv64_groups(const BlockMatrix& A, const double* __restrict__ x,
                                                double* __restrict__ y) {
  const int lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double2* __restrict__ x2 = reinterpret_cast<const double2*>(x);
  const double2* __restrict__ v2 = reinterpret_cast<const double2*>(A.vals);
  const int N = A.n_nodes;
  double dot = 0.0;
  for (int base = warp * 4; base < N; base += nwarps * 4) {
    const int n = base + sub;
    double ya = 0.0, yb = 0.0;
    if (n < N) {
      const int b0 = __ldg(&A.node_ptr[n]), deg = __ldg(&A.node_ptr[n + 1]) - b0;
      for (int k = l8; k < deg; k += 8) {
        const int m = __ldg(&A.bnbr[b0 + k]);
        const double2 xv = x2[m];
        const double2 a = __ldcs(v2 + 2L * b0 + k), c = __ldcs(v2 + 2L * b0 + deg + k);
        ya = fma(a.x, xv.x, fma(a.y, xv.y, ya));
        yb = fma(c.x, xv.x, fma(c.y, xv.y, yb));
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      ya += __shfl_xor_sync(kFull, ya, o);
      yb += __shfl_xor_sync(kFull, yb, o);
    }
    if (l8 == 0 && n < N) {
      st2(y, n) = make_double2(ya, yb);
      const double2 pv = x2[n];
      dot = fma(pv.x, ya, fma(pv.y, yb, dot));
    }
  }
  return dot;
}

// One thread per node: the node's off-diagonal blocks are one contiguous run of float4s, so a
// warp reads 32 adjacent runs (~3 KB) through L1, and each thread keeps its six or so block
// loads and x gathers in flight independently. (For FP32 blocks this beats the lane-per-block
// split of the FP64 kernel, which is latency-bound at half the bytes per lane.)
template <bool PCG>
__global__ void __launch_bounds__(kThreads) k_spmv_mixed(MixedMatrix A, BlockMatrix A64,
                                                         const double* __restrict__ x,
                                                         double* __restrict__ y, double* partials,
                                                         PcgState* st) {
  if (PCG && __ldcg(&st->done)) return;
  const double2* __restrict__ x2 = reinterpret_cast<const double2*>(x);
  int N = A.n_nodes;
  double dot = 0.0;
  if (PCG && __ldcg(&st->fp64_mode)) {
    dot = spmv64_groups(A64, x, y);
    N = 0;  // skip the FP32 loop below
  }
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const int b = __ldg(&A.node_ptr[n]);
    const int o = b - n, c = __ldg(&A.node_ptr[n + 1]) - b - 1;
    const double2 xs = x2[n];
    double ya = 0.0, yb = 0.0;
    for (int k = 0; k < c; ++k) {
      const int m = __ldg(&A.nbr32[o + k]);
      const float4 a = __ldg(&A.val32[o + k]);
      const double2 xm = x2[m];
      const double dx = xm.x - xs.x, dy = xm.y - xs.y;
      ya = fma((double)a.x, dx, fma((double)a.y, dy, ya));
      yb = fma((double)a.z, dx, fma((double)a.w, dy, yb));
    }
    const double2 sa = __ldg(&A.S64[2 * n]), sb = __ldg(&A.S64[2 * n + 1]);
    ya = fma(sa.x, xs.x, fma(sa.y, xs.y, ya));
    yb = fma(sb.x, xs.x, fma(sb.y, xs.y, yb));
    st2(y, n) = make_double2(ya, yb);
    if (PCG) dot = fma(xs.x, ya, fma(xs.y, yb, dot));
  }
  if (!PCG) return;
  const double v[1] = {dot};
  double tot[1];
  if (last_block_reduce_m<1>(v, partials, &st->ticket[0], tot) && threadIdx.x == 0) {
    const double pAp = tot[0];
    st->pAp = pAp;
    if (!(pAp > 0.0)) {
      st->alpha = 0.0;
      st->done = CSTG_SOLVE_BREAKDOWN + 1;
    } else {
      st->alpha = st->rz / pAp;
    }
  }
}

// ---- vector kernels (pairs of DOFs = one node; n is even on the mesh path) -------------------

// x = 0, r = b, p = D^-1 b, ||b||, r'z (solver.cpp:42-58) and the reliable-update state
__global__ void __launch_bounds__(kThreads) k_init_mixed(int N, const double* __restrict__ b,
                                                         const double* __restrict__ invd,
                                                         double* __restrict__ x, double* __restrict__ r,
                                                         double* __restrict__ p, double* partials,
                                                         PcgState* st, double* history, double rtol,
                                                         int max_iter, int hist_on, double delta) {
  double bb = 0.0, rz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double2 bi = ld2(b, i), di = ld2(invd, i);
    st2(x, i) = make_double2(0.0, 0.0);
    st2(r, i) = bi;
    st2(p, i) = make_double2(di.x * bi.x, di.y * bi.y);
    bb = fma(bi.x, bi.x, fma(bi.y, bi.y, bb));
    rz = fma(bi.x, di.x * bi.x, fma(bi.y, di.y * bi.y, rz));
  }
  const double v[2] = {bb, rz};
  double tot[2];
  if (last_block_reduce_m<2>(v, partials, &st->ticket[3], tot) && threadIdx.x == 0) {
    const double bnorm = sqrt(tot[0]);
    st->bnorm = bnorm;
    st->rtol = rtol;
    st->max_iter = max_iter;
    st->hist_on = hist_on;
    st->iter = 0;
    st->alpha = st->beta = 0.0;
    st->pAp = 0.0;
    st->true_rel = 0.0;
    st->replace_count = 0;
    st->restart_pending = 0;
    st->final_checks = 0;
    st->rr = tot[0];
    st->rmax = bnorm;
    st->delta = delta;
    st->rz_prev = 0.0;
    st->last_replace = 0;
    st->cycle_limit = kReplaceCycleLimit;
    st->fp64_mode = 0;
    st->fp64_switch_iter = 0;
    st->stall_cycles = 0;
    st->best_true = 1.0;
    if (bnorm == 0.0) {
      st->rel = 0.0;
      st->rz = 0.0;
      st->done = CSTG_SOLVE_ZERO_RHS + 1;
      if (hist_on) history[0] = 0.0;
    } else {
      st->rel = 1.0;
      st->rz = tot[1];
      st->done = max_iter <= 0 ? CSTG_SOLVE_MAX_ITER + 1 : 0;
      if (hist_on) history[0] = 1.0;
    }
  }
}

// x += alpha p; r -= alpha Ap; r'r, r'D^-1 r; decide on a reliable update; beta
__global__ void __launch_bounds__(kThreads) k_update_mixed(int N, double* __restrict__ x,
                                                           double* __restrict__ r,
                                                           const double* __restrict__ p,
                                                           const double* __restrict__ Ap,
                                                           const double* __restrict__ invd,
                                                           double* partials, PcgState* st,
                                                           double* history) {
  if (__ldcg(&st->done)) return;
  const double alpha = __ldcg(&st->alpha);
  double rr = 0.0, rz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double2 pi = ld2(p, i), ai = ld2(Ap, i), di = ld2(invd, i);
    double2 xi = ld2(x, i), ri = ld2(r, i);
    xi.x = fma(alpha, pi.x, xi.x);
    xi.y = fma(alpha, pi.y, xi.y);
    ri.x = fma(-alpha, ai.x, ri.x);
    ri.y = fma(-alpha, ai.y, ri.y);
    st2(x, i) = xi;
    st2(r, i) = ri;
    rr = fma(ri.x, ri.x, fma(ri.y, ri.y, rr));
    rz = fma(ri.x, di.x * ri.x, fma(ri.y, di.y * ri.y, rz));
  }
  const double v[2] = {rr, rz};
  double tot[2];
  if (last_block_reduce_m<2>(v, partials, &st->ticket[1], tot) && threadIdx.x == 0) {
    const int it = st->iter + 1;
    st->iter = it;
    const double rn = sqrt(tot[0]);
    const double rel = rn / st->bnorm;
    st->rel = rel;
    st->rr = tot[0];
    if (st->hist_on) history[it] = rel;
    st->rmax = fmax(st->rmax, rn);
    if (rel < st->rtol)
      st->restart_pending = 2;  // confirm on the FP64 true residual
    else if (!st->fp64_mode && rn < st->delta * st->rmax)
      st->restart_pending = 1;  // reliable update
    else if (!st->fp64_mode && it - st->last_replace >= st->cycle_limit)
      st->restart_pending = 3;  // a long cycle: replace anyway (bounds the FP32 operator's drift)
    // (after the switch to FP64 the iteration is plain FP64 CG: replacements at its accuracy
    // limit break the conjugacy of p and made the recursion drift from x, measured at 8M DOFs)
    else if (it >= st->max_iter)
      st->done = CSTG_SOLVE_MAX_ITER + 1;
    st->rz_prev = st->rz;
    st->beta = tot[1] / st->rz;
    st->rz = tot[1];
  }
}

// Reliable update: r = b - A x with the FP64 matrix (block SpMV of x fused with the residual),
// r'r and r'D^-1 r. Runs only when k_update_mixed asked for it.
__global__ void __launch_bounds__(kThreads) k_replace_mixed(BlockMatrix A, const double* __restrict__ x,
                                                            const double* __restrict__ b,
                                                            const double* __restrict__ invd,
                                                            double* __restrict__ r, double* partials,
                                                            PcgState* st, double* history,
                                                            int max_final_checks) {
  if (__ldcg(&st->done) || !__ldcg(&st->restart_pending)) return;
  const int lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double2* __restrict__ x2 = reinterpret_cast<const double2*>(x);
  const double2* __restrict__ v2 = reinterpret_cast<const double2*>(A.vals);
  const int N = A.n_nodes;
  double rr = 0.0, rz = 0.0;
  for (int base = warp * 4; base < N; base += nwarps * 4) {
    const int n = base + sub;
    double ya = 0.0, yb = 0.0;
    if (n < N) {
      const int b0 = __ldg(&A.node_ptr[n]), deg = __ldg(&A.node_ptr[n + 1]) - b0;
      for (int k = l8; k < deg; k += 8) {
        const int m = __ldg(&A.bnbr[b0 + k]);
        const double2 xv = x2[m];
        const double2 a = v2[2L * b0 + k], c = v2[2L * b0 + deg + k];
        ya = fma(a.x, xv.x, fma(a.y, xv.y, ya));
        yb = fma(c.x, xv.x, fma(c.y, xv.y, yb));
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      ya += __shfl_xor_sync(kFull, ya, o);
      yb += __shfl_xor_sync(kFull, yb, o);
    }
    if (l8 == 0 && n < N) {
      const double2 bv = ld2(b, n), dv = ld2(invd, n);
      const double rx = bv.x - ya, ry = bv.y - yb;
      st2(r, n) = make_double2(rx, ry);
      rr = fma(rx, rx, fma(ry, ry, rr));
      rz = fma(rx, dv.x * rx, fma(ry, dv.y * ry, rz));
    }
  }
  const double v[2] = {rr, rz};
  double tot[2];
  if (last_block_reduce_m<2>(v, partials, &st->ticket[4], tot) && threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    const double tr = rn / st->bnorm;
    const int kind = st->restart_pending;
    const double rec = st->rel;  // the recursive residual this replacement corrects
    st->true_rel = tr;
    st->rel = tr;
    st->rr = tot[0];
    st->rmax = rn;
    st->replace_count += 1;
    st->last_replace = st->iter;
    if (st->hist_on) history[st->iter] = tr;
    // the search direction is kept (a restart would throw away the Krylov information)
    st->beta = st->rz_prev > 0.0 ? tot[1] / st->rz_prev : 0.0;
    st->rz = tot[1];
    st->restart_pending = 0;
    if (tr < st->rtol) {
      st->done = CSTG_SOLVE_CONVERGED + 1;
    } else {
      // Precision switch: the recursive residual met rtol but the FP64 true residual did not
      // (or a delta cycle did not halve the true residual, or, below kStallGate, two forced
      // replacements in a row found it no lower than 0.9 of its best or above kGapRatio times the
      // recursive residual it replaced — the FP32 recursion still converges while the true
      // residual does not; above kStallGate such cycles are the early rise of the CG residual):
      // the FP32 operator has reached its accuracy floor, so the remaining iterations use the
      // FP64 matrix.
      if (kind == 3)
        st->stall_cycles = ((tr > 0.9 * st->best_true || tr > kGapRatio * rec) && st->best_true < kStallGate)
                               ? st->stall_cycles + 1
                               : 0;
      if (!st->fp64_mode && (kind == 2 || (kind == 1 && tr > 0.5 * st->best_true) ||
                                (kind == 3 && st->stall_cycles >= 2))) {
        st->fp64_mode = 1;
        st->fp64_switch_iter = st->iter;
        st->beta = 0.0;  // restart the direction: p = D^-1 r, plain FP64 CG from here
      } else if (st->fp64_mode) {
        st->beta = 0.0;  // an FP64 confirmation that missed: restart from the true residual
      }
      if (kind == 2 && ++st->final_checks > max_final_checks) st->done = CSTG_SOLVE_CONVERGED + 1;
      if (st->iter >= st->max_iter) st->done = CSTG_SOLVE_MAX_ITER + 1;
    }
    st->best_true = fmin(st->best_true, tr);
  }
}

// p = D^-1 r + beta p
__global__ void __launch_bounds__(kThreads) k_pupdate_mixed(int N, const double* __restrict__ r,
                                                            const double* __restrict__ invd,
                                                            double* __restrict__ p, PcgState* st) {
  if (__ldcg(&st->done)) return;
  const double beta = __ldcg(&st->beta);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double2 ri = ld2(r, i), di = ld2(invd, i);
    double2 pi = ld2(p, i);
    pi.x = fma(beta, pi.x, di.x * ri.x);
    pi.y = fma(beta, pi.y, di.y * ri.y);
    st2(p, i) = pi;
  }
}

// ---- launchers -----------------------------------------------------------------------------

cudaError_t launch_make_mixed(int N, const int* node_ptr, const int* bnbr, const double* vals,
                              float4* val32, int* nbr32, double2* S64, cudaStream_t s) {
  if (N) {
    k_make_mixed<<<(N + 127) / 128, 128, 0, s>>>(N, node_ptr, bnbr, vals, val32, nbr32, S64);
    count_launches(1);
  }
  return cudaGetLastError();
}

cudaError_t launch_mixed_init(const MixedBuffers& w, double rtol, int max_iter, bool hist, double delta,
                              cudaStream_t s) {
  k_init_mixed<<<wave_grid_m<k_init_mixed>(), kThreads, 0, s>>>(w.n_nodes, w.b, w.inv_diag, w.x, w.r, w.p,
                                                                w.partials, w.st, w.history, rtol, max_iter,
                                                                hist ? 1 : 0, delta);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mixed_iteration(const MixedBuffers& w, const MixedMatrix& A32, const BlockMatrix& A64,
                                   int max_final_checks, cudaStream_t s) {
  k_spmv_mixed<true><<<wave_grid_m<k_spmv_mixed<true>>(), kThreads, 0, s>>>(A32, A64, w.p, w.Ap, w.partials,
                                                                          w.st);
  k_update_mixed<<<wave_grid_m<k_update_mixed>(), kThreads, 0, s>>>(w.n_nodes, w.x, w.r, w.p, w.Ap, w.inv_diag,
                                                                    w.partials, w.st, w.history);
  k_replace_mixed<<<wave_grid_m<k_replace_mixed>(), kThreads, 0, s>>>(A64, w.x, w.b, w.inv_diag, w.r,
                                                                      w.partials, w.st, w.history,
                                                                      max_final_checks);
  k_pupdate_mixed<<<wave_grid_m<k_pupdate_mixed>(), kThreads, 0, s>>>(w.n_nodes, w.r, w.inv_diag, w.p, w.st);
  count_launches(4);
  return cudaGetLastError();
}

cudaError_t launch_spmv_mixed_pcg(const MixedMatrix& A32, const BlockMatrix& A64, const double* p, double* q,
                                  double* partials, PcgState* st, cudaStream_t s) {
  k_spmv_mixed<true><<<wave_grid_m<k_spmv_mixed<true>>(), kThreads, 0, s>>>(A32, A64, p, q, partials, st);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_spmv_mixed(const MixedMatrix& A32, const double* x, double* y, cudaStream_t s) {
  k_spmv_mixed<false><<<wave_grid_m<k_spmv_mixed<false>>(), kThreads, 0, s>>>(A32, BlockMatrix{}, x, y, nullptr,
                                                                            nullptr);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
