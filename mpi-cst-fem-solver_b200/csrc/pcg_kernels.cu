// Jacobi-PCG kernels (FP64): SpMV with the fused p'Ap reduction, the x/r update with the
// fused r'r and r'z reductions, the p update, initialisation and the true residual.
//
// Reductions are deterministic: every kernel runs on a fixed grid (kReduceBlocks x kThreads)
// with a fixed work assignment; each block reduces with a fixed shuffle tree and writes one
// partial per quantity; the last block to finish (atomic ticket) sums the partials in index
// order and updates the CG scalars in PcgState. The recurrence is the reference's
// pcg_iterate (src/solver.cpp:35-105); only the summation order of the dot products differs.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

constexpr unsigned kFull = 0xffffffffu;

// Writes this block's NV partial sums; in the last block to arrive, tot[] receives the sums
// over all blocks (index order) and the function returns true.
template <int NV>
__device__ __forceinline__ bool last_block_reduce(const double (&v)[NV], double* partials,
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
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
      s += __ldcg(&partials[q * gridDim.x + i]);
    tot[q] = block_sum<kThreads>(s, sm);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

__device__ __forceinline__ int done_flag(const PcgState* st) {
  return __ldcg(&st->done);
}

// ---- SpMV, 2x2 node blocks ---------------------------------------------------------------
// A warp takes 4 nodes; 8 lanes per node, one 2x2 block per lane per step. Lane loads are
// double2 (16 B): the block's two row pairs and the x pair of its neighbour. Node n's values
// are one contiguous run (row 2n then row 2n+1), so a warp reads 4 adjacent runs.
template <bool PCG>
__global__ void __launch_bounds__(kThreads) k_spmv_block(BlockMatrix A, const double* __restrict__ x,
                                                         double* __restrict__ y, double* partials,
                                                         PcgState* st) {
  if (PCG && done_flag(st)) return;
  const int lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double2* __restrict__ x2 = reinterpret_cast<const double2*>(x);
  const double2* __restrict__ v2 = reinterpret_cast<const double2*>(A.vals);
  double dot = 0.0;
  for (int base = warp * 4; base < A.n_nodes; base += nwarps * 4) {
    const int n = base + sub;
    double ya = 0.0, yb = 0.0;
    if (n < A.n_nodes) {
      const int b0 = __ldg(&A.node_ptr[n]), deg = __ldg(&A.node_ptr[n + 1]) - b0;
      const double2* ra = v2 + 2L * b0;
      const double2* rb = ra + deg;
      for (int k = l8; k < deg; k += 8) {
        const int m = __ldg(&A.bnbr[b0 + k]);
        const double2 xv = x2[m];
        const double2 a = __ldcs(ra + k);
        const double2 c = __ldcs(rb + k);
        ya = fma(a.x, xv.x, ya);
        ya = fma(a.y, xv.y, ya);
        yb = fma(c.x, xv.x, yb);
        yb = fma(c.y, xv.y, yb);
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      ya += __shfl_xor_sync(kFull, ya, o);
      yb += __shfl_xor_sync(kFull, yb, o);
    }
    if (l8 == 0 && n < A.n_nodes) {
      reinterpret_cast<double2*>(y)[n] = make_double2(ya, yb);
      if (PCG) {
        const double2 pv = x2[n];
        dot = fma(pv.x, ya, dot);
        dot = fma(pv.y, yb, dot);
      }
    }
  }
  if (!PCG) return;
  const double v[1] = {dot};
  double tot[1];
  if (last_block_reduce<1>(v, partials, &st->ticket[0], tot) && threadIdx.x == 0) {
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

// ---- SpMV, scalar CSR (any matrix) ---------------------------------------------------------
// S lanes per row (a power of two picked from the mean row length).
template <int S, bool PCG>
__global__ void __launch_bounds__(kThreads) k_spmv_csr(CsrMatrixDev A, const double* __restrict__ x,
                                                       double* __restrict__ y, double* partials,
                                                       PcgState* st) {
  if (PCG && done_flag(st)) return;
  constexpr int R = 32 / S;
  const int lane = threadIdx.x & 31, g = lane / S, ls = lane % S;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int base = warp * R; base < A.n_rows; base += nwarps * R) {
    const int i = base + g;
    double s = 0.0;
    if (i < A.n_rows) {
      const int hi = __ldg(&A.row_ptr[i + 1]);
      for (int k = __ldg(&A.row_ptr[i]) + ls; k < hi; k += S)
        s = fma(__ldcs(&A.vals[k]), x[__ldg(&A.cols[k])], s);
    }
#pragma unroll
    for (int o = S / 2; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (ls == 0 && i < A.n_rows) {
      y[i] = s;
      if (PCG) dot = fma(x[i], s, dot);
    }
  }
  if (!PCG) return;
  const double v[1] = {dot};
  double tot[1];
  if (last_block_reduce<1>(v, partials, &st->ticket[0], tot) && threadIdx.x == 0) {
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

// ---- vector kernels -------------------------------------------------------------------------

// x = 0, r = b, p = z = D^-1 b, ||b||, r'z   (solver.cpp:42-58)
__global__ void __launch_bounds__(kThreads) k_init(int n, const double* __restrict__ b,
                                                   const double* __restrict__ invd,
                                                   double* __restrict__ x, double* __restrict__ r,
                                                   double* __restrict__ p, double* partials,
                                                   PcgState* st, double* history, double rtol,
                                                   int max_iter, int hist_on) {
  double bb = 0.0, rz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double bi = b[i], zi = invd[i] * bi;
    x[i] = 0.0;
    r[i] = bi;
    p[i] = zi;
    bb = fma(bi, bi, bb);
    rz = fma(bi, zi, rz);
  }
  const double v[2] = {bb, rz};
  double tot[2];
  if (last_block_reduce<2>(v, partials, &st->ticket[3], tot) && threadIdx.x == 0) {
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
    st->rr = tot[0];
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

// x += alpha p; r -= alpha Ap; z = D^-1 r; r'r, r'z; convergence test; beta (solver.cpp:72-96)
__global__ void __launch_bounds__(kThreads) k_update(int n, double* __restrict__ x,
                                                     double* __restrict__ r,
                                                     const double* __restrict__ p,
                                                     const double* __restrict__ Ap,
                                                     const double* __restrict__ invd,
                                                     double* partials, PcgState* st,
                                                     double* history) {
  if (done_flag(st)) return;
  const double alpha = __ldcg(&st->alpha);
  double rr = 0.0, rz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, Ap[i], r[i]);
    r[i] = ri;
    rr = fma(ri, ri, rr);
    rz = fma(ri, invd[i] * ri, rz);
  }
  const double v[2] = {rr, rz};
  double tot[2];
  if (last_block_reduce<2>(v, partials, &st->ticket[1], tot) && threadIdx.x == 0) {
    const int it = st->iter + 1;
    st->iter = it;
    const double rel = sqrt(tot[0]) / st->bnorm;
    st->rel = rel;
    st->rr = tot[0];
    if (st->hist_on) history[it] = rel;
    if (rel < st->rtol)
      st->done = CSTG_SOLVE_CONVERGED + 1;
    else if (it >= st->max_iter)
      st->done = CSTG_SOLVE_MAX_ITER + 1;
    st->beta = tot[1] / st->rz;
    st->rz = tot[1];
  }
}

// p = D^-1 r + beta p
__global__ void __launch_bounds__(kThreads) k_pupdate(int n, const double* __restrict__ r,
                                                      const double* __restrict__ invd,
                                                      double* __restrict__ p, PcgState* st) {
  if (done_flag(st)) return;
  const double beta = __ldcg(&st->beta);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = fma(beta, p[i], invd[i] * r[i]);
}

// r_true = b - A x (A x given in `ax`); ||r_true|| / ||b|| -> st->true_rel (solver.cpp:117-122).
// With `restart` the iteration may continue from x: r = r_true, p = D^-1 r, r'z, and when
// the true residual is still >= rtol the solve is re-opened (done = 0).
__global__ void __launch_bounds__(kThreads) k_true_residual(int n, const double* __restrict__ b,
                                                            const double* __restrict__ ax,
                                                            const double* __restrict__ invd,
                                                            double* __restrict__ r,
                                                            double* __restrict__ p,
                                                            double* partials, PcgState* st,
                                                            int restart, int max_replacements) {
  double rr = 0.0, rz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = b[i] - ax[i];
    rr = fma(ri, ri, rr);
    if (restart) {
      const double zi = invd[i] * ri;
      r[i] = ri;
      p[i] = zi;
      rz = fma(ri, zi, rz);
    }
  }
  const double v[2] = {rr, rz};
  double tot[2];
  if (last_block_reduce<2>(v, partials, &st->ticket[2], tot) && threadIdx.x == 0) {
    const double bn = st->bnorm;
    const double tr = bn > 0.0 ? sqrt(tot[0]) / bn : 0.0;
    st->true_rel = tr;
    if (restart && st->done == CSTG_SOLVE_CONVERGED + 1 && !(tr < st->rtol) &&
        st->replace_count < max_replacements && st->iter < st->max_iter) {
      st->replace_count += 1;
      st->rz = tot[1];
      st->rr = tot[0];
      st->rel = tr;
      st->done = 0;
    }
  }
}

// ---- launchers --------------------------------------------------------------------------------

template <bool PCG>
static void spmv_dispatch(const BlockMatrix* bm, const CsrMatrixDev* cm, const double* x, double* y,
                          double* partials, PcgState* st, cudaStream_t s) {
  count_launches(1);
  if (bm) {
    k_spmv_block<PCG><<<kReduceBlocks, kThreads, 0, s>>>(*bm, x, y, partials, st);
    return;
  }
  switch (cm->sub) {
    case 1: k_spmv_csr<1, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 2: k_spmv_csr<2, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 4: k_spmv_csr<4, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 8: k_spmv_csr<8, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 16: k_spmv_csr<16, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    default: k_spmv_csr<32, PCG><<<kReduceBlocks, kThreads, 0, s>>>(*cm, x, y, partials, st); break;
  }
}

cudaError_t launch_pcg_init(const PcgBuffers& w, double rtol, int max_iter, bool hist,
                            cudaStream_t s) {
  k_init<<<kReduceBlocks, kThreads, 0, s>>>(w.n, w.b, w.inv_diag, w.x, w.r, w.p, w.partials, w.st,
                                            w.history, rtol, max_iter, hist ? 1 : 0);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_pcg_iteration(const PcgBuffers& w, const BlockMatrix* bm,
                                 const CsrMatrixDev* cm, cudaStream_t s) {
  spmv_dispatch<true>(bm, cm, w.p, w.Ap, w.partials, w.st, s);
  k_update<<<kReduceBlocks, kThreads, 0, s>>>(w.n, w.x, w.r, w.p, w.Ap, w.inv_diag, w.partials,
                                              w.st, w.history);
  k_pupdate<<<kReduceBlocks, kThreads, 0, s>>>(w.n, w.r, w.inv_diag, w.p, w.st);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_spmv(const BlockMatrix* bm, const CsrMatrixDev* cm, const double* x, double* y,
                        cudaStream_t s) {
  spmv_dispatch<false>(bm, cm, x, y, nullptr, nullptr, s);
  return cudaGetLastError();
}

cudaError_t launch_true_residual(const PcgBuffers& w, bool restart, int max_replacements,
                                 cudaStream_t s) {
  k_true_residual<<<kReduceBlocks, kThreads, 0, s>>>(w.n, w.b, w.Ap, w.inv_diag, w.r, w.p,
                                                     w.partials, w.st, restart ? 1 : 0,
                                                     max_replacements);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
