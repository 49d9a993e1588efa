// Jacobi-PCG kernels (FP64): SpMV with the fused p'Ap reduction, the x/r update with the
// fused r'r and r'z reductions, the p update, initialisation and the true residual.
//
// Reductions are deterministic: every kernel runs on a fixed one-wave grid (SMs x resident
// blocks of kThreads, from the occupancy calculator) with a fixed work assignment; each block reduces with a fixed shuffle tree and writes one
// partial per quantity; the last block to finish (atomic ticket) sums the partials in index
// order and updates the CG scalars in PcgState. The recurrence is the reference's
// pcg_iterate (src/solver.cpp:35-105); only the summation order of the dot products differs.
#include <cuda_runtime.h>

#include <algorithm>

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
// Node n's two rows are one contiguous run: row 2n's deg(n) double2 pairs, then row 2n+1's.
// 8 lanes per node, one 2x2 block per lane per step: the lane loads the block's two 16-byte
// row pairs, its neighbour from bnbr and that neighbour's 16-byte x pair. The SpMV is
// latency-bound on the chain node_ptr -> bnbr -> x, so a warp works on two groups of four
// nodes at once (eight nodes per iteration): both groups' loads are issued before either is
// used, which doubles the loads in flight per warp. The grid is one wave (SMs x resident
// blocks per SM, from the occupancy calculator).
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
  const int N = A.n_nodes;
  double dot = 0.0;
  for (int base = warp * 8; base < N; base += nwarps * 8) {
    const int n0 = base + sub, n1 = base + 4 + sub;
    int b00 = 0, d0 = 0, b01 = 0, d1 = 0;
    if (n0 < N) {
      b00 = __ldg(&A.node_ptr[n0]);
      d0 = __ldg(&A.node_ptr[n0 + 1]) - b00;
    }
    if (n1 < N) {
      b01 = __ldg(&A.node_ptr[n1]);
      d1 = __ldg(&A.node_ptr[n1 + 1]) - b01;
    }
    double ya0 = 0.0, yb0 = 0.0, ya1 = 0.0, yb1 = 0.0;
    const int dmax = max(d0, d1);
    for (int k = l8; k < dmax; k += 8) {
      const bool ok0 = k < d0, ok1 = k < d1;
      const int m0 = ok0 ? __ldg(&A.bnbr[b00 + k]) : 0;
      const int m1 = ok1 ? __ldg(&A.bnbr[b01 + k]) : 0;
      double2 a0 = make_double2(0.0, 0.0), c0 = a0, a1 = a0, c1 = a0;
      if (ok0) {
        a0 = __ldcs(v2 + 2L * b00 + k);
        c0 = __ldcs(v2 + 2L * b00 + d0 + k);
      }
      if (ok1) {
        a1 = __ldcs(v2 + 2L * b01 + k);
        c1 = __ldcs(v2 + 2L * b01 + d1 + k);
      }
      const double2 x0 = x2[m0], x1 = x2[m1];
      ya0 = fma(a0.x, x0.x, fma(a0.y, x0.y, ya0));
      yb0 = fma(c0.x, x0.x, fma(c0.y, x0.y, yb0));
      ya1 = fma(a1.x, x1.x, fma(a1.y, x1.y, ya1));
      yb1 = fma(c1.x, x1.x, fma(c1.y, x1.y, yb1));
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      ya0 += __shfl_xor_sync(kFull, ya0, o);
      yb0 += __shfl_xor_sync(kFull, yb0, o);
      ya1 += __shfl_xor_sync(kFull, ya1, o);
      yb1 += __shfl_xor_sync(kFull, yb1, o);
    }
    if (l8 == 0) {
      if (n0 < N) {
        reinterpret_cast<double2*>(y)[n0] = make_double2(ya0, yb0);
        if (PCG) {
          const double2 pv = x2[n0];
          dot = fma(pv.x, ya0, dot);
          dot = fma(pv.y, yb0, dot);
        }
      }
      if (n1 < N) {
        reinterpret_cast<double2*>(y)[n1] = make_double2(ya1, yb1);
        if (PCG) {
          const double2 pv = x2[n1];
          dot = fma(pv.x, ya1, dot);
          dot = fma(pv.y, yb1, dot);
        }
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
// DOFs are processed in 16-byte pairs (grid-stride over pairs); an odd last DOF is handled by
// thread 0 of block 0, so the work assignment (and the reduction order) is fixed.

__device__ __forceinline__ const double2& L2(const double* a, int i) {
  return reinterpret_cast<const double2*>(a)[i];
}
__device__ __forceinline__ double2& S2(double* a, int i) { return reinterpret_cast<double2*>(a)[i]; }
__device__ __forceinline__ bool tail_thread(int n) {
  return (n & 1) && blockIdx.x == 0 && threadIdx.x == 0;
}

// x = 0, r = b, p = z = D^-1 b, ||b||, r'z   (solver.cpp:42-58)
__global__ void __launch_bounds__(kThreads) k_init(int n, const double* __restrict__ b,
                                                   const double* __restrict__ invd,
                                                   double* __restrict__ x, double* __restrict__ r,
                                                   double* __restrict__ p, double* partials,
                                                   PcgState* st, double* history, double rtol,
                                                   int max_iter, int hist_on) {
  double bb = 0.0, rz = 0.0;
  const int np = n >> 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const double2 bi = L2(b, i), di = L2(invd, i);
    const double2 zi = make_double2(di.x * bi.x, di.y * bi.y);
    S2(x, i) = make_double2(0.0, 0.0);
    S2(r, i) = bi;
    S2(p, i) = zi;
    bb = fma(bi.x, bi.x, bb);
    bb = fma(bi.y, bi.y, bb);
    rz = fma(bi.x, zi.x, rz);
    rz = fma(bi.y, zi.y, rz);
  }
  if (tail_thread(n)) {
    const int i = n - 1;
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
  const int np = n >> 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const double2 pi = L2(p, i), ai = L2(Ap, i), di = L2(invd, i);
    double2 xi = L2(x, i), ri = L2(r, i);
    xi.x = fma(alpha, pi.x, xi.x);
    xi.y = fma(alpha, pi.y, xi.y);
    ri.x = fma(-alpha, ai.x, ri.x);
    ri.y = fma(-alpha, ai.y, ri.y);
    S2(x, i) = xi;
    S2(r, i) = ri;
    rr = fma(ri.x, ri.x, rr);
    rr = fma(ri.y, ri.y, rr);
    rz = fma(ri.x, di.x * ri.x, rz);
    rz = fma(ri.y, di.y * ri.y, rz);
  }
  if (tail_thread(n)) {
    const int i = n - 1;
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
  const int np = n >> 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const double2 ri = L2(r, i), di = L2(invd, i);
    double2 pi = L2(p, i);
    pi.x = fma(beta, pi.x, di.x * ri.x);
    pi.y = fma(beta, pi.y, di.y * ri.y);
    S2(p, i) = pi;
  }
  if (tail_thread(n)) p[n - 1] = fma(beta, p[n - 1], invd[n - 1] * r[n - 1]);
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

// One full wave of `kernel` on the current device: SMs x resident blocks per SM at kThreads
// threads, capped at kMaxGrid. Cached per device; the same binary on the same GPU always
// gets the same grid, so the reductions keep their order.
template <auto KERNEL>
static int wave_grid() {
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

template <bool PCG>
static void spmv_dispatch(const BlockMatrix* bm, const CsrMatrixDev* cm, const double* x, double* y,
                          double* partials, PcgState* st, cudaStream_t s) {
  count_launches(1);
  if (bm) {
    k_spmv_block<PCG><<<wave_grid<k_spmv_block<PCG>>(), kThreads, 0, s>>>(*bm, x, y, partials, st);
    return;
  }
  switch (cm->sub) {
    case 1: k_spmv_csr<1, PCG><<<wave_grid<k_spmv_csr<1, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 2: k_spmv_csr<2, PCG><<<wave_grid<k_spmv_csr<2, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 4: k_spmv_csr<4, PCG><<<wave_grid<k_spmv_csr<4, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 8: k_spmv_csr<8, PCG><<<wave_grid<k_spmv_csr<8, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    case 16: k_spmv_csr<16, PCG><<<wave_grid<k_spmv_csr<16, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
    default: k_spmv_csr<32, PCG><<<wave_grid<k_spmv_csr<32, PCG>>(), kThreads, 0, s>>>(*cm, x, y, partials, st); break;
  }
}

cudaError_t launch_pcg_init(const PcgBuffers& w, double rtol, int max_iter, bool hist,
                            cudaStream_t s) {
  k_init<<<wave_grid<k_init>(), kThreads, 0, s>>>(w.n, w.b, w.inv_diag, w.x, w.r, w.p, w.partials, w.st,
                                            w.history, rtol, max_iter, hist ? 1 : 0);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_pcg_iteration(const PcgBuffers& w, const BlockMatrix* bm,
                                 const CsrMatrixDev* cm, cudaStream_t s) {
  spmv_dispatch<true>(bm, cm, w.p, w.Ap, w.partials, w.st, s);
  k_update<<<wave_grid<k_update>(), kThreads, 0, s>>>(w.n, w.x, w.r, w.p, w.Ap, w.inv_diag, w.partials,
                                              w.st, w.history);
  k_pupdate<<<wave_grid<k_pupdate>(), kThreads, 0, s>>>(w.n, w.r, w.inv_diag, w.p, w.st);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t kernel_binary_version(int* version) {
  cudaFuncAttributes attr{};
  const cudaError_t e = cudaFuncGetAttributes(&attr, k_pupdate);
  if (e == cudaSuccess) *version = attr.binaryVersion;
  return e;
}

cudaError_t launch_spmv_phase(const PcgBuffers& w, const BlockMatrix* bm, const CsrMatrixDev* cm, cudaStream_t s) {
  spmv_dispatch<true>(bm, cm, w.p, w.Ap, w.partials, w.st, s);
  return cudaGetLastError();
}

cudaError_t launch_vector_phase(const PcgBuffers& w, cudaStream_t s) {
  k_update<<<wave_grid<k_update>(), kThreads, 0, s>>>(w.n, w.x, w.r, w.p, w.Ap, w.inv_diag, w.partials,
                                              w.st, w.history);
  k_pupdate<<<wave_grid<k_pupdate>(), kThreads, 0, s>>>(w.n, w.r, w.inv_diag, w.p, w.st);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_spmv_pcg(const BlockMatrix& A, const double* p, double* q, double* partials, PcgState* st,
                            cudaStream_t s) {
  spmv_dispatch<true>(&A, nullptr, p, q, partials, st, s);
  return cudaGetLastError();
}

cudaError_t launch_spmv(const BlockMatrix* bm, const CsrMatrixDev* cm, const double* x, double* y,
                        cudaStream_t s) {
  spmv_dispatch<false>(bm, cm, x, y, nullptr, nullptr, s);
  return cudaGetLastError();
}

cudaError_t launch_true_residual(const PcgBuffers& w, bool restart, int max_replacements,
                                 cudaStream_t s) {
  k_true_residual<<<wave_grid<k_true_residual>(), kThreads, 0, s>>>(w.n, w.b, w.Ap, w.inv_diag, w.r, w.p,
                                                     w.partials, w.st, restart ? 1 : 0,
                                                     max_replacements);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
