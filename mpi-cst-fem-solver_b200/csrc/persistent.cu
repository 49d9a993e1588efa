// Persistent Jacobi-PCG: one cooperative launch runs every iteration of a solve on the mesh
// (2x2-block) pattern, FP64 or mixed precision, instead of three or four kernels per iteration.
//
// Per iteration (FP64; the mixed method swaps the SpMV operator and may add the replacement
// phase R, see mixed_kernels.cu for the method):
//   A  Ap = A p, p'Ap                      -> grid reduction: alpha (or breakdown)
//   B  x += alpha p, r -= alpha Ap, r'r, r'z -> grid reduction: convergence test, beta
//   R  (mixed, when due) r = b - A64 x       -> grid reduction: reliable update / switch
//   C  p = D^-1 r + beta p                  -> grid barrier
//
// Grid barriers: the grid is one wave of co-resident blocks (cooperative launch). A block
// writes its partial sums, fences, and arrives on an atomic counter; the last block to arrive
// sums all partials in index order (deterministic), runs the scalar update and releases the
// others by bumping a generation word. Every wait is bounded (spin_limit polls, by default
// kBarrierSpinDefault ~ 2 s):
// a block that gives up sets bar_err and done = TIMEOUT and returns, and so do all others,
// so a fault can never leave the GPU spinning. Data written by other blocks inside this
// kernel is read with ld.global.cg (L2), since L1 is not coherent within a kernel.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ double2 ldcg2(const double* a, int i) {
  return __ldcg(reinterpret_cast<const double2*>(a) + i);
}
__device__ __forceinline__ void stcg2(double* a, int i, double2 v) {
  __stcg(reinterpret_cast<double2*>(a) + i, v);
}

// One 1024-thread block per SM: 148 arrivals per grid barrier instead of ~740.
constexpr int kPT = 1024;

struct Shared {
  double red[kPT / 32];
  long long limit;  // polls of a barrier wait before it gives up
  int last;
  int ok;
};

// Arrive at the grid barrier after writing NV partial sums; the last block reduces them and
// calls epi(tot) in thread 0 before releasing. Returns false (in every thread) when this
// block's wait ran out.
template <int NV, class Epi>
__device__ __forceinline__ bool grid_reduce(const double (&v)[NV], double* partials, PcgState* st,
                                            Shared& sh, Epi epi) {
  const unsigned G = gridDim.x;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double s = block_sum<kPT>(v[q], sh.red);
    if (threadIdx.x == 0) __stcg(&partials[q * G + blockIdx.x], s);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_acquire(&st->bar_gen);
    __threadfence();
    const unsigned arrived = atomicAdd(&st->bar_count, 1u);
    sh.last = arrived == G - 1;
    sh.ok = 1;
    if (!sh.last) {
      long long spins = 0;
      while (ld_acquire(&st->bar_gen) == gen) {
        if (++spins > sh.limit || __ldcg(&st->bar_err)) {
          atomicExch(&st->bar_err, 1);
          st->done = CSTG_SOLVE_TIMEOUT + 1;
          sh.ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  if (sh.last) {
    __threadfence();
    double tot[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int i = threadIdx.x; i < (int)G; i += blockDim.x) s += __ldcg(&partials[q * G + i]);
      tot[q] = block_sum<kPT>(s, sh.red);
    }
    if (threadIdx.x == 0) {
      epi(tot);
      st->bar_count = 0;
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    }
    __syncthreads();
  }
  return sh.ok != 0;
}

__device__ __forceinline__ bool grid_barrier(PcgState* st, Shared& sh, double* partials) {
  const double z[1] = {0.0};
  return grid_reduce<1>(z, partials, st, sh, [](const double*) {});
}

// ---- SpMV phases (the work split of the standalone kernels) -------------------------------------

__device__ __forceinline__ double spmv64(const BlockMatrix& A, const double* __restrict__ x,
                                         double* __restrict__ y) {
  const int lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
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
      const double2 x0 = ldcg2(x, m0), x1 = ldcg2(x, m1);
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
        stcg2(y, n0, make_double2(ya0, yb0));
        const double2 pv = ldcg2(x, n0);
        dot = fma(pv.x, ya0, fma(pv.y, yb0, dot));
      }
      if (n1 < N) {
        stcg2(y, n1, make_double2(ya1, yb1));
        const double2 pv = ldcg2(x, n1);
        dot = fma(pv.x, ya1, fma(pv.y, yb1, dot));
      }
    }
  }
  return dot;
}

// One thread per node (see k_spmv_mixed): FP32 difference-form blocks, FP64 vectors.
__device__ __forceinline__ double spmv32(const MixedMatrix& A, const double* __restrict__ x,
                                         double* __restrict__ y) {
  const int N = A.n_nodes;
  double dot = 0.0;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const int b = __ldg(&A.node_ptr[n]);
    const int o = b - n, c = __ldg(&A.node_ptr[n + 1]) - b - 1;
    const double2 xs = ldcg2(x, n);
    double ya = 0.0, yb = 0.0;
    for (int k = 0; k < c; ++k) {
      const int m = __ldg(&A.nbr32[o + k]);
      const float4 av = __ldg(&A.val32[o + k]);
      const double2 xm = ldcg2(x, m);
      const double dx = xm.x - xs.x, dy = xm.y - xs.y;
      ya = fma((double)av.x, dx, fma((double)av.y, dy, ya));
      yb = fma((double)av.z, dx, fma((double)av.w, dy, yb));
    }
    const double2 sa = __ldg(&A.S64[2 * n]), sb = __ldg(&A.S64[2 * n + 1]);
    ya = fma(sa.x, xs.x, fma(sa.y, xs.y, ya));
    yb = fma(sb.x, xs.x, fma(sb.y, xs.y, yb));
    stcg2(y, n, make_double2(ya, yb));
    dot = fma(xs.x, ya, fma(xs.y, yb, dot));
  }
  return dot;
}

// r = b - A64 x (FP64), partial r'r and r'D^-1 r
__device__ __forceinline__ void residual64(const BlockMatrix& A, const double* __restrict__ x,
                                           const double* __restrict__ b, const double* __restrict__ invd,
                                           double* __restrict__ r, double& rr, double& rz) {
  const int lane = threadIdx.x & 31, sub = lane >> 3, l8 = lane & 7;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const double2* __restrict__ v2 = reinterpret_cast<const double2*>(A.vals);
  const int N = A.n_nodes;
  for (int base = warp * 4; base < N; base += nwarps * 4) {
    const int n = base + sub;
    double ya = 0.0, yb = 0.0;
    if (n < N) {
      const int b0 = __ldg(&A.node_ptr[n]), deg = __ldg(&A.node_ptr[n + 1]) - b0;
      for (int k = l8; k < deg; k += 8) {
        const int m = __ldg(&A.bnbr[b0 + k]);
        const double2 xv = ldcg2(x, m);
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
      const double2 bv = reinterpret_cast<const double2*>(b)[n];
      const double2 dv = reinterpret_cast<const double2*>(invd)[n];
      const double rx = bv.x - ya, ry = bv.y - yb;
      stcg2(r, n, make_double2(rx, ry));
      rr = fma(rx, rx, fma(ry, ry, rr));
      rz = fma(rx, dv.x * rx, fma(ry, dv.y * ry, rz));
    }
  }
}

}  // namespace

struct PersistArgs {
  BlockMatrix A64;
  MixedMatrix A32;
  double* x;
  double* r;
  double* p;
  double* Ap;
  const double* invd;
  const double* b;
  double* partials;
  double* history;
  PcgState* st;
  int max_final_checks;
  long long spin_limit;
};

template <bool MIXED>
__global__ void __launch_bounds__(kPT, 1) k_pcg_persistent(PersistArgs a) {
  __shared__ Shared sh;
  if (threadIdx.x == 0) sh.limit = a.spin_limit;
  __syncthreads();
  PcgState* st = a.st;
  const int npairs = a.A64.n_nodes;  // DOF pairs = nodes
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  while (true) {
    if (__ldcg(&st->done)) return;
    // ---- A: SpMV + p'Ap -> alpha
    {
      const bool use64 = !MIXED || __ldcg(&st->fp64_mode);
      const double d[1] = {use64 ? spmv64(a.A64, a.p, a.Ap) : spmv32(a.A32, a.p, a.Ap)};
      if (!grid_reduce<1>(d, a.partials, st, sh, [&](const double* tot) {
            st->pAp = tot[0];
            if (!(tot[0] > 0.0)) {
              st->alpha = 0.0;
              st->done = CSTG_SOLVE_BREAKDOWN + 1;
            } else {
              st->alpha = st->rz / tot[0];
            }
          }))
        return;
    }
    if (__ldcg(&st->done)) return;
    // ---- B: x, r update -> convergence test, beta
    {
      const double alpha = __ldcg(&st->alpha);
      double rr = 0.0, rz = 0.0;
      for (int i = tid; i < npairs; i += nth) {
        const double2 pi = ldcg2(a.p, i), ai = ldcg2(a.Ap, i), di = ldcg2(a.invd, i);
        double2 xi = ldcg2(a.x, i), ri = ldcg2(a.r, i);
        xi.x = fma(alpha, pi.x, xi.x);
        xi.y = fma(alpha, pi.y, xi.y);
        ri.x = fma(-alpha, ai.x, ri.x);
        ri.y = fma(-alpha, ai.y, ri.y);
        stcg2(a.x, i, xi);
        stcg2(a.r, i, ri);
        rr = fma(ri.x, ri.x, fma(ri.y, ri.y, rr));
        rz = fma(ri.x, di.x * ri.x, fma(ri.y, di.y * ri.y, rz));
      }
      const double v[2] = {rr, rz};
      if (!grid_reduce<2>(v, a.partials, st, sh, [&](const double* tot) {
            const int it = st->iter + 1;
            st->iter = it;
            const double rn = sqrt(tot[0]);
            const double rel = rn / st->bnorm;
            st->rel = rel;
            st->rr = tot[0];
            if (st->hist_on) a.history[it] = rel;
            if (!MIXED) {
              if (rel < st->rtol)
                st->done = CSTG_SOLVE_CONVERGED + 1;
              else if (it >= st->max_iter)
                st->done = CSTG_SOLVE_MAX_ITER + 1;
            } else {
              st->rmax = fmax(st->rmax, rn);
              if (rel < st->rtol)
                st->restart_pending = 2;
              else if (!st->fp64_mode && rn < st->delta * st->rmax)
                st->restart_pending = 1;
              else if (!st->fp64_mode && it - st->last_replace >= st->cycle_limit)
                st->restart_pending = 3;  // (plain FP64 CG after the switch, as in mixed_kernels.cu)
              else if (it >= st->max_iter)
                st->done = CSTG_SOLVE_MAX_ITER + 1;
            }
            st->rz_prev = st->rz;
            st->beta = tot[1] / st->rz;
            st->rz = tot[1];
          }))
        return;
    }
    if (__ldcg(&st->done)) return;
    // ---- R (mixed): reliable update with the FP64 residual
    if (MIXED && __ldcg(&st->restart_pending)) {
      double rr = 0.0, rz = 0.0;
      residual64(a.A64, a.x, a.b, a.invd, a.r, rr, rz);
      const double v[2] = {rr, rz};
      if (!grid_reduce<2>(v, a.partials, st, sh, [&](const double* tot) {
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
            if (st->hist_on) a.history[st->iter] = tr;
            st->beta = st->rz_prev > 0.0 ? tot[1] / st->rz_prev : 0.0;
            st->rz = tot[1];
            st->restart_pending = 0;
            if (tr < st->rtol) {
              st->done = CSTG_SOLVE_CONVERGED + 1;
            } else {
              // (the precision switch of mixed_kernels.cu's k_replace_mixed, same rule)
              if (kind == 3)
                st->stall_cycles =
                    ((tr > 0.9 * st->best_true || tr > kGapRatio * rec) && st->best_true < kStallGate)
                        ? st->stall_cycles + 1
                        : 0;
              if (!st->fp64_mode && (kind == 2 || (kind == 1 && tr > 0.5 * st->best_true) ||
                                (kind == 3 && st->stall_cycles >= 2))) {
                st->fp64_mode = 1;
                st->fp64_switch_iter = st->iter;
                st->beta = 0.0;
              } else if (st->fp64_mode) {
                st->beta = 0.0;
              }
              if (kind == 2 && ++st->final_checks > a.max_final_checks) st->done = CSTG_SOLVE_CONVERGED + 1;
              if (st->iter >= st->max_iter) st->done = CSTG_SOLVE_MAX_ITER + 1;
            }
            st->best_true = fmin(st->best_true, tr);
          }))
        return;
      if (__ldcg(&st->done)) return;
    }
    // ---- C: p = D^-1 r + beta p
    {
      const double beta = __ldcg(&st->beta);
      for (int i = tid; i < npairs; i += nth) {
        const double2 ri = ldcg2(a.r, i), di = ldcg2(a.invd, i);
        double2 pi = ldcg2(a.p, i);
        pi.x = fma(beta, pi.x, di.x * ri.x);
        pi.y = fma(beta, pi.y, di.y * ri.y);
        stcg2(a.p, i, pi);
      }
      if (!grid_barrier(st, sh, a.partials)) return;
    }
  }
}

template <bool MIXED>
static int persistent_grid() {
  static int cache[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!cache[dev]) {
    int sms = kSMs, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_persistent<MIXED>, kPT, 0);
    cache[dev] = std::min(kMaxGrid, sms * std::max(per, 0));
  }
  return cache[dev];
}

// Launches the persistent solve on an initialised state (k_init / k_init_mixed done).
cudaError_t launch_pcg_persistent(const PcgBuffers& w, const BlockMatrix& A64, const MixedMatrix* A32,
                                  int max_final_checks, long long spin_limit, cudaStream_t s) {
  PersistArgs a;
  a.A64 = A64;
  if (A32) a.A32 = *A32;
  a.x = w.x;
  a.r = w.r;
  a.p = w.p;
  a.Ap = w.Ap;
  a.invd = w.inv_diag;
  a.b = w.b;
  a.partials = w.partials;
  a.history = w.history;
  a.st = w.st;
  a.max_final_checks = max_final_checks;
  a.spin_limit = spin_limit;
  // barrier words start from zero
  cudaError_t e = cudaMemsetAsync(&w.st->bar_count, 0, sizeof(unsigned) * 2 + sizeof(int), s);
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  const int grid = A32 ? persistent_grid<true>() : persistent_grid<false>();
  if (grid <= 0) return cudaErrorCooperativeLaunchTooLarge;
  e = A32 ? cudaLaunchCooperativeKernel((void*)k_pcg_persistent<true>, grid, kPT, args, 0, s)
          : cudaLaunchCooperativeKernel((void*)k_pcg_persistent<false>, grid, kPT, args, 0, s);
  count_launches(1);
  return e;
}

}  // namespace cstg
