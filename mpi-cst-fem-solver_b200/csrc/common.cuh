// Shared device helpers for the CST / Jacobi-PCG kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cstfem_b200.h"

namespace cstg {

// Launch geometry. 148 SMs on a B200; the fixed grids below are multiples of it so that the
// deterministic reductions see the same partial-sum layout on every run.
constexpr int kSMs = 148;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Largest grid of the reduction kernels (their partial-sum buffers hold 4 x kMaxGrid doubles).
// The actual grid is one full wave: SMs x resident blocks per SM (occupancy calculator).
constexpr int kMaxGrid = 2048;

// Largest node neighbourhood (self included) the pattern builder accepts.
constexpr int kMaxNeighbours = 64;

// Bounded spin limit for grid barriers (iterations of a ~100 ns poll): about 2 s.
constexpr long long kSpinLimit = 20000000LL;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum: fixed shuffle tree, then warp 0 sums the warp totals in order.
// Every thread must call it; the result is valid in all threads.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* smem /* >= NT/32 */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < NT / 32 ? smem[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) smem[0] = t;
  }
  __syncthreads();
  t = smem[0];
  __syncthreads();
  return t;
}

// Loads that bypass L1 (data written by other blocks of the same grid).
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }

}  // namespace cstg
