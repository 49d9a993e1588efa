// Learned preconditioner: a message-passing network over the node graph of the stiffness
// pattern, z = M(r) = D^-1 (r + s Y(r / s)), s = RMS(r). Inference and training kernels.
//
//   X_n  = [r/s (2), d/d_mean (2), xy/coord_scale (2), material (2)]       BF16 inputs
//   H0   = relu(W_in X + b_in)                                            BF16 [N][64]
//   A_l  = mean over neighbours m of H_{l-1,m}                             BF16 [N][64]
//   H_l  = H_{l-1} + relu(W_l [H_{l-1}; A_l] + b_l)      l = 1..3          BF16 [N][64]
//   Y    = W_out H3 + b_out                                                FP32 [N][2]
// Weights are BF16 (biases FP32); every product accumulates in FP32.
//
// The three message-passing layers run on the 5th-generation tensor cores: a CTA of 128
// threads owns a tile of 128 nodes, gathers each node's own row and the mean of its
// neighbours' rows into shared memory as the A operand ([128 nodes] x [128 = own 64 | mean 64],
// K-major, no swizzle), holds W_l as the B operand, and one thread issues eight
// tcgen05.mma.kind::f16 (M=128, N=64, K=16) into a 64-column FP32 accumulator in tensor memory.
// tcgen05.commit signals an mbarrier; each warp then reads its 32 accumulator lanes
// (tcgen05.ld.32x32b) and applies bias, ReLU and the residual add in the epilogue.
//
// Training: the forward pass also stores the inputs X, the aggregates A_l and the ReLU outputs
// G_l; the backward pass (CUDA cores, FP32 accumulation of BF16 operands) produces weight
// gradients as per-block partial sums added in block order (deterministic). The loss of a
// (residual r, error e = A^-1 r) pair is 1 - (z'r)^2 / ((z'Az)(e'r)), the squared sine of the
// energy-norm angle between z and e.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {

constexpr int F = kMpF;
constexpr int kTile = 128;             // nodes per tensor-core tile (the MMA's M)
constexpr int kASmem = kTile * 2 * F * 2;  // A operand bytes (128 x 128 BF16)
constexpr int kBSmem = F * 2 * F * 2;      // B operand bytes (64 x 128 BF16)
constexpr int kTcSmem = kASmem + kBSmem + 1024;
constexpr long long kMbarSpinLimit = 1LL << 22;  // bounded wait for the MMA (far above its ~us)

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major, no swizzle: core matrices of 8 rows x 16 bytes;
// `lbo` = byte distance between the two 8-element K halves of one MMA's K=16 slice, `sbo` =
// byte distance between 8-row groups. Bit 46 = descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of tcgen05.mma.kind::f16: D FP32, A and B BF16, both K-major,
// N = 64 (bits 17-22: N >> 3), M = 128 (bits 24-28: M >> 4).
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(F >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  for (long long i = 0; i < kMbarSpinLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

// Deterministic sum over the grid: per-block sums, then the last block adds them in order.
template <int NV, int NT>
__device__ __forceinline__ bool grid_sum(const double (&v)[NV], double* partials, unsigned int* ticket,
                                         double (&tot)[NV]) {
  __shared__ double sm[NT / 32];
  __shared__ bool am_last;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double s = block_sum<NT>(v[q], sm);
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
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) s += __ldcg(&partials[q * gridDim.x + i]);
    tot[q] = block_sum<NT>(s, sm);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

constexpr int kRedGrid = 296;  // fixed grid of the reductions here (2 x 148): a fixed sum order

// ---- residual scale ----------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_mp_rr(int n, const double* __restrict__ r, MpScratch* sc) {
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a = fma(r[i], r[i], a);
  const double v[1] = {a};
  double tot[1];
  if (grid_sum<1, 256>(v, sc->partials, &sc->ticket[0], tot) && threadIdx.x == 0) sc->rr = tot[0];
}

// ---- encoder: H0 = relu(W_in X + b_in) ------------------------------------------------------------

template <bool TRAIN>
__global__ void __launch_bounds__(256) k_mp_encode(int N, const double* __restrict__ r, const double* rr,
                                                   double inv_n, const float* __restrict__ sf, MpnnParams P,
                                                   const int* skip, __nv_bfloat16* __restrict__ H0,
                                                   __nv_bfloat16* __restrict__ Xout) {
  if (skip && *skip) return;
  __shared__ float w[F * kMpIn], b[F];
  for (int i = threadIdx.x; i < F * kMpIn; i += blockDim.x) w[i] = bf(P.pb[kMpOffWin + i]);
  for (int i = threadIdx.x; i < F; i += blockDim.x) b[i] = P.pf[kMpOffBin + i];
  __syncthreads();
  const double s = sqrt(*rr * inv_n);
  const double sd = s > 0.0 ? s : 1.0;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    float x[kMpIn];
    x[0] = (float)(r[2 * n] / sd);
    x[1] = (float)(r[2 * n + 1] / sd);
#pragma unroll
    for (int k = 0; k < 6; ++k) x[2 + k] = sf[(size_t)n * 6 + k];
#pragma unroll
    for (int k = 0; k < kMpIn; ++k) x[k] = __bfloat162float(__float2bfloat16_rn(x[k]));
    if (TRAIN) {
      uint4 xv;
      xv.x = pack_bf2(x[0], x[1]);
      xv.y = pack_bf2(x[2], x[3]);
      xv.z = pack_bf2(x[4], x[5]);
      xv.w = pack_bf2(x[6], x[7]);
      reinterpret_cast<uint4*>(Xout)[n] = xv;
    }
    uint4* out = reinterpret_cast<uint4*>(H0 + (size_t)n * F);
#pragma unroll 1
    for (int c = 0; c < F / 8; ++c) {
      float h[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int o = c * 8 + j;
        float u = b[o];
#pragma unroll
        for (int k = 0; k < kMpIn; ++k) u = fmaf(w[o * kMpIn + k], x[k], u);
        h[j] = fmaxf(u, 0.f);
      }
      out[c] = make_uint4(pack_bf2(h[0], h[1]), pack_bf2(h[2], h[3]), pack_bf2(h[4], h[5]), pack_bf2(h[6], h[7]));
    }
  }
}

// ---- message-passing layer on the tensor cores ----------------------------------------------------

template <bool TRAIN>
__global__ void __launch_bounds__(128, 3) k_mp_layer_tc(int N, const int* __restrict__ node_ptr,
                                                         const int* __restrict__ nbr,
                                                         const __nv_bfloat16* __restrict__ Hin, MpnnParams P,
                                                         int layer, const int* skip,
                                                         __nv_bfloat16* __restrict__ Hout,
                                                         __nv_bfloat16* __restrict__ Gout,
                                                         __nv_bfloat16* __restrict__ Aout, int* err) {
  if (skip && *skip) return;  // uniform: before any barrier or tensor-memory allocation
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = base;            // element (m, k): (k/8)*2048 + (m/8)*128 + (m%8)*16 + (k%8)*2
  uint8_t* sB = base + kASmem;   // element (n, k): (k/8)*1024 + (n/8)*128 + (n%8)*16 + (k%8)*2
  const int t = threadIdx.x, warp = t >> 5;
  const __nv_bfloat16* W = P.pb + kMpOffL0 + layer * kMpLStride;
  const float* bias = P.pf + kMpOffL0 + layer * kMpLStride + F * 2 * F;

  for (int idx = t; idx < F * 16; idx += 128) {  // 64 rows x 16 chunks of 8 BF16
    const int n = idx >> 4, kc = idx & 15;
    const uint4 v = *reinterpret_cast<const uint4*>(W + n * 2 * F + kc * 8);
    *reinterpret_cast<uint4*>(sB + kc * 1024 + (n >> 3) * 128 + (n & 7) * 16) = v;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                 "r"(F));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t a_addr = smem_u32(sA), b_addr = smem_u32(sB), mbar_addr = smem_u32(&mbar);
  uint32_t phase = 0;

  for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x) {
    const int n = tile * kTile + t;
    uint4 own[8];
    float acc[F];
#pragma unroll
    for (int o = 0; o < F; ++o) acc[o] = 0.f;
    int deg = 0;
    if (n < N) {
      const uint4* hr = reinterpret_cast<const uint4*>(Hin + (size_t)n * F);
#pragma unroll
      for (int c = 0; c < 8; ++c) own[c] = __ldg(hr + c);
      const int k0 = __ldg(&node_ptr[n]), k1 = __ldg(&node_ptr[n + 1]);
      for (int k = k0; k < k1; ++k) {
        const int m = __ldg(&nbr[k]);
        if (m == n) continue;
        ++deg;
        const uint4* hm = reinterpret_cast<const uint4*>(Hin + (size_t)m * F);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint4 v = __ldg(hm + c);
          acc[c * 8 + 0] += bf_lo(v.x);
          acc[c * 8 + 1] += bf_hi(v.x);
          acc[c * 8 + 2] += bf_lo(v.y);
          acc[c * 8 + 3] += bf_hi(v.y);
          acc[c * 8 + 4] += bf_lo(v.z);
          acc[c * 8 + 5] += bf_hi(v.z);
          acc[c * 8 + 6] += bf_lo(v.w);
          acc[c * 8 + 7] += bf_hi(v.w);
        }
      }
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) own[c] = make_uint4(0u, 0u, 0u, 0u);
    }
    const float inv = deg ? 1.f / (float)deg : 0.f;
    const uint32_t row_off = (uint32_t)((t >> 3) * 128 + (t & 7) * 16);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      *reinterpret_cast<uint4*>(sA + c * 2048 + row_off) = own[c];
      uint4 av;
      av.x = pack_bf2(acc[c * 8 + 0] * inv, acc[c * 8 + 1] * inv);
      av.y = pack_bf2(acc[c * 8 + 2] * inv, acc[c * 8 + 3] * inv);
      av.z = pack_bf2(acc[c * 8 + 4] * inv, acc[c * 8 + 5] * inv);
      av.w = pack_bf2(acc[c * 8 + 6] * inv, acc[c * 8 + 7] * inv);
      *reinterpret_cast<uint4*>(sA + (8 + c) * 2048 + row_off) = av;
      if (TRAIN && n < N) reinterpret_cast<uint4*>(Aout + (size_t)n * F)[c] = av;
    }
    // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // K = 128 in slices of 16: two 8-element halves each
        const uint64_t ad = umma_desc(a_addr + (uint32_t)(2 * j) * 2048u, 2048u, 128u);
        const uint64_t bd = umma_desc(b_addr + (uint32_t)(2 * j) * 1024u, 1024u, 128u);
        const uint32_t acc_flag = j > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc_flag), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       mbar_addr)
                   : "memory");
    }
    if (!mbar_wait(mbar_addr, phase) && err) atomicMin(&err[kErrTimeout], tile);
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    uint32_t v[F];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t part[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * 16), part);
#pragma unroll
      for (int j = 0; j < 16; ++j) v[q * 16 + j] = part[j];
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    if (n < N) {
      uint4* ho = reinterpret_cast<uint4*>(Hout + (size_t)n * F);
      uint4* go = TRAIN ? reinterpret_cast<uint4*>(Gout + (size_t)n * F) : nullptr;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint32_t ow[4] = {own[c].x, own[c].y, own[c].z, own[c].w};
        uint32_t hw[4], gw[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int o = c * 8 + 2 * j;
          const float g0 = fmaxf(__uint_as_float(v[o]) + bias[o], 0.f);
          const float g1 = fmaxf(__uint_as_float(v[o + 1]) + bias[o + 1], 0.f);
          hw[j] = pack_bf2(bf_lo(ow[j]) + g0, bf_hi(ow[j]) + g1);
          gw[j] = pack_bf2(g0, g1);
        }
        ho[c] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        if (TRAIN) go[c] = make_uint4(gw[0], gw[1], gw[2], gw[3]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();  // tensor memory and the A tile are free for the next tile
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(F));
}

// ---- decoder + preconditioner output: z = D^-1 (r + s (W_out H3 + b_out)) -------------------------

template <bool TRAIN>
__global__ void __launch_bounds__(256) k_mp_decode(int N, const __nv_bfloat16* __restrict__ H3, MpnnParams P,
                                                   const double* __restrict__ r, const double* __restrict__ invd,
                                                   const double* rr, double inv_n, const int* skip,
                                                   double* __restrict__ z, float* __restrict__ Yout) {
  const bool jacobi = skip && *skip;
  __shared__ float w[2 * F];
  __shared__ float b[2];
  for (int i = threadIdx.x; i < 2 * F; i += blockDim.x) w[i] = bf(P.pb[kMpOffWout + i]);
  if (threadIdx.x < 2) b[threadIdx.x] = P.pf[kMpOffBout + threadIdx.x];
  __syncthreads();
  const double s = sqrt(*rr * inv_n);
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double r0 = r[2 * n], r1 = r[2 * n + 1];
    if (jacobi) {
      z[2 * n] = invd[2 * n] * r0;
      z[2 * n + 1] = invd[2 * n + 1] * r1;
      continue;
    }
    float y0 = b[0], y1 = b[1];
    const uint4* h = reinterpret_cast<const uint4*>(H3 + (size_t)n * F);
#pragma unroll 2
    for (int c = 0; c < 8; ++c) {
      const uint4 v = h[c];
      const uint32_t hw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = c * 8 + 2 * j;
        y0 = fmaf(w[k], bf_lo(hw[j]), y0);
        y0 = fmaf(w[k + 1], bf_hi(hw[j]), y0);
        y1 = fmaf(w[F + k], bf_lo(hw[j]), y1);
        y1 = fmaf(w[F + k + 1], bf_hi(hw[j]), y1);
      }
    }
    if (TRAIN) {
      Yout[2 * n] = y0;
      Yout[2 * n + 1] = y1;
    }
    z[2 * n] = invd[2 * n] * (r0 + s * (double)y0);
    z[2 * n + 1] = invd[2 * n + 1] * (r1 + s * (double)y1);
  }
}

// ---- training: loss and dL/dY ------------------------------------------------------------------

// c = z'r, zAz = z'(Az), er = e'r
__global__ void __launch_bounds__(256) k_mp_loss_dots(int n, const double* __restrict__ z,
                                                      const double* __restrict__ az, const double* __restrict__ r,
                                                      const double* __restrict__ e, MpScratch* sc) {
  double c = 0.0, zaz = 0.0, er = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    c = fma(z[i], r[i], c);
    zaz = fma(z[i], az[i], zaz);
    er = fma(e[i], r[i], er);
  }
  const double v[3] = {c, zaz, er};
  double tot[3];
  if (grid_sum<3, 256>(v, sc->partials, &sc->ticket[1], tot) && threadIdx.x == 0) {
    sc->dots[0] = tot[0];
    sc->dots[1] = tot[1];
    sc->dots[2] = tot[2];
    sc->loss = 1.0 - tot[0] * tot[0] / (tot[1] * tot[2]);
  }
}

// dY_i = s D^-1_i (f1 r_i + f2 (Az)_i), f1 = -2c/(zAz er), f2 = 2c^2/(zAz^2 er)
__global__ void __launch_bounds__(256) k_mp_dy(int n, const double* __restrict__ r, const double* __restrict__ az,
                                               const double* __restrict__ invd, double inv_n, const MpScratch* sc,
                                               float* __restrict__ dY) {
  const double c = sc->dots[0], zaz = sc->dots[1], er = sc->dots[2];
  const double f1 = -2.0 * c / (zaz * er), f2 = 2.0 * c * c / (zaz * zaz * er);
  const double s = sqrt(sc->rr * inv_n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dY[i] = (float)(s * invd[i] * (f1 * r[i] + f2 * az[i]));
}

// ---- training: backward ------------------------------------------------------------------------

// dH3 = W_out' dY; partial gradients of W_out (2 x 64) and b_out (2) per block
__global__ void __launch_bounds__(256) k_mp_dec_bwd(int N, const __nv_bfloat16* __restrict__ H3, MpnnParams P,
                                                    const float* __restrict__ dY, float* __restrict__ dH,
                                                    float* __restrict__ part /* [grid][130] */) {
  __shared__ float w[2 * F];
  __shared__ float red[2 * F + 2];
  for (int i = threadIdx.x; i < 2 * F; i += blockDim.x) w[i] = bf(P.pb[kMpOffWout + i]);
  for (int i = threadIdx.x; i < 2 * F + 2; i += blockDim.x) red[i] = 0.f;
  __syncthreads();
  // thread layout: 64 features x 4 node lanes
  const int k = threadIdx.x & 63, lane4 = threadIdx.x >> 6;
  float gw0 = 0.f, gw1 = 0.f, gb0 = 0.f, gb1 = 0.f;
  for (int n = blockIdx.x * 4 + lane4; n < N; n += gridDim.x * 4) {
    const float d0 = dY[2 * n], d1 = dY[2 * n + 1];
    const float h = bf(H3[(size_t)n * F + k]);
    dH[(size_t)n * F + k] = d0 * w[k] + d1 * w[F + k];
    gw0 = fmaf(d0, h, gw0);
    gw1 = fmaf(d1, h, gw1);
    if (k == 0) {
      gb0 += d0;
      gb1 += d1;
    }
  }
  // fixed-order block reduction: the four node lanes in order
  for (int l = 0; l < 4; ++l) {
    if (lane4 == l) {
      red[k] += gw0;
      red[F + k] += gw1;
      if (k == 0) {
        red[2 * F] += gb0;
        red[2 * F + 1] += gb1;
      }
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < 2 * F + 2; i += blockDim.x) part[(size_t)blockIdx.x * (2 * F + 2) + i] = red[i];
}

// Layer backward, part 1: dU = dH (G > 0); dHprev = dH + W_h' dU; dAs = (W_a' dU) / deg.
// 64 threads per node (feature k), four nodes per 256-thread block step.
__global__ void __launch_bounds__(256) k_mp_layer_bwd_a(int N, const int* __restrict__ node_ptr,
                                                        const int* __restrict__ nbr, MpnnParams P, int layer,
                                                        const float* __restrict__ dH,
                                                        const __nv_bfloat16* __restrict__ G,
                                                        float* __restrict__ dU, float* __restrict__ dHprev,
                                                        float* __restrict__ dAs) {
  extern __shared__ float wsm[];  // W_l as float [64][128]
  __shared__ float du[4][F];
  const __nv_bfloat16* W = P.pb + kMpOffL0 + layer * kMpLStride;
  for (int i = threadIdx.x; i < F * 2 * F; i += blockDim.x) wsm[i] = bf(W[i]);
  const int k = threadIdx.x & 63, g = threadIdx.x >> 6;
  for (int base = blockIdx.x * 4; base < N; base += gridDim.x * 4) {
    const int n = base + g;
    __syncthreads();
    float dh = 0.f;
    if (n < N) {
      dh = dH[(size_t)n * F + k];
      const float u = bf(G[(size_t)n * F + k]) > 0.f ? dh : 0.f;
      du[g][k] = u;
      dU[(size_t)n * F + k] = u;
    } else {
      du[g][k] = 0.f;
    }
    __syncthreads();
    if (n < N) {
      float sh = 0.f, sa = 0.f;
#pragma unroll 8
      for (int o = 0; o < F; ++o) {
        const float u = du[g][o];
        sh = fmaf(u, wsm[o * 2 * F + k], sh);
        sa = fmaf(u, wsm[o * 2 * F + F + k], sa);
      }
      int deg = 0;
      for (int q = node_ptr[n]; q < node_ptr[n + 1]; ++q) deg += nbr[q] != n;
      dHprev[(size_t)n * F + k] = dh + sh;
      dAs[(size_t)n * F + k] = deg ? sa / (float)deg : 0.f;
    }
  }
}

// Layer backward, part 2: dHprev_m += sum over neighbours n of m of dAs_n (the mean's transpose)
__global__ void __launch_bounds__(256) k_mp_layer_bwd_b(int N, const int* __restrict__ node_ptr,
                                                        const int* __restrict__ nbr, const float* __restrict__ dAs,
                                                        float* __restrict__ dHprev) {
  const int k = threadIdx.x & 63;
  for (int m = blockIdx.x * 4 + (threadIdx.x >> 6); m < N; m += gridDim.x * 4) {
    float s = 0.f;
    for (int q = node_ptr[m]; q < node_ptr[m + 1]; ++q) {
      const int n = nbr[q];
      if (n != m) s += dAs[(size_t)n * F + k];
    }
    dHprev[(size_t)m * F + k] += s;
  }
}

// Weight gradient of a layer: dW[o][k] = sum_n dU[n][o] Xc[n][k], Xc = [Hprev | A] (BF16),
// db[o] = sum_n dU[n][o]; per-block partials [grid][64 * KW + 64]. KW = 128 (layers) or 8 (encoder,
// Xc = X). Each thread owns outputs o = tid / 4 and a quarter of the K columns.
template <int KW>
__global__ void __launch_bounds__(256) k_mp_wgrad(int N, const float* __restrict__ dU,
                                                  const __nv_bfloat16* __restrict__ X1,
                                                  const __nv_bfloat16* __restrict__ X2, float* __restrict__ part) {
  constexpr int KQ = KW / 4;
  constexpr int CH = 32;  // nodes per staged chunk
  __shared__ float sdu[CH][F];
  __shared__ float sx[CH][KW];
  const int o = threadIdx.x >> 2, q = threadIdx.x & 3;
  float acc[KQ];
#pragma unroll
  for (int i = 0; i < KQ; ++i) acc[i] = 0.f;
  float bacc = 0.f;
  const int per = (N + gridDim.x - 1) / gridDim.x;
  const int n0 = blockIdx.x * per, n1 = min(N, n0 + per);
  for (int c0 = n0; c0 < n1; c0 += CH) {
    __syncthreads();
    for (int i = threadIdx.x; i < CH * F; i += 256) {
      const int j = i / F, f = i % F, n = c0 + j;
      sdu[j][f] = n < n1 ? dU[(size_t)n * F + f] : 0.f;
    }
    for (int i = threadIdx.x; i < CH * KW; i += 256) {
      const int j = i / KW, f = i % KW, n = c0 + j;
      float v = 0.f;
      if (n < n1) {
        if (KW == 2 * F)
          v = f < F ? bf(X1[(size_t)n * F + f]) : bf(X2[(size_t)n * F + f - F]);
        else
          v = bf(X1[(size_t)n * KW + f]);
      }
      sx[j][f] = v;
    }
    __syncthreads();
    for (int j = 0; j < CH; ++j) {
      const float u = sdu[j][o];
      bacc += q == 0 ? u : 0.f;
#pragma unroll
      for (int i = 0; i < KQ; ++i) acc[i] = fmaf(u, sx[j][q * KQ + i], acc[i]);
    }
  }
  float* p = part + (size_t)blockIdx.x * (F * KW + F);
#pragma unroll
  for (int i = 0; i < KQ; ++i) p[o * KW + q * KQ + i] = acc[i];
  if (q == 0) p[F * KW + o] = bacc;
}

// Encoder backward: dU0 = dH0 (H0 > 0)
__global__ void __launch_bounds__(256) k_mp_enc_bwd(int N, const float* __restrict__ dH,
                                                    const __nv_bfloat16* __restrict__ H0, float* __restrict__ dU) {
  const size_t total = (size_t)N * F;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    dU[i] = bf(H0[i]) > 0.f ? dH[i] : 0.f;
}

// grad[dst + i] += sum over blocks b (in order) of part[b][src + i], for i < count
__global__ void k_mp_reduce_parts(const float* __restrict__ part, int nblocks, int stride, int src, int count,
                                  float* __restrict__ grad, int dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * stride + src + i];
    grad[dst + i] += s;
  }
}

// Adam (decoupled weight decay off): master FP32 parameters, BF16 copies for the kernels.
__global__ void k_mp_adam(int n, float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                          const float* __restrict__ g, float lr, float b1, float b2, float eps, float bc1,
                          float bc2, float scale, __nv_bfloat16* __restrict__ pb, float* __restrict__ pf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i] * scale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16_rn(pi);
    pf[i] = pi;
  }
}

__global__ void k_mp_convert(int n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb,
                             float* __restrict__ pf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    pb[i] = __float2bfloat16_rn(p[i]);
    pf[i] = p[i];
  }
}

int grid_nodes(long long work, int per_block) {
  const long long g = (work + per_block - 1) / per_block;
  return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

int tc_grid(int N) {
  const int tiles = (N + kTile - 1) / kTile;
  return std::max(1, std::min(tiles, 148 * 3));
}

template <bool TRAIN>
cudaError_t set_tc_attr() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(k_mp_layer_tc<TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

}  // namespace

cudaError_t mpnn_prepare_device() {
  cudaError_t e = set_tc_attr<false>();
  if (e != cudaSuccess) return e;
  return set_tc_attr<true>();
}

cudaError_t launch_mp_params(const float* p32, __nv_bfloat16* pb, float* pf, cudaStream_t s) {
  k_mp_convert<<<grid_nodes(kMpParams, 256), 256, 0, s>>>(kMpParams, p32, pb, pf);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_rr(int n, const double* r, MpScratch* sc, cudaStream_t s) {
  k_mp_rr<<<kRedGrid, 256, 0, s>>>(n, r, sc);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_forward(const MpnnGraph& g, const MpnnParams& P, const double* r, const double* invd,
                              const double* rr, const float* sf, const int* skip, MpnnWork& w, bool train,
                              double* z, int* err, cudaStream_t s) {
  const int N = g.n_nodes;
  if (N <= 0) return cudaSuccess;
  const double inv_n = 1.0 / (2.0 * N);
  const int ge = grid_nodes(N, 256);
  if (train)
    k_mp_encode<true><<<ge, 256, 0, s>>>(N, r, rr, inv_n, sf, P, skip, w.H[0], w.X);
  else
    k_mp_encode<false><<<ge, 256, 0, s>>>(N, r, rr, inv_n, sf, P, skip, w.H[0], nullptr);
  for (int l = 0; l < kMpL; ++l) {
    __nv_bfloat16* hout = train ? w.H[l + 1] : w.H[(l + 1) & 1];
    const __nv_bfloat16* hin = train ? w.H[l] : w.H[l & 1];
    if (train)
      k_mp_layer_tc<true><<<tc_grid(N), 128, kTcSmem, s>>>(N, g.node_ptr, g.nbr, hin, P, l, skip, hout,
                                                           w.G[l], w.A[l], err);
    else
      k_mp_layer_tc<false><<<tc_grid(N), 128, kTcSmem, s>>>(N, g.node_ptr, g.nbr, hin, P, l, skip, hout,
                                                            nullptr, nullptr, err);
  }
  const __nv_bfloat16* h3 = train ? w.H[kMpL] : w.H[kMpL & 1];
  if (train)
    k_mp_decode<true><<<ge, 256, 0, s>>>(N, h3, P, r, invd, rr, inv_n, skip, z, w.Y);
  else
    k_mp_decode<false><<<ge, 256, 0, s>>>(N, h3, P, r, invd, rr, inv_n, skip, z, nullptr);
  count_launches(2 + kMpL);
  return cudaGetLastError();
}

cudaError_t launch_mp_loss(int N, const double* z, const double* az, const double* r, const double* e,
                           const double* invd, MpScratch* sc, MpnnWork& w, cudaStream_t s) {
  const int n = 2 * N;
  k_mp_loss_dots<<<kRedGrid, 256, 0, s>>>(n, z, az, r, e, sc);
  k_mp_dy<<<grid_nodes(n, 256), 256, 0, s>>>(n, r, az, invd, 1.0 / n, sc, w.dY);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_mp_backward(const MpnnGraph& g, const MpnnParams& P, MpnnWork& w, float* grad, cudaStream_t s) {
  const int N = g.n_nodes;
  if (N <= 0) return cudaSuccess;
  const int G = kMpPartBlocks;
  // decoder
  k_mp_dec_bwd<<<G, 256, 0, s>>>(N, w.H[kMpL], P, w.dY, w.dH, w.part);
  k_mp_reduce_parts<<<1, 256, 0, s>>>(w.part, G, 2 * F + 2, 0, 2 * F, grad, kMpOffWout);
  k_mp_reduce_parts<<<1, 32, 0, s>>>(w.part, G, 2 * F + 2, 2 * F, 2, grad, kMpOffBout);
  long long k = 3;
  // layers 3..1
  float* dh = w.dH;
  float* dprev = w.dH2;
  for (int l = kMpL - 1; l >= 0; --l) {
    k_mp_layer_bwd_a<<<grid_nodes(N, 4), 256, F * 2 * F * sizeof(float), s>>>(N, g.node_ptr, g.nbr, P, l, dh,
                                                                               w.G[l], w.dU, dprev, w.dAs);
    k_mp_wgrad<2 * F><<<G, 256, 0, s>>>(N, w.dU, w.H[l], w.A[l], w.part);
    k_mp_layer_bwd_b<<<grid_nodes(N, 4), 256, 0, s>>>(N, g.node_ptr, g.nbr, w.dAs, dprev);
    const int off = kMpOffL0 + l * kMpLStride;
    k_mp_reduce_parts<<<grid_nodes(F * 2 * F + F, 256), 256, 0, s>>>(w.part, G, F * 2 * F + F, 0, F * 2 * F + F,
                                                                      grad, off);
    std::swap(dh, dprev);
    k += 4;
  }
  // encoder
  k_mp_enc_bwd<<<grid_nodes((long long)N * F, 256), 256, 0, s>>>(N, dh, w.H[0], w.dU);
  k_mp_wgrad<kMpIn><<<G, 256, 0, s>>>(N, w.dU, w.X, nullptr, w.part);
  k_mp_reduce_parts<<<grid_nodes(F * kMpIn + F, 256), 256, 0, s>>>(w.part, G, F * kMpIn + F, 0, F * kMpIn + F,
                                                                    grad, kMpOffWin);
  k += 3;
  count_launches(k);
  return cudaGetLastError();
}

cudaError_t launch_mp_adam(float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
                           int step, float scale, __nv_bfloat16* pb, float* pf, cudaStream_t s) {
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_mp_adam<<<grid_nodes(kMpParams, 256), 256, 0, s>>>(kMpParams, p, m, v, g, lr, b1, b2, eps, bc1, bc2, scale,
                                                       pb, pf);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
