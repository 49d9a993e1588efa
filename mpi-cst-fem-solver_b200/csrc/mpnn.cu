// Learned preconditioner: a message-passing network over the node graph of the stiffness
// pattern, z = M(r) = D^-1 (r + s Y(r / s)), s = RMS(r). Inference and training kernels.
//
//   X_n  = [r/s (2), d/d_mean (2), xy/coord_scale (2), material (2)]       BF16 inputs
//   H0   = relu(W_in X + b_in)                                            BF16 [N][64]
//   A_l  = mean over neighbours m of H_{l-1,m}                             BF16 [N][64]
//   H_l  = H_{l-1} + relu(W_l [H_{l-1}; A_l] + b_l)      l = 1..3          BF16 [N][64]
//   Y    = W_out H3 + b_out                                                FP32 [N][2]
// Weights are BF16 (biases FP32); every product accumulates in FP32. The encoder's 8 -> 64 product
// runs on the tensor cores too (one K=16 MMA per 128 nodes, the FP32 bias entering as three exact
// BF16 parts against constant ones in the A operand).
//
// The three message-passing layers run on the 5th-generation tensor cores: per tile of 128 nodes
// the A operand is [own row 64 | mean of the neighbours' rows 64] (BF16, K-major, 128-byte
// swizzle), W_l is the B operand, and one thread issues eight tcgen05.mma.kind::f16 (M=128, N=64,
// K=16) plus one for the bias into a 64-column FP32 accumulator in tensor memory; tcgen05.commit
// signals an mbarrier and the epilogue reads the accumulator (tcgen05.ld.32x32b), applies ReLU and
// the residual add. Two kernels give the same bits: k_mp_layer_ws on patterns with a gather plan
// (one warp-specialised CTA per SM: tensor and bulk copies, gathers, MMAs and epilogues of
// consecutive tiles overlap) and k_mp_layer_tc row by row from global memory.
//
// Training: the forward pass also stores the inputs X, the aggregates A_l and the ReLU outputs
// G_l. The backward pass runs the per-node parts (ReLU masks, the mean aggregation's transpose as
// a gather over the symmetric pattern) on CUDA cores and the layers' weight gradients on the
// tensor cores (k_mp_wgrad_tc: FP32 accumulation in tensor memory), each as per-block partial sums
// added in block order (deterministic). The loss of a (residual r, error e = A^-1 r) pair is
// 1 - (z'r)^2 / ((z'Az)(e'r)), the squared sine of the energy-norm angle between z and e.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {

constexpr int F = kMpF;
constexpr int kTile = 128;             // nodes per tensor-core tile (the MMA's M)
static_assert(kTile == kMpTile, "the gather plan is built per tensor-core tile");
constexpr int kASmem = kTile * 2 * F * 2;  // A operand bytes (128 x 128 BF16)
constexpr int kBSmem = F * 2 * F * 2;      // B operand bytes (64 x 128 BF16)
constexpr long long kMbarSpinLimit = kMpMbarSpinDefault;  // bounded wait for the MMA (far above its ~us)

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

// UMMA shared-memory descriptor, K-major, 128-byte swizzle: atoms of 8 rows x 128 bytes (1024-byte
// aligned), the 16-byte chunk q of row r stored at chunk q ^ (r % 8); `sbo` = byte distance between
// 8-row groups. A K=16 slice inside an atom starts 32 bytes further per slice (the hardware applies
// the XOR to the address bits). Bits 61-63 = 2: 128-byte swizzle.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;  // leading byte offset: unused by swizzled K-major layouts
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// Offset of 16-byte chunk c (features 8c..8c+7) of row m of the A tile: half 0 = the node's own
// row (K 0..63), half 1 = the neighbours' mean (K 64..127); each half is a 128-row column of
// 128-byte-swizzled atoms (16 KB), so the 8 chunks of one row sit in 8 different bank groups.
__device__ __forceinline__ uint32_t a_chunk(int m, int c, int half) {
  return (uint32_t)(half * 16384 + m * 128 + ((c ^ (m & 7)) << 4));
}

// Instruction descriptor of tcgen05.mma.kind::f16: D FP32, A and B BF16, both K-major,
// N = 64 (bits 17-22: N >> 3), M = 128 (bits 24-28: M >> 4).
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(F >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

// Bounded wait on an mbarrier phase; false when `limit` polls ran out (0: give up at once).
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i) {
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

// r'r over a fixed grid (a fixed order). VEC: r 16-byte aligned, pairs read as double2, four
// pairs in flight per thread.
template <bool VEC>
__global__ void __launch_bounds__(256) k_mp_rr(int n, const double* __restrict__ r, MpScratch* sc, const int* skip) {
  if (skip && *skip) return;  // uniform: every block returns before the ticket
  double a = 0.0;
  const int stride = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (VEC) {
    const double2* r2 = reinterpret_cast<const double2*>(r);
    const int n2 = n >> 1;
    int i = t0;
    for (; i + 3 * stride < n2; i += 4 * stride) {
      const double2 x0 = r2[i], x1 = r2[i + stride], x2 = r2[i + 2 * stride], x3 = r2[i + 3 * stride];
      a = fma(x0.x, x0.x, a);
      a = fma(x0.y, x0.y, a);
      a = fma(x1.x, x1.x, a);
      a = fma(x1.y, x1.y, a);
      a = fma(x2.x, x2.x, a);
      a = fma(x2.y, x2.y, a);
      a = fma(x3.x, x3.x, a);
      a = fma(x3.y, x3.y, a);
    }
    for (; i < n2; i += stride) {
      const double2 x = r2[i];
      a = fma(x.x, x.x, a);
      a = fma(x.y, x.y, a);
    }
    if ((n & 1) && t0 == 0) a = fma(r[n - 1], r[n - 1], a);
  } else {
    for (int i = t0; i < n; i += stride) a = fma(r[i], r[i], a);
  }
  const double v[1] = {a};
  double tot[1];
  if (grid_sum<1, 256>(v, sc->partials, &sc->ticket[0], tot) && threadIdx.x == 0) sc->rr = tot[0];
}

// ---- per-node static inputs: diagonal / its mean, coordinates / scale, material ---------------------

__global__ void __launch_bounds__(256) k_mp_dsum(int n, const double* __restrict__ invd, MpScratch* sc) {
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a += 1.0 / invd[i];
  const double v[1] = {a};
  double tot[1];
  if (grid_sum<1, 256>(v, sc->partials, &sc->ticket[2], tot) && threadIdx.x == 0) sc->dsum = tot[0];
}

__global__ void k_mp_static(int N, const double* __restrict__ invd, const double* __restrict__ xy,
                            const float* __restrict__ mat, const MpScratch* sc, double coord_scale,
                            float* __restrict__ sf) {
  const double d_mean = N > 0 ? sc->dsum / (2.0 * N) : 1.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    float* o = sf + (size_t)k * 6;
    o[0] = (float)((1.0 / invd[2 * k]) / d_mean);
    o[1] = (float)((1.0 / invd[2 * k + 1]) / d_mean);
    o[2] = (float)(xy[2 * k] / coord_scale);
    o[3] = (float)(xy[2 * k + 1] / coord_scale);
    o[4] = mat[2 * k];
    o[5] = mat[2 * k + 1];
  }
}

// ---- the layers' gather plan: one CTA per tile of 128 nodes -------------------------------------

__global__ void __launch_bounds__(256) k_mp_tile_plan(int N, const int* __restrict__ node_ptr,
                                                      const int* __restrict__ nbr, int4* __restrict__ hdr,
                                                      int2* __restrict__ runs, uint4* __restrict__ local) {
  constexpr int W = kPlanSpan / 32;
  __shared__ unsigned bits[W];
  __shared__ int wpre[W + 1], spre[W + 1], epre[W + 1];
  __shared__ int s_lo, s_hi, s_fail;
  __shared__ int rs[kPlanMaxRuns], re[kPlanMaxRuns];
  const int t = threadIdx.x, tile = blockIdx.x;
  const int a = tile * kTile, b = min(N, a + kTile);
  if (t == 0) {
    s_lo = INT_MAX;
    s_hi = -1;
    s_fail = 0;
  }
  for (int w = t; w < W; w += blockDim.x) bits[w] = 0u;
  __syncthreads();
  const int e0 = node_ptr[a], e1 = node_ptr[b];
  int lo = INT_MAX, hi = -1;
  for (int e = e0 + t; e < e1; e += blockDim.x) {
    const int v = nbr[e];
    lo = min(lo, v);
    hi = max(hi, v);
  }
  if (lo <= hi) {
    atomicMin(&s_lo, lo);
    atomicMax(&s_hi, hi);
  }
  if (t < b - a) {  // every node lists itself (first the own row) and at most kPlanMaxLocal others
    const int d = node_ptr[a + t + 1] - node_ptr[a + t];
    if (d < 1 || d - 1 > kPlanMaxLocal) s_fail = 1;
  }
  __syncthreads();
  const int wlo = s_lo;
  if (s_fail || s_hi - wlo + 1 > kPlanSpan) {
    if (t == 0) hdr[tile] = make_int4(0, 0, 1, 0);
    return;
  }
  for (int e = e0 + t; e < e1; e += blockDim.x) {
    const int d = nbr[e] - wlo;
    atomicOr(&bits[d >> 5], 1u << (d & 31));
  }
  __syncthreads();
  if (t == 0) {  // word prefix counts of the set bits, the run starts and the run ends
    int c = 0, cs = 0, ce = 0;
    for (int w = 0; w < W; ++w) {
      const unsigned x = bits[w];
      const unsigned prev_top = w > 0 ? bits[w - 1] >> 31 : 0u;
      const unsigned next_low = w + 1 < W ? (bits[w + 1] & 1u) << 31 : 0u;
      const unsigned st = x & ~((x << 1) | prev_top);
      const unsigned en = x & ~((x >> 1) | next_low);
      wpre[w] = c;
      spre[w] = cs;
      epre[w] = ce;
      c += __popc(x);
      cs += __popc(st);
      ce += __popc(en);
    }
    wpre[W] = c;
    spre[W] = cs;
    epre[W] = ce;
    if (c > kPlanMaxUnion || cs > kPlanMaxRuns) s_fail = 1;
  }
  __syncthreads();
  if (s_fail) {
    if (t == 0) hdr[tile] = make_int4(0, 0, 1, 0);
    return;
  }
  for (int w = t; w < W; w += blockDim.x) {  // the runs' first and last nodes, in order
    const unsigned x = bits[w];
    const unsigned prev_top = w > 0 ? bits[w - 1] >> 31 : 0u;
    const unsigned next_low = w + 1 < W ? (bits[w + 1] & 1u) << 31 : 0u;
    unsigned st = x & ~((x << 1) | prev_top), en = x & ~((x >> 1) | next_low);
    for (int j = spre[w]; st; ++j, st &= st - 1) rs[j] = wlo + 32 * w + __ffs(st) - 1;
    for (int j = epre[w]; en; ++j, en &= en - 1) re[j] = wlo + 32 * w + __ffs(en) - 1;
  }
  __syncthreads();
  const int nruns = spre[W];
  if (t < kPlanMaxRuns)
    runs[(size_t)tile * kPlanMaxRuns + t] = t < nruns ? make_int2(rs[t], re[t] - rs[t] + 1) : make_int2(0, 0);
  if (t == 0) hdr[tile] = make_int4(nruns, wpre[W], 0, 0);
  if (t < b - a) {  // the node's own row first, then its neighbours in pattern order
    const int n = a + t;
    auto rank = [&](int v) {
      const int d = v - wlo;
      return wpre[d >> 5] + __popc(bits[d >> 5] & ((1u << (d & 31)) - 1u));
    };
    uint16_t slot[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) slot[j] = (uint16_t)kPlanNone;
    int k = 1;
    for (int e = node_ptr[n]; e < node_ptr[n + 1]; ++e) {
      const int v = nbr[e];
      if (v != n) slot[k++] = (uint16_t)rank(v);
    }
    slot[0] = (uint16_t)(k - 1);  // the degree (the layers read their own rows elsewhere)
    local[n] = make_uint4((uint32_t)slot[0] | ((uint32_t)slot[1] << 16), (uint32_t)slot[2] | ((uint32_t)slot[3] << 16),
                          (uint32_t)slot[4] | ((uint32_t)slot[5] << 16), (uint32_t)slot[6] | ((uint32_t)slot[7] << 16));
  }
}

// ---- the learned cycle's post-smoother weights: out = factor / lambda_max * D^-1 ------------------

__global__ void k_mp_smoother_weights(int n, const double* __restrict__ invd, const double* lam, double factor,
                                      double* __restrict__ out) {
  const double w = factor / *lam;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = w * invd[i];
}

// ---- message-passing layer on the tensor cores ----------------------------------------------------
//
// A CTA owns a tile of 128 nodes at a time (persistent over tiles); its 8 tile warps build the A
// operand, issue the MMA and run the epilogue:
//  A tile:   16 rows per warp, four nodes at once with 8 lanes per node (lane c holds features
//            8c..8c+7, one 16-byte chunk): the node's own chunk and the sum of its neighbours'
//            chunks in ascending pattern order (the mean is the same sum in the same order as a
//            serial loop, wherever the rows come from).
//  MMA:      one thread issues 8 x tcgen05.mma (M=128, N=64, K=16) into 64 TMEM columns and waits
//            on the commit's mbarrier (bounded); the tile warps learn the outcome through shared
//            memory.
//  epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31, columns 32 (w / 4) .. +31 (its node's half
//            row), adds bias, ReLU and the residual, and stages the BF16 row half in shared memory
//            (16-byte chunks XOR-swizzled by row, so the stores do not collide on banks); the tile
//            then leaves in coalesced 16-byte stores. The last layer also runs the decoder there:
//            y = W_out H3 + b_out, summed over the 64 features in order (the first half by the
//            warps of columns 0..31, handed through shared memory to those of columns 32..63), and
//            z = zbase + invd (r + s y).
// The rows reach the A tile from global memory: four CTAs of 8 warps per SM; each lane loads its
// nodes' chunks, a warp's node pointers and neighbour lists in two loads (the next tile's lists
// prefetched with cp.async during the MMA and the epilogue). Patterns with a gather plan run the
// warp-specialised kernel below (k_mp_layer_ws) instead; both give the same bits.
constexpr int kLT = 256;                 // the tile warps' threads
constexpr int kNbrCache = 128;           // neighbour-list entries a warp keeps in shared memory
constexpr int kLayerCtasPerSm = 3;       // rows: resident CTAs per SM (registers capped to fit them)
// the bias slice: A's constant K-slice of ones (128 x 16 BF16) and B's bias rows (64 x 16 BF16)
constexpr int kBiasSmem = 4096 + 2048;
constexpr int kTcSmem = kASmem + kBSmem + kBiasSmem + 1024;  // dynamic shared memory (1024-byte aligned base)

struct MpLayerArgs {
  int N;
  const int* node_ptr;
  const int* nbr;
  MpTilePlan plan;
  const __nv_bfloat16* Hin;
  MpnnParams P;
  int layer;
  const int* skip;
  __nv_bfloat16* Hout;  // may be null in the last layer (inference)
  __nv_bfloat16* Gout;  // TRAIN: ReLU outputs
  __nv_bfloat16* Aout;  // TRAIN: neighbour means
  // decoder (last layer)
  const double* r;
  const double* invd;
  const double* rr;
  double inv_n;
  const double* zbase;  // may be null (z = the network's output alone)
  double* z;
  float* Yout;          // TRAIN
  long long spin_limit;
  int* err;
};

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// ---- encoder on the tensor cores: H0 = relu(W_in X + b_in) -----------------------------------------
//
// Persistent CTAs over tiles of 128 consecutive nodes. Thread 0 brings a tile's inputs (r: 16 B
// per node, the static inputs: 24 B per node, both contiguous) into shared memory with two bulk
// copies completing on an mbarrier, one tile ahead (two stages). Two threads per node form the
// node's BF16 input row X (thread pair half 0: r/s and the first two static inputs, half 1: the
// other four) as the A operand (K-major, no swizzle; K = 16: the 8 inputs, then three ones and
// zeros). B holds W_in (K 0..7) and the bias split exactly into three BF16 parts (K 8..10:
// b = b_hi + b_mid + b_lo), so one tcgen05.mma (M=128, N=64, K=16) gives W_in X + b in FP32 in
// tensor memory. Epilogue: each warp reads 32 lanes x 32 columns (tcgen05.ld.32x32b.x32), applies
// ReLU, stages the BF16 rows XOR-swizzled in shared memory and the tile leaves in coalesced
// 16-byte stores. Every wait is bounded; a timeout is recorded and the CTA leaves through the
// common exit. The static inputs' buffer holds 16 bytes past its 24 N (a ragged last tile's copy
// is rounded up to 16 bytes).
constexpr int kEncT = 256;                          // threads of the encoder
constexpr int kEncTile = 128;                       // nodes per tile (the MMA's M)
constexpr int kEncStage = kEncTile * 16 + kEncTile * 24;  // one stage: r, then the static inputs
constexpr int kEncCtasPerSm = 4;

template <bool TRAIN>
__global__ void __launch_bounds__(kEncT, kEncCtasPerSm) k_mp_encode(int N, const double* __restrict__ r, const double* rr,
                                                     double inv_n, const float* __restrict__ sf, MpnnParams P,
                                                     const int* skip, __nv_bfloat16* __restrict__ H0,
                                                     __nv_bfloat16* __restrict__ Xout, long long spin_limit,
                                                     int* err) {
  if (skip && *skip) return;  // uniform: before any barrier or tensor-memory allocation
  __shared__ __align__(128) uint8_t stage[2][kEncStage];
  __shared__ __align__(128) uint8_t sX[4096];   // A: k 0..7 at +0, k 8..15 at +2048 (rows of 16 B)
  __shared__ __align__(128) uint8_t sB[2048];   // B: k 0..7 at +0, k 8..15 at +1024
  __shared__ __align__(128) uint8_t sOut[kEncTile * 128];
  __shared__ uint64_t bar[2], mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int mma_ok;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int tiles = (N + kEncTile - 1) / kEncTile;
  // constant operand parts: the ones of A's second K half, W_in and the split bias in B
  if (t < kEncTile) {
    const int m = t;
    *reinterpret_cast<uint4*>(sX + 2048 + (m >> 3) * 128 + (m & 7) * 16) =
        make_uint4(0x3F803F80u, 0x00003F80u, 0u, 0u);  // BF16 1, 1, 1, 0, 0, 0, 0, 0
  } else if (t < kEncTile + F) {
    const int n = t - kEncTile;
    const uint4 wrow = *reinterpret_cast<const uint4*>(P.pb + kMpOffWin + n * kMpIn);
    *reinterpret_cast<uint4*>(sB + (n >> 3) * 128 + (n & 7) * 16) = wrow;
    const float b = P.pf[kMpOffBin + n];
    const __nv_bfloat16 b0 = __float2bfloat16_rn(b);
    const float r1 = b - __bfloat162float(b0);
    const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 b2 = __float2bfloat16_rn(r1 - __bfloat162float(b1));
    const uint32_t w0 = (uint32_t)__bfloat16_as_ushort(b0) | ((uint32_t)__bfloat16_as_ushort(b1) << 16);
    *reinterpret_cast<uint4*>(sB + 1024 + (n >> 3) * 128 + (n & 7) * 16) =
        make_uint4(w0, (uint32_t)__bfloat16_as_ushort(b2), 0u, 0u);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                 "r"(F));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  const uint32_t bar0 = smem_u32(&bar[0]), bar1 = smem_u32(&bar[1]), mbar_addr = smem_u32(&mbar);
  auto issue = [&](int tl, int st) {  // thread 0: tile tl's inputs into stage st
    const int first = tl * kEncTile, cnt = min(kEncTile, N - first);
    const uint32_t rb = (uint32_t)cnt * 16u, sb = ((uint32_t)cnt * 24u + 15u) & ~15u;
    const uint32_t b = st ? bar1 : bar0;
    // the stage's earlier generic reads are ordered before the copies' writes
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(rb + sb) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(stage[st])),
                 "l"(r + 2 * (size_t)first), "r"(rb), "r"(b)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(stage[st] + kEncTile * 16)),
                 "l"(sf + 6 * (size_t)first), "r"(sb), "r"(b)
                 : "memory");
  };
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar0), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar1), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar_addr), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    if ((int)blockIdx.x < tiles) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < tiles) issue(blockIdx.x + gridDim.x, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint64_t adesc = umma_desc(smem_u32(sX), 2048u, 128u);
  const uint64_t bdesc = umma_desc(smem_u32(sB), 1024u, 128u);
  const double s = sqrt(*rr * inv_n);
  const double sd = s > 0.0 ? s : 1.0;
  const int q = warp & 3, h = warp >> 2;  // epilogue: TMEM lane quarter, column half
  uint32_t phase = 0;
  int it = 0, used = 0;  // loop iterations; tiles whose inputs were consumed
  // (thread 0) tiles whose inputs were issued and not yet consumed
  int pending = ((int)blockIdx.x < tiles ? 1 : 0) + ((int)(blockIdx.x + gridDim.x) < tiles ? 1 : 0);
  for (int tl = blockIdx.x; tl < tiles; tl += gridDim.x, ++it) {
    const int st = it & 1;
    const uint32_t b = st ? bar1 : bar0;
    // thread 0 waits for the copies; the barrier hands their data (and the outcome) to the block
    const int got = t == 0 ? (mbar_wait(b, (uint32_t)(it >> 1) & 1u, spin_limit) ? 1 : 0) : 1;
    if (!__syncthreads_and(got)) {
      if (t == 0 && err) atomicMin(&err[kErrTimeout], tl);
      break;
    }
    --pending;
    ++used;
    const int first = tl * kEncTile, cnt = min(kEncTile, N - first);
    {  // the input rows: thread pair (node m, half hf)
      const int m = t & (kEncTile - 1), hf = t >> 7;
      const double* sr = reinterpret_cast<const double*>(stage[st]);
      const float* ss = reinterpret_cast<const float*>(stage[st] + kEncTile * 16);
      uint2 xv = make_uint2(0u, 0u);
      if (m < cnt) {
        float x0, x1, x2, x3;
        if (hf == 0) {
          x0 = (float)(sr[2 * m] / sd);
          x1 = (float)(sr[2 * m + 1] / sd);
          x2 = ss[6 * m];
          x3 = ss[6 * m + 1];
        } else {
          x0 = ss[6 * m + 2];
          x1 = ss[6 * m + 3];
          x2 = ss[6 * m + 4];
          x3 = ss[6 * m + 5];
        }
        xv = make_uint2(pack_bf2(x0, x1), pack_bf2(x2, x3));
        if (TRAIN) reinterpret_cast<uint2*>(Xout + (size_t)(first + m) * kMpIn)[hf] = xv;
      }
      *reinterpret_cast<uint2*>(sX + (m >> 3) * 128 + (m & 7) * 16 + hf * 8) = xv;
    }
    // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      if (tl + 2 * (int)gridDim.x < tiles) {  // the stage is read: the tile after next into it
        issue(tl + 2 * gridDim.x, st);
        ++pending;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_addr)
                   : "memory");
      int ok = mbar_wait(mbar_addr, phase, spin_limit) ? 1 : 0;
      if (!ok) {  // report, then let the MMA finish (bounded) before memory is released
        if (err) atomicMin(&err[kErrTimeout], tl);
        mbar_wait(mbar_addr, phase, kMbarSpinLimit);
      }
      mma_ok = ok;
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    phase ^= 1u;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!mma_ok) break;  // uniform
    {  // epilogue: ReLU, BF16, staged rows
      const int m = q * 32 + lane;
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * 32), v);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const int ch = 4 * h + cc;
        uint32_t o[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          o[j] = pack_bf2(fmaxf(__uint_as_float(v[cc * 8 + 2 * j]), 0.f),
                          fmaxf(__uint_as_float(v[cc * 8 + 2 * j + 1]), 0.f));
        *reinterpret_cast<uint4*>(sOut + m * 128 + ((ch ^ (m & 7)) * 16)) = make_uint4(o[0], o[1], o[2], o[3]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {  // the staged tile, in coalesced 16-byte stores
      const int u = t + kEncT * i, row = u >> 3, ch = u & 7;
      if (row < cnt)
        reinterpret_cast<uint4*>(H0 + (size_t)(first + row) * F)[ch] =
            *reinterpret_cast<const uint4*>(sOut + row * 128 + ((ch ^ (row & 7)) * 16));
    }
    __syncthreads();  // sOut, sX and tensor memory are free for the next tile
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  }
  if (t == 0) {  // copies still in flight (after a timeout) land before the CTA leaves (bounded)
    for (int j = 0; j < pending; ++j) {
      const int jt = used + j;
      mbar_wait((jt & 1) ? bar1 : bar0, (uint32_t)(jt >> 1) & 1u, kMbarSpinLimit);
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(F));
}


// Neighbour sums in FP32: acc[j] += feature j of the chunk v (8 BF16) with the mixed-precision
// add.rn.f32.bf16 (the BF16 operand widened exactly, one IEEE round-to-nearest add: the same result
// as widening and a scalar add, in one instruction per feature).
__device__ __forceinline__ void add_chunk_bf(float (&acc)[8], const uint4 v) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int q = 0; q < 4; ++q)
    asm("{\n\t.reg .b16 lo, hi;\n\t"
        "mov.b32 {lo, hi}, %2;\n\t"
        "add.rn.f32.bf16 %0, lo, %0;\n\t"
        "add.rn.f32.bf16 %1, hi, %1;\n\t}\n"
        : "+f"(acc[2 * q]), "+f"(acc[2 * q + 1])
        : "r"(w[q]));
}
// g + the low / high BF16 of w, widened exactly: one IEEE round-to-nearest add (the bits of
// bf_lo(w) + g, in one instruction).
__device__ __forceinline__ float add_bf_lo(uint32_t w, float g) {
  float d;
  asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\tadd.rn.f32.bf16 %0, lo, %2;\n\t}\n" : "=f"(d) : "r"(w), "f"(g));
  return d;
}
__device__ __forceinline__ float add_bf_hi(uint32_t w, float g) {
  float d;
  asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\tadd.rn.f32.bf16 %0, hi, %2;\n\t}\n" : "=f"(d) : "r"(w), "f"(g));
  return d;
}
// Eight BF16 -0.0: the chunk a missing neighbour contributes. x + (-0) = x exactly for every x
// (both zeros included), so a sum padded with it has the bits of the sum without it, and the
// neighbour loop needs no branch around its adds (a branch around inline assembly cannot be
// predicated: it diverges).
constexpr uint32_t kNegZero2 = 0x80008000u;
// 1/deg as the IEEE quotient 1.f / deg (constants folded by the compiler), no division at run time.
__device__ __forceinline__ float inv_deg(int deg) {
  if (deg > 7) return 1.f / (float)deg;
  float r = 0.f;
  r = deg == 1 ? 1.f : r;
  r = deg == 2 ? 1.f / 2.f : r;
  r = deg == 3 ? 1.f / 3.f : r;
  r = deg == 4 ? 1.f / 4.f : r;
  r = deg == 5 ? 1.f / 5.f : r;
  r = deg == 6 ? 1.f / 6.f : r;
  r = deg == 7 ? 1.f / 7.f : r;
  return r;
}
// The chunk's mean as 8 BF16: each sum times inv, rounded to nearest.
__device__ __forceinline__ uint4 mean_chunk(const float (&acc)[8], float inv) {
  return make_uint4(pack_bf2(acc[0] * inv, acc[1] * inv), pack_bf2(acc[2] * inv, acc[3] * inv),
                    pack_bf2(acc[4] * inv, acc[5] * inv), pack_bf2(acc[6] * inv, acc[7] * inv));
}

// A tile the plan takes: its union fits one stage in at most kPlanMaxRuns runs.
__device__ __forceinline__ bool plan_takes(const int4 h) {
  return h.z == 0 && h.x >= 1 && h.x <= kPlanMaxRuns && h.y >= 1 && h.y <= kPlanMaxUnion;
}

template <bool TRAIN, bool LAST>
__global__ void __launch_bounds__(kLT, kLayerCtasPerSm) k_mp_layer_tc(const MpLayerArgs a) {
  const int N = a.N;
  if (a.skip && *a.skip) {  // uniform: before any barrier or tensor-memory allocation
    if (LAST)                 // the network is off: the Jacobi step
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * N; i += gridDim.x * blockDim.x)
        a.z[i] = (a.zbase ? a.zbase[i] : 0.0) + a.invd[i] * a.r[i];
    return;
  }
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int mma_ok;
  __shared__ float wout[2 * F], bout[2];
  __shared__ float2 ypart[kTile];
  // each warp's neighbour lists for row-by-row tiles (the first kNbrCache entries)
  __shared__ int s_nbr[(kLT / 32) * kNbrCache];
  // 1024-byte aligned base as an offset into the shared array (the compiler keeps the shared
  // address space through pointer arithmetic on it: plain C++ accesses become ld/st.shared)
  uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* sA = base;               // chunk k/8 of row m at a_chunk(m, (k/8) % 8, k/64), + (k%8)*2
  uint8_t* sB = base + kASmem;      // element (n, k): (k/8)*1024 + (n/8)*128 + (n%8)*16 + (k%8)*2
  uint8_t* sOut = sA + kASmem / 2;  // staged output tile (the mean half of A, free after the MMA)
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const __nv_bfloat16* W = a.P.pb + kMpOffL0 + a.layer * kMpLStride;
  // the bias enters the MMA as a ninth K-slice: ones in A (K 0..2) against the FP32 bias split
  // exactly into three BF16 parts in B (b = b_hi + b_mid + b_lo)
  uint8_t* sOnes = sB + kBSmem;
  uint8_t* sBias = sOnes + 4096;
  if (t < kTile) {
    *reinterpret_cast<uint4*>(sOnes + (t >> 3) * 128 + (t & 7) * 16) = make_uint4(0x3F803F80u, 0x00003F80u, 0u, 0u);
    *reinterpret_cast<uint4*>(sOnes + 2048 + (t >> 3) * 128 + (t & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
  } else if (t < kTile + F) {
    const int n = t - kTile;
    const float b = a.P.pf[kMpOffL0 + a.layer * kMpLStride + F * 2 * F + n];
    const __nv_bfloat16 b0 = __float2bfloat16_rn(b);
    const float r1 = b - __bfloat162float(b0);
    const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 b2 = __float2bfloat16_rn(r1 - __bfloat162float(b1));
    const uint32_t w0 = (uint32_t)__bfloat16_as_ushort(b0) | ((uint32_t)__bfloat16_as_ushort(b1) << 16);
    *reinterpret_cast<uint4*>(sBias + (n >> 3) * 128 + (n & 7) * 16) =
        make_uint4(w0, (uint32_t)__bfloat16_as_ushort(b2), 0u, 0u);
    *reinterpret_cast<uint4*>(sBias + 1024 + (n >> 3) * 128 + (n & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
  }

  for (int idx = t; idx < F * 16; idx += blockDim.x) {  // 64 rows x 16 chunks of 8 BF16
    const int n = idx >> 4, kc = idx & 15;
    const uint4 v = *reinterpret_cast<const uint4*>(W + n * 2 * F + kc * 8);
    *reinterpret_cast<uint4*>(sB + kc * 1024 + (n >> 3) * 128 + (n & 7) * 16) = v;
  }
  if (LAST) {
    for (int i = t; i < 2 * F; i += blockDim.x) wout[i] = bf(a.P.pb[kMpOffWout + i]);
    if (t < 2) bout[t] = a.P.pf[kMpOffBout + t];
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
  const double s = LAST ? sqrt(*a.rr * a.inv_n) : 0.0;
  uint32_t phase = 0;
  const int g = lane >> 3, c = lane & 7;  // gather: node group of the warp, feature chunk
  const int q = warp & 3, h = warp >> 2;  // epilogue: TMEM lane quarter, column half
  int np = 0;         // lanes 0..16: node pointers of the warp's 16 nodes (+ the end) in this tile
  bool first = true;  // the first tile's lists come synchronously, later ones were prefetched

  for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x) {
    const int next = tile + (int)gridDim.x;
    {
      // ---- A tile row by row: the warp's 17 node pointers in one load, its nodes' neighbour lists
      // (contiguous in the pattern) in one more into shared memory, so each round of four nodes is
      // one round trip: the own chunk and up to eight neighbour chunks per lane in flight.
      const int wbase = tile * kTile + warp * 16;
      int* wnbr = s_nbr + warp * kNbrCache;
      if (first) {
        if (lane <= 16) np = __ldg(&a.node_ptr[min(wbase + lane, N)]);
        const int f0 = __shfl_sync(0xffffffffu, np, 0);
        const int fc = __shfl_sync(0xffffffffu, np, 16) - f0;
        for (int j = lane; j < min(fc, kNbrCache); j += 32) wnbr[j] = __ldg(&a.nbr[f0 + j]);
        first = false;
      } else {
        asm volatile("cp.async.wait_all;\n" ::: "memory");
      }
      __syncwarp();
      const int np0 = __shfl_sync(0xffffffffu, np, 0);
      // rows: the next tile's node pointers, used after this tile's rounds
      const int wnext = next * kTile + warp * 16;
      int np_next = 0;
      if (lane <= 16 && next * kTile < N) np_next = __ldg(&a.node_ptr[min(wnext + lane, N)]);
#pragma unroll 1
      for (int rnd = 0; rnd < 4; ++rnd) {
        const int li = rnd * 4 + g;
        const int m = warp * 16 + li;
        const int n = wbase + li;
        const int k0 = __shfl_sync(0xffffffffu, np, li) - np0;
        const int k1 = __shfl_sync(0xffffffffu, np, li + 1) - np0;
        uint4 own = make_uint4(0u, 0u, 0u, 0u);
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int deg = 0;
        if (n < N) {
          own = __ldg(reinterpret_cast<const uint4*>(a.Hin + (size_t)n * F) + c);
          for (int k = k0; k < k1; k += 8) {
            int mm[8];
            uint4 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int q8 = k + j;
              mm[j] = q8 < k1 ? (q8 < kNbrCache ? wnbr[q8] : __ldg(&a.nbr[np0 + q8])) : n;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
              v[j] = mm[j] != n ? __ldg(reinterpret_cast<const uint4*>(a.Hin + (size_t)mm[j] * F) + c)
                                : make_uint4(kNegZero2, kNegZero2, kNegZero2, kNegZero2);
#pragma unroll
            for (int j = 0; j < 8; ++j) {  // (a missing neighbour adds -0: no branch)
              deg += mm[j] != n ? 1 : 0;
              add_chunk_bf(acc, v[j]);
            }
          }
        }
        const float inv = inv_deg(deg);
        const uint4 av = mean_chunk(acc, inv);
        *reinterpret_cast<uint4*>(sA + a_chunk(m, c, 0)) = own;
        *reinterpret_cast<uint4*>(sA + a_chunk(m, c, 1)) = av;
        if (TRAIN && n < N) reinterpret_cast<uint4*>(a.Aout + (size_t)n * F)[c] = av;
      }
      {  // prefetch the next tile's neighbour lists (asynchronous copies, done during the MMA and the
         // epilogue); every lane has finished reading this tile's lists
        __syncwarp();
        const int n0 = __shfl_sync(0xffffffffu, np_next, 0);
        const int nc = __shfl_sync(0xffffffffu, np_next, 16) - n0;
        for (int j = lane; j < min(nc, kNbrCache); j += 32)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(wnbr + j)), "l"(a.nbr + n0 + j)
                       : "memory");
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        np = np_next;
      }
    }
    // the decoder's per-node inputs (last layer), loaded now so they arrive during the MMA
    double2 rn_e = make_double2(0.0, 0.0), dn_e = rn_e, zb_e = rn_e;
    if (LAST && (warp >> 2) == 1) {
      const int ne = tile * kTile + (warp & 3) * 32 + lane;
      if (ne < N) {
        rn_e = reinterpret_cast<const double2*>(a.r)[ne];
        dn_e = reinterpret_cast<const double2*>(a.invd)[ne];
        if (a.zbase) zb_e = reinterpret_cast<const double2*>(a.zbase)[ne];
      }
    }
    // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // K = 128 in slices of 16: four per 64-wide swizzled half
        const uint64_t ad = umma_desc_sw128(a_addr + (uint32_t)(j >> 2) * 16384u + (uint32_t)(j & 3) * 32u, 1024u);
        const uint64_t bd = umma_desc(b_addr + (uint32_t)(2 * j) * 1024u, 1024u, 128u);
        const uint32_t acc_flag = j > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc_flag), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      {  // + ones x bias parts
        const uint64_t ad = umma_desc(smem_u32(sOnes), 2048u, 128u);
        const uint64_t bd = umma_desc(smem_u32(sBias), 1024u, 128u);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(1u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       mbar_addr)
                   : "memory");
      int ok = mbar_wait(mbar_addr, phase, a.spin_limit) ? 1 : 0;
      if (!ok) {
        // the wait gave up: report it, then let the MMA finish (bounded) before the tile's
        // shared memory and tensor memory are released
        if (a.err) atomicMin(&a.err[kErrTimeout], tile);
        mbar_wait(mbar_addr, phase, kMbarSpinLimit);
      }
      mma_ok = ok;
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    phase ^= 1u;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!mma_ok) break;  // uniform: every tile thread reads the same flag

    // ---- epilogue: bias, ReLU, residual; stage the output half row
    const int m = q * 32 + lane;
    const int n = tile * kTile + m;
    uint32_t v[32];
    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * 32), v);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    uint32_t hw[16];
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
      const int ch = 4 * h + cc;
      const uint4 o4 = *reinterpret_cast<const uint4*>(sA + a_chunk(m, ch, 0));
      const uint32_t ow[4] = {o4.x, o4.y, o4.z, o4.w};
      uint32_t gw[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {  // (the accumulator holds the bias already)
        const float g0 = fmaxf(__uint_as_float(v[cc * 8 + 2 * j]), 0.f);
        const float g1 = fmaxf(__uint_as_float(v[cc * 8 + 2 * j + 1]), 0.f);
        hw[cc * 4 + j] = pack_bf2(bf_lo(ow[j]) + g0, bf_hi(ow[j]) + g1);
        gw[j] = pack_bf2(g0, g1);
      }
      if (TRAIN && n < N)
        reinterpret_cast<uint4*>(a.Gout + (size_t)n * F)[ch] = make_uint4(gw[0], gw[1], gw[2], gw[3]);
    }
    if (a.Hout) {
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const int ch = 4 * h + cc;
        *reinterpret_cast<uint4*>(sOut + m * 128 + ((ch ^ (m & 7)) * 16)) =
            make_uint4(hw[cc * 4], hw[cc * 4 + 1], hw[cc * 4 + 2], hw[cc * 4 + 3]);
      }
    }
    float y0 = 0.f, y1 = 0.f;
    if (LAST) {
      // decoder: y = b_out + sum over features 0..63 in order of W_out[:, f] H3[f]
      if (h == 0) {
        y0 = bout[0];
        y1 = bout[1];
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int f = 32 * h + 2 * j;
        if (h == 0) {
          y0 = fmaf(wout[f], bf_lo(hw[j]), y0);
          y0 = fmaf(wout[f + 1], bf_hi(hw[j]), y0);
          y1 = fmaf(wout[F + f], bf_lo(hw[j]), y1);
          y1 = fmaf(wout[F + f + 1], bf_hi(hw[j]), y1);
        }
      }
      if (h == 0) ypart[m] = make_float2(y0, y1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (LAST && h == 1 && n < N) {
      const float2 yp = ypart[m];
      y0 = yp.x;
      y1 = yp.y;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int f = 32 + 2 * j;
        y0 = fmaf(wout[f], bf_lo(hw[j]), y0);
        y0 = fmaf(wout[f + 1], bf_hi(hw[j]), y0);
        y1 = fmaf(wout[F + f], bf_lo(hw[j]), y1);
        y1 = fmaf(wout[F + f + 1], bf_hi(hw[j]), y1);
      }
      if (TRAIN) reinterpret_cast<float2*>(a.Yout)[n] = make_float2(y0, y1);
      double2 zn = make_double2(dn_e.x * (rn_e.x + s * (double)y0), dn_e.y * (rn_e.y + s * (double)y1));
      if (a.zbase) {
        zn.x += zb_e.x;
        zn.y += zb_e.y;
      }
      reinterpret_cast<double2*>(a.z)[n] = zn;
    }
    if (a.Hout) {  // the staged tile, in coalesced 16-byte stores
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int u = t + kLT * i, row = u >> 3, ch = u & 7;
        const int nr = tile * kTile + row;
        if (nr < N)
          reinterpret_cast<uint4*>(a.Hout + (size_t)nr * F)[ch] =
              *reinterpret_cast<const uint4*>(sOut + row * 128 + ((ch ^ (row & 7)) * 16));
      }
    }
    __syncthreads();  // tensor memory and the A tile are free for the next tile
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy in flight when the CTA leaves
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(F));
}

// ---- message-passing layer on planned patterns: one warp-specialised CTA per SM ------------------
//
// The same layer as k_mp_layer_tc (same operands, same order of every addition: the same bits),
// arranged as a pipeline of roles over the CTA's tiles so that the copies, the gathers, the MMAs
// and the epilogues of consecutive tiles overlap. Shared memory holds a ring of three stages of the
// tiles' own rows in the layout the MMA reads (used by the MMA and the epilogue), a ring of two
// stages of the tiles' unions in plain layout (used by the gathers alone, so a stage is refilled as
// soon as its gathers are done), two buffers of the A operand's mean half and, in tensor memory,
// two accumulators of 64 columns.
//  own producer (warp 20): copies a tile's own 128 rows with one 2-D tensor copy
//            (cp.async.bulk.tensor, no multicast) in the 128-byte swizzle (K-major: the A operand's
//            own half needs no copy through registers) into a stage its previous tile's epilogue has
//            released.
//  union producer (warp 22): copies the tile's union, one bulk copy per run of consecutive rows
//            (cp.async.bulk), and the node slots with one more, into a stage its previous tile's
//            gathers have released. Row kPlanNone of every stage holds -0.0 (the unused slots'
//            row). A tile the plan does not take gets no union: its neighbours come from global
//            memory.
//  gather (warps 0..15): 8 nodes per warp, four at once with 8 lanes per node (lane c: features
//            8c..8c+7); each node's 7 neighbour slots read (row address = one multiply-add, unused
//            slots at the -0.0 row) and summed in pattern order with add.rn.f32.bf16, times 1/deg,
//            rounded to BF16 into the mean half (K-major, 128-byte swizzle); one arrival per warp on
//            the union stage (free) and on the mean half (ready).
//  MMA (warp 21, one thread): 8 x tcgen05.mma (M=128, N=64, K=16: four K-slices of the own rows,
//            four of the means) and the bias slice (ones x the FP32 bias split into three BF16
//            parts) into the accumulator; tcgen05.commit arrives on the accumulator's barrier,
//            which frees the mean half and starts the epilogue.
//  epilogue (warps 16..19, warp 16+q on TMEM lanes 32q..32q+31, one thread per node): reads the
//            node's own row (the residual; its first half while the MMA runs) and the accumulator
//            (2 x tcgen05.ld.32x32b.x32), applies ReLU and the residual, writes each chunk into a
//            128-byte swizzled staging buffer, releases the accumulator and the own stage, and
//            stores the warp's 32 rows with one 2-D tensor store. The last layer runs the decoder per thread (features
//            0..63 in order) and writes z.
// Waits suspend in the hardware between polls (a 2 us hint), so the waiting warps take few
// issue slots; each is bounded (spin_limit polls). A role that gives up records the timeout and
// raises the CTA's abort flag, which every other wait polls. Before the CTA leaves, the copies and
// MMAs already issued have completed (bounded waits) and the tensor stores have read their staging.
// Measured on the 2M-DOF plate (120.8 us for the previous two-CTA kernel whose tile warps gathered,
// issued and ran the epilogue in turn): 8 gather warps and a union in swizzled 8-row boxes 186 us,
// one own box and bulk runs 154 us; the gather was the limit, two warps per scheduler with a
// swizzled-or-plain address per neighbour and a branch around each neighbour's adds. This layout
// (16 gather warps, plain union addressing, no branches) ran at 106 us, and at 88 us (0.47 of the
// measured HBM bandwidth) once the tile headers and runs were loaded a tile ahead; it is then
// bound by instruction issue and shared-memory latency, not by HBM.
constexpr int kWsGatherWarps = 16, kWsEpiWarps = 4;
constexpr int kWsEpi0 = kWsGatherWarps;                    // warps 16..19 (TMEM lane quarters 0..3)
constexpr int kWsOwnProd = kWsEpi0 + kWsEpiWarps;          // warp 20
constexpr int kWsMma = kWsOwnProd + 1;                     // warp 21
constexpr int kWsUnionProd = kWsMma + 1;                   // warp 22
constexpr int kWsT = (kWsUnionProd + 1) * 32;              // 736 threads (at most 88 registers each)
constexpr int kWsOwnStages = 3, kWsUStages = 2;
constexpr int kWsOwn = kTile * 128;                        // own stage: 128 rows
constexpr int kWsSlots = (kPlanMaxUnion + 1) * 128;        // union stage: the rows, the -0.0 row,
constexpr int kWsUStage = kWsSlots + kTile * 16;           // then the tile's node slots
constexpr int kWsStore = 32 * 128;                         // staging: a warp's 32 rows
constexpr int kWsOffOwn = kBSmem + kBiasSmem;              // after B, the ones and the bias parts
constexpr int kWsOffMean = kWsOffOwn + kWsOwnStages * kWsOwn;
constexpr int kWsOffSt = kWsOffMean + 2 * kTile * 128;
constexpr int kWsOffU = kWsOffSt + kWsEpiWarps * kWsStore;
constexpr int kWsSmem = kWsOffU + kWsUStages * kWsUStage + 1024;  // (+ the 1024-byte alignment)
static_assert(kWsOffOwn % 1024 == 0 && kWsOffMean % 1024 == 0 && kWsOffSt % 1024 == 0,
              "the 128-byte swizzle's atoms start on 1024-byte boundaries");
static_assert(kWsOffU % 16 == 0 && kWsUStage % 16 == 0, "bulk copies land on 16-byte boundaries");
static_assert(kWsSmem + 1024 <= 227 * 1024, "one CTA per SM");
constexpr uint32_t kWsSuspendNs = 2000;  // suspend hint of a wait's poll

// 2-D tensor copy of a box of rows into shared memory, completing on an mbarrier (no multicast).
__device__ __forceinline__ void tma_load_rows(uint32_t dst, const CUtensorMap* map, int row, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(bar)
      : "memory");
}
// 2-D tensor store of a box of rows from shared memory (rows past the tensor's end are not written).
__device__ __forceinline__ void tma_store_rows(const CUtensorMap* map, int row, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(0), "r"(row), "r"(src)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
// 16-byte shared-memory accesses by 32-bit shared address (ordered with the barrier waits)
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr)
               : "memory");
  return v;
}
__device__ __forceinline__ void sts128(uint32_t addr, const uint4 v) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

// Bounded wait that suspends between polls (up to kWsSuspendNs each); false when `limit` polls
// ran out or another role raised `abort_flag`.
__device__ __forceinline__ bool ws_poll(uint32_t bar, uint32_t parity, long long limit, const volatile int* abort_flag) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kWsSuspendNs)
        : "memory");
    if (ok) return true;
    if (*abort_flag) return false;
  }
  return false;
}
// A role's wait: true when the phase completed; false when another role stopped first or the limit
// ran out (then the timeout is recorded and every role told to stop). `warp_wide`: the whole warp
// waits and takes the same decision.
__device__ __forceinline__ bool ws_wait(uint32_t bar, uint32_t parity, long long limit, volatile int* abort_v,
                                        int* err, int tile, bool warp_wide = true) {
  const bool ok = ws_poll(bar, parity, limit, abort_v);
  if (!ok && !*abort_v) {
    if (err) atomicMin(&err[kErrTimeout], tile);
    *abort_v = 1;
  }
  return warp_wide ? __all_sync(0xffffffffu, ok) : ok;
}

template <bool TRAIN, bool LAST>
__global__ void __launch_bounds__(kWsT, 1)
    k_mp_layer_ws(const MpLayerArgs a, const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout) {
  const int N = a.N;
  if (a.skip && *a.skip) {  // uniform: before any barrier or tensor-memory allocation
    if (LAST)               // the network is off: the Jacobi step
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * N; i += gridDim.x * blockDim.x)
        a.z[i] = (a.zbase ? a.zbase[i] : 0.0) + a.invd[i] * a.r[i];
    return;
  }
  extern __shared__ uint8_t smem_raw[];
  // own ring (3): full / empty; union ring (2): full / empty; mean halves and accumulators (2):
  // mean ready, MMA done, accumulator empty
  __shared__ uint64_t o_full[kWsOwnStages], o_empty[kWsOwnStages], u_full[kWsUStages], u_empty[kWsUStages];
  __shared__ uint64_t m_full[2], mma_done[2], acc_empty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ __align__(16) float wout[2 * F];
  __shared__ float bout[2];
  __shared__ float s_inv[kPlanMaxLocal + 1];  // 1/deg (IEEE quotients), 0 for no neighbour
  uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* sB = base;  // element (n, k): (k/8)*1024 + (n/8)*128 + (n%8)*16 + (k%8)*2
  uint8_t* sOnes = base + kBSmem;
  uint8_t* sBias = sOnes + 4096;
  uint8_t* sOwn = base + kWsOffOwn;    // own stage s: row m at m*128, 128-byte swizzle
  uint8_t* sMean = base + kWsOffMean;  // mean half b: row m at m*128, 128-byte swizzle
  uint8_t* sSt = base + kWsOffSt;      // epilogue warp q's staging: 32 rows, 128-byte swizzle
  uint8_t* sU = base + kWsOffU;        // union stage s: slot j at j*128 (plain), then the node slots
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const __nv_bfloat16* W = a.P.pb + kMpOffL0 + a.layer * kMpLStride;
  if (t < kTile) {
    *reinterpret_cast<uint4*>(sOnes + (t >> 3) * 128 + (t & 7) * 16) = make_uint4(0x3F803F80u, 0x00003F80u, 0u, 0u);
    *reinterpret_cast<uint4*>(sOnes + 2048 + (t >> 3) * 128 + (t & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
  } else if (t < kTile + F) {
    const int n = t - kTile;
    const float b = a.P.pf[kMpOffL0 + a.layer * kMpLStride + F * 2 * F + n];
    const __nv_bfloat16 b0 = __float2bfloat16_rn(b);
    const float r1 = b - __bfloat162float(b0);
    const __nv_bfloat16 b1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 b2 = __float2bfloat16_rn(r1 - __bfloat162float(b1));
    const uint32_t w0 = (uint32_t)__bfloat16_as_ushort(b0) | ((uint32_t)__bfloat16_as_ushort(b1) << 16);
    *reinterpret_cast<uint4*>(sBias + (n >> 3) * 128 + (n & 7) * 16) =
        make_uint4(w0, (uint32_t)__bfloat16_as_ushort(b2), 0u, 0u);
    *reinterpret_cast<uint4*>(sBias + 1024 + (n >> 3) * 128 + (n & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
  } else if (t < kTile + F + 8 * kWsUStages) {  // the -0.0 row of each union stage
    const int j = t - kTile - F;
    *reinterpret_cast<uint4*>(sU + (size_t)(j >> 3) * kWsUStage + kPlanNone * 128 + (j & 7) * 16) =
        make_uint4(kNegZero2, kNegZero2, kNegZero2, kNegZero2);
  }
  for (int idx = t; idx < F * 16; idx += blockDim.x) {  // 64 rows x 16 chunks of 8 BF16
    const int n = idx >> 4, kc = idx & 15;
    const uint4 v = *reinterpret_cast<const uint4*>(W + n * 2 * F + kc * 8);
    *reinterpret_cast<uint4*>(sB + kc * 1024 + (n >> 3) * 128 + (n & 7) * 16) = v;
  }
  if (LAST) {
    for (int i = t; i < 2 * F; i += blockDim.x) wout[i] = bf(a.P.pb[kMpOffWout + i]);
    if (t < 2) bout[t] = a.P.pf[kMpOffBout + t];
  }
  if (t <= kPlanMaxLocal) s_inv[t] = inv_deg(t);
  // B, the ones and the bias parts (generic writes) are read by the tensor core (async proxy)
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (warp == kWsMma) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                 "r"(2 * F));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (t == 0) {
    for (int j = 0; j < kWsOwnStages; ++j) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&o_full[j])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&o_empty[j])), "r"(kWsEpiWarps));
    }
    for (int j = 0; j < kWsUStages; ++j) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&u_full[j])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&u_empty[j])), "r"(kWsGatherWarps));
    }
    for (int j = 0; j < 2; ++j) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&m_full[j])), "r"(kWsGatherWarps));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&mma_done[j])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&acc_empty[j])), "r"(kWsEpiWarps));
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  volatile int* abort_v = &abort_flag;
  const long long lim = a.spin_limit;
  const uint32_t ofull0 = smem_u32(&o_full[0]), oempty0 = smem_u32(&o_empty[0]), ufull0 = smem_u32(&u_full[0]),
                 uempty0 = smem_u32(&u_empty[0]), mfull0 = smem_u32(&m_full[0]), mdone0 = smem_u32(&mma_done[0]),
                 aempty0 = smem_u32(&acc_empty[0]);
  // tile k of this CTA: own stage k % 3 (use k / 3); union stage, mean half and accumulator k % 2
  // (use k / 2)

  if (warp < kWsGatherWarps) {
    // ---- gather: the mean half of the A operand
    const int g = lane >> 3, c = lane & 7;
    int kt = 0;
    int4 ph = (int)blockIdx.x * kTile < N ? __ldg(&a.plan.hdr[blockIdx.x]) : make_int4(0, 0, 1, 0);
    for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x, ++kt) {
      const int hs = kt & 1;
      const uint32_t hpar = (uint32_t)(kt >> 1) & 1u;
      const bool planned = plan_takes(ph);
      const int next = tile + (int)gridDim.x;  // its header arrives during this tile
      ph = next * kTile < N ? __ldg(&a.plan.hdr[next]) : make_int4(0, 0, 1, 0);
      if (!ws_wait(ufull0 + 8u * hs, hpar, lim, abort_v, a.err, tile)) break;
      if (kt >= 2 && !ws_wait(mdone0 + 8u * hs, hpar ^ 1u, lim, abort_v, a.err, tile)) break;  // mean half free
      const uint32_t row_a = smem_u32(sU + (size_t)hs * kWsUStage) + ((uint32_t)c << 4);  // chunk c of slot 0
      const uint32_t slot_a = smem_u32(sU + (size_t)hs * kWsUStage + kWsSlots);
      const uint32_t mean_a = smem_u32(sMean + (size_t)hs * kTile * 128);
      uint4 lp[2];  // both rounds' slots first
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int m = warp * 8 + u * 4 + g;
        constexpr uint32_t kNone2 = (uint32_t)kPlanNone * 0x10001u;
        lp[u] = planned && tile * kTile + m < N ? lds128(slot_a + (uint32_t)m * 16u)
                                                : make_uint4((uint32_t)kPlanNone << 16, kNone2, kNone2, kNone2);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int m = warp * 8 + u * 4 + g;
        const int n = tile * kTile + m;
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int deg = 0;
        if (planned) {
          const uint32_t sl[7] = {lp[u].x >> 16, lp[u].y & 0xFFFFu, lp[u].y >> 16, lp[u].z & 0xFFFFu,
                                  lp[u].z >> 16, lp[u].w & 0xFFFFu, lp[u].w >> 16};
          uint4 v[7];
#pragma unroll
          for (int j = 0; j < 7; ++j) v[j] = lds128(row_a + sl[j] * 128u);  // (unused: the -0.0 row)
          deg = (int)(lp[u].x & 0xFFFFu);
#pragma unroll
          for (int j = 0; j < 7; ++j) add_chunk_bf(acc, v[j]);
        } else if (n < N) {  // neighbours from global memory, in pattern order
          const int k0 = __ldg(&a.node_ptr[n]), k1 = __ldg(&a.node_ptr[n + 1]);
          for (int k = k0; k < k1; k += 8) {
            int mm[8];
            uint4 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) mm[j] = k + j < k1 ? __ldg(&a.nbr[k + j]) : n;
#pragma unroll
            for (int j = 0; j < 8; ++j)
              v[j] = mm[j] != n ? __ldg(reinterpret_cast<const uint4*>(a.Hin + (size_t)mm[j] * F) + c)
                                : make_uint4(kNegZero2, kNegZero2, kNegZero2, kNegZero2);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              deg += mm[j] != n ? 1 : 0;
              add_chunk_bf(acc, v[j]);
            }
          }
        }
        const uint4 av = mean_chunk(acc, deg <= kPlanMaxLocal ? s_inv[deg] : inv_deg(deg));
        sts128(mean_a + (uint32_t)m * 128u + ((uint32_t)(c ^ (m & 7)) << 4), av);
        if (TRAIN && n < N) reinterpret_cast<uint4*>(a.Aout + (size_t)n * F)[c] = av;
      }
      // the mean half (generic writes) is read by the tensor core (async proxy)
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(uempty0 + 8u * hs);  // the union stage is free
        mbar_arrive(mfull0 + 8u * hs);   // the mean half is ready
      }
    }
  } else if (warp < kWsOwnProd) {
    // ---- epilogue: one node per thread, its row chunk by chunk
    const int q = warp - kWsEpi0;
    const int m = q * 32 + lane;
    const double sc = LAST ? sqrt(*a.rr * a.inv_n) : 0.0;
    const uint32_t st = smem_u32(sSt + (size_t)q * kWsStore) + (uint32_t)lane * 128u;  // the thread's staged row
    int kt = 0;
    for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x, ++kt) {
      const int os = kt % kWsOwnStages, hs = kt & 1;
      const uint32_t opar = (uint32_t)(kt / kWsOwnStages) & 1u, hpar = (uint32_t)(kt >> 1) & 1u;
      const int n = tile * kTile + m;
      const int row0 = tile * kTile + q * 32;
      const bool store = a.Hout && row0 < N;  // warp-uniform
      // the decoder's per-node inputs, loaded before the waits
      double2 rn_e = make_double2(0.0, 0.0), dn_e = rn_e, zb_e = rn_e;
      if (LAST && n < N) {
        rn_e = reinterpret_cast<const double2*>(a.r)[n];
        dn_e = reinterpret_cast<const double2*>(a.invd)[n];
        if (a.zbase) zb_e = reinterpret_cast<const double2*>(a.zbase)[n];
      }
      if (store && lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");  // staging free
      if (!ws_wait(ofull0 + 8u * os, opar, lim, abort_v, a.err, tile)) break;
      // the residual (the node's own row): the first half read while the MMA runs, the second
      // while the accumulator's second half is read
      const uint32_t own_a = smem_u32(sOwn + (size_t)os * kWsOwn) + (uint32_t)m * 128u;
      uint4 res[4];
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) res[cc] = lds128(own_a + ((uint32_t)(cc ^ (m & 7)) << 4));
      if (!ws_wait(mdone0 + 8u * hs, hpar, lim, abort_v, a.err, tile)) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      float y0 = LAST ? bout[0] : 0.f, y1 = LAST ? bout[1] : 0.f;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(hs * F + hh * 32), v);
        if (hh == 1)
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) res[cc] = lds128(own_a + ((uint32_t)((4 + cc) ^ (m & 7)) << 4));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const int ch = 4 * hh + cc;
          const uint32_t ow[4] = {res[cc].x, res[cc].y, res[cc].z, res[cc].w};
          uint32_t hw[4], gw[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {  // (the accumulator holds the bias already)
            const float g0 = fmaxf(__uint_as_float(v[cc * 8 + 2 * j]), 0.f);
            const float g1 = fmaxf(__uint_as_float(v[cc * 8 + 2 * j + 1]), 0.f);
            hw[j] = pack_bf2(add_bf_lo(ow[j], g0), add_bf_hi(ow[j], g1));
            gw[j] = pack_bf2(g0, g1);
          }
          if (TRAIN && n < N)
            reinterpret_cast<uint4*>(a.Gout + (size_t)n * F)[ch] = make_uint4(gw[0], gw[1], gw[2], gw[3]);
          if (LAST) {  // decoder: y = b_out + sum over features 0..63 in order of W_out[:, f] H3[f]
            const float4* w4 = reinterpret_cast<const float4*>(wout);
#pragma unroll
            for (int o = 0; o < 2; ++o) {  // output o's chain over the chunk's 8 features, in order
              const float4 p0 = w4[o * (F >> 2) + 2 * ch], p1 = w4[o * (F >> 2) + 2 * ch + 1];
              const float w[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
              float y = o ? y1 : y0;
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                y = fmaf(w[2 * j], bf_lo(hw[j]), y);
                y = fmaf(w[2 * j + 1], bf_hi(hw[j]), y);
              }
              if (o) y1 = y; else y0 = y;
            }
          }
          if (store) sts128(st + ((uint32_t)(ch ^ (lane & 7)) << 4), make_uint4(hw[0], hw[1], hw[2], hw[3]));
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(aempty0 + 8u * hs);  // the accumulator is free
        mbar_arrive(oempty0 + 8u * os);  // the own stage is free (its MMA has completed)
      }
      if (LAST && n < N) {
        if (TRAIN) reinterpret_cast<float2*>(a.Yout)[n] = make_float2(y0, y1);
        double2 zn = make_double2(dn_e.x * (rn_e.x + sc * (double)y0), dn_e.y * (rn_e.y + sc * (double)y1));
        if (a.zbase) {
          zn.x += zb_e.x;
          zn.y += zb_e.y;
        }
        reinterpret_cast<double2*>(a.z)[n] = zn;
      }
      if (store) {  // the warp's 32 rows: one tensor store
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          tma_store_rows(&tout, row0, smem_u32(sSt + (size_t)q * kWsStore));
          asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
        }
      }
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
  } else if (warp == kWsOwnProd) {
    // ---- own producer: the tiles' own rows, one tensor copy each
    int kt = 0;
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tin)) : "memory");
      for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x, ++kt) {
        const int os = kt % kWsOwnStages;
        if (kt >= kWsOwnStages &&
            !ws_wait(oempty0 + 8u * os, (uint32_t)(kt / kWsOwnStages - 1) & 1u, lim, abort_v, a.err, tile, false))
          break;
        const uint32_t fb = ofull0 + 8u * os;
        // the epilogue's generic reads of this stage are ordered before the copy's writes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"((uint32_t)kWsOwn)
                     : "memory");
        tma_load_rows(smem_u32(sOwn + (size_t)os * kWsOwn), &tin, tile * kTile, fb);  // (past N: zeros)
      }
      // the copies issued land before the CTA leaves (bounded)
      for (int j = max(0, kt - kWsOwnStages); j < kt; ++j)
        mbar_wait(ofull0 + 8u * (j % kWsOwnStages), (uint32_t)(j / kWsOwnStages) & 1u, kMbarSpinLimit);
    }
  } else if (warp == kWsUnionProd) {
    // ---- union producer: each tile's union and its node slots
    int kt = 0;
    // lane j: run j (first node, rows) of the tile; the next tile's header and runs are loaded
    // while this tile waits for its stage
    auto tile_runs = [&](int tl, int4& h, int2& r) {
      h = tl * kTile < N ? __ldg(&a.plan.hdr[tl]) : make_int4(0, 0, 1, 0);
      r = plan_takes(h) && lane < h.x ? __ldg(&a.plan.runs[(size_t)tl * kPlanMaxRuns + lane]) : make_int2(0, 0);
    };
    int4 ph_next;
    int2 rn_next;
    tile_runs(blockIdx.x, ph_next, rn_next);
    for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x, ++kt) {
      const int us = kt & 1;
      const int4 ph = ph_next;
      const int2 rn = rn_next;
      tile_runs(tile + (int)gridDim.x, ph_next, rn_next);
      if (kt >= kWsUStages && !ws_wait(uempty0 + 8u * us, (uint32_t)((kt >> 1) - 1) & 1u, lim, abort_v, a.err, tile))
        break;
      const bool planned = plan_takes(ph);
      const int cnt = min(kTile, N - tile * kTile);
      int off = rn.y;  // inclusive prefix of the run lengths over the lanes
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, off, d);
        if (lane >= d) off += v;
      }
      off -= rn.y;
      const uint32_t stg = smem_u32(sU + (size_t)us * kWsUStage);
      const uint32_t fb = ufull0 + 8u * us;
      if (lane == 0) {
        // the gathers' generic reads of this stage are ordered before the copies' writes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb),
                     "r"(planned ? (uint32_t)ph.y * 128u + (uint32_t)cnt * 16u : 0u)
                     : "memory");
        if (planned)
          asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                           stg + kWsSlots),
                       "l"(a.plan.local + (size_t)tile * kTile), "r"((uint32_t)cnt * 16u), "r"(fb)
                       : "memory");
      }
      __syncwarp();
      if (rn.y > 0)  // run j lands after the earlier runs
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                         stg + (uint32_t)off * 128u),
                     "l"(a.Hin + (size_t)rn.x * F), "r"((uint32_t)rn.y * 128u), "r"(fb)
                     : "memory");
    }
    // the copies issued land before the CTA leaves (bounded)
    if (lane == 0)
      for (int j = max(0, kt - kWsUStages); j < kt; ++j)
        mbar_wait(ufull0 + 8u * (j & 1), (uint32_t)(j >> 1) & 1u, kMbarSpinLimit);
  } else if (lane == 0) {
    // ---- MMA: one thread
    const uint32_t b_addr = smem_u32(sB);
    int kt = 0;
    for (int tile = blockIdx.x; tile * kTile < N; tile += gridDim.x, ++kt) {
      const int os = kt % kWsOwnStages, hs = kt & 1;
      const uint32_t opar = (uint32_t)(kt / kWsOwnStages) & 1u, hpar = (uint32_t)(kt >> 1) & 1u;
      if (!ws_wait(mfull0 + 8u * hs, hpar, lim, abort_v, a.err, tile, false) ||
          !ws_wait(ofull0 + 8u * os, opar, lim, abort_v, a.err, tile, false) ||
          (kt >= 2 && !ws_wait(aempty0 + 8u * hs, hpar ^ 1u, lim, abort_v, a.err, tile, false)))
        break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t d = tmem + (uint32_t)(hs * F);
      const uint32_t own = smem_u32(sOwn + (size_t)os * kWsOwn), mean = smem_u32(sMean + (size_t)hs * kTile * 128);
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // K = 128 in slices of 16: four of the own rows, four of the means
        const uint64_t ad = umma_desc_sw128((j < 4 ? own : mean) + (uint32_t)(j & 3) * 32u, 1024u);
        const uint64_t bd = umma_desc(b_addr + (uint32_t)(2 * j) * 1024u, 1024u, 128u);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(j > 0 ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      {  // + ones x bias parts
        const uint64_t ad = umma_desc(smem_u32(sOnes), 2048u, 128u);
        const uint64_t bd = umma_desc(smem_u32(sBias), 1024u, 128u);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(1u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mdone0 + 8u * hs)
                   : "memory");
    }
    // the MMAs issued complete before their shared and tensor memory are released (bounded)
    for (int j = max(0, kt - 2); j < kt; ++j) mbar_wait(mdone0 + 8u * (j & 1), (uint32_t)(j >> 1) & 1u, kMbarSpinLimit);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == kWsMma) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * F));
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

// Weight gradient of a message-passing layer on the tensor cores:
//   dW^T[k][o] = sum_n Xc[n][k] dU[n][o]  (k < 128: Xc = [Hprev | A], o < 64),  db[o] = sum_n dU[n][o].
// One CTA of 256 threads per contiguous node range (the same ranges as k_mp_wgrad, so the
// partial sums per block keep their block order). Per chunk of 128 nodes: the Xc rows (BF16) and
// the dU rows (FP32, rounded to BF16; db summed in FP32 on the CUDA cores in node order) are
// staged row-major, transposed into the K-major core-matrix layouts of the MMA operands
// (A = Xc^T: 128 features x 128 nodes, B = dU^T: 64 outputs x 128 nodes; 8 nodes per 16-byte unit),
// and one thread issues 8 tcgen05.mma (M=128, N=64, K=16) accumulating into 64 TMEM columns over
// all chunks. Each warp of the first four then reads its 32 feature rows x 64 outputs.
constexpr int kWgNodes = 128;
constexpr int kWgSmem = kWgNodes * 2 * F * 2 /*Xc rows*/ + kWgNodes * F * 2 /*dU rows*/ + kASmem + kBSmem + 1024;

__global__ void __launch_bounds__(256, 1) k_mp_wgrad_tc(int N, const float* __restrict__ dU,
                                                        const __nv_bfloat16* __restrict__ X1,
                                                        const __nv_bfloat16* __restrict__ X2, long long spin_limit,
                                                        float* __restrict__ part, int* err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int mma_ok;
  __shared__ float bsum[4][F];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = base;                                  // A: element (feat m, node k), K-major core matrices
  uint8_t* sB = sA + kASmem;                           // B: element (output n, node k)
  __nv_bfloat16* rowX = reinterpret_cast<__nv_bfloat16*>(sB + kBSmem);  // [128 nodes][128 feats]
  __nv_bfloat16* rowU = rowX + kWgNodes * 2 * F;                          // [128 nodes][64 outputs]
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
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
  const int per = (N + gridDim.x - 1) / gridDim.x;
  const int n0 = blockIdx.x * per, n1 = min(N, n0 + per);
  // db: thread (column o = t % 64, node lane t / 64) sums its nodes in order
  float db = 0.f;
  bool any = false, ok_all = true;
  for (int c0 = n0; c0 < n1; c0 += kWgNodes) {
    // stage rows (zero past the range)
    for (int u = t; u < kWgNodes * 16; u += 256) {  // Xc: 16 chunks of 8 BF16 per node
      const int j = u >> 4, ch = u & 15, n = c0 + j;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (n < n1) v = ch < 8 ? __ldg(reinterpret_cast<const uint4*>(X1 + (size_t)n * F) + ch)
                             : __ldg(reinterpret_cast<const uint4*>(X2 + (size_t)n * F) + (ch - 8));
      reinterpret_cast<uint4*>(rowX)[u] = v;
    }
    for (int u = t; u < kWgNodes * F / 4; u += 256) {  // dU: float4 -> 4 BF16
      const int j = u / (F / 4), q = u % (F / 4), n = c0 + j;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (n < n1) v = __ldg(reinterpret_cast<const float4*>(dU + (size_t)n * F) + q);
      uint2 pk;
      pk.x = pack_bf2(v.x, v.y);
      pk.y = pack_bf2(v.z, v.w);
      reinterpret_cast<uint2*>(rowU)[u] = pk;
    }
    {
      const int o = t & 63, jl = t >> 6;
      for (int j = jl; j < kWgNodes; j += 4)
        if (c0 + j < n1) db += __ldg(&dU[(size_t)(c0 + j) * F + o]);
    }
    __syncthreads();
    // transpose into the K-major operands: unit (row m, node group g) = 8 consecutive nodes
    for (int u = t; u < 2 * F * (kWgNodes / 8); u += 256) {
      const int m = u % (2 * F), g = u / (2 * F);
      uint32_t w4[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const uint16_t lo = reinterpret_cast<const uint16_t*>(rowX)[(size_t)(8 * g + 2 * h) * 2 * F + m];
        const uint16_t hi = reinterpret_cast<const uint16_t*>(rowX)[(size_t)(8 * g + 2 * h + 1) * 2 * F + m];
        w4[h] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
      *reinterpret_cast<uint4*>(sA + g * 2048 + (m >> 3) * 128 + (m & 7) * 16) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
    for (int u = t; u < F * (kWgNodes / 8); u += 256) {
      const int m = u % F, g = u / F;
      uint32_t w4[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const uint16_t lo = reinterpret_cast<const uint16_t*>(rowU)[(size_t)(8 * g + 2 * h) * F + m];
        const uint16_t hi = reinterpret_cast<const uint16_t*>(rowU)[(size_t)(8 * g + 2 * h + 1) * F + m];
        w4[h] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
      *reinterpret_cast<uint4*>(sB + g * 1024 + (m >> 3) * 128 + (m & 7) * 16) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int j = 0; j < kWgNodes / 16; ++j) {
        const uint64_t ad = umma_desc(a_addr + (uint32_t)(2 * j) * 2048u, 2048u, 128u);
        const uint64_t bd = umma_desc(b_addr + (uint32_t)(2 * j) * 1024u, 1024u, 128u);
        const uint32_t acc_flag = (any || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc_flag), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_addr)
                   : "memory");
      int ok = mbar_wait(mbar_addr, phase, spin_limit) ? 1 : 0;
      if (!ok) {
        if (err) atomicMin(&err[kErrTimeout], blockIdx.x);
        mbar_wait(mbar_addr, phase, kMbarSpinLimit);
      }
      mma_ok = ok;
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    phase ^= 1u;
    any = true;
    __syncthreads();  // the operands are free for the next chunk
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!mma_ok) {
      ok_all = false;
      break;
    }
  }
  // db: the four node lanes added in order
  bsum[t >> 6][t & 63] = db;
  __syncthreads();
  float* p = part + (size_t)blockIdx.x * (F * 2 * F + F);
  if (t < F) p[F * 2 * F + t] = ((bsum[0][t] + bsum[1][t]) + bsum[2][t]) + bsum[3][t];
  // dW: warp w < 4 holds features 32 w .. 32 w + 31 (TMEM lanes) x 64 outputs (columns)
  if (warp < 4) {
    uint32_t v[32];
    for (int half = 0; half < 2; ++half) {
      if (any && ok_all) {
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(half * 32), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = 0u;
      }
      const int k = warp * 32 + lane;
#pragma unroll
      for (int j = 0; j < 32; ++j) p[(half * 32 + j) * 2 * F + k] = __uint_as_float(v[j]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(F));
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

int g_sms[64] = {};          // SM count per device (set by mpnn_prepare_device)
bool g_tc_attr[8][64] = {};  // the layer kernels' attributes set: [TRAIN * 4 + LAST * 2 + WS][device]

int dev_slot() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev >= 0 && dev < 64 ? dev : 0;
}

template <bool TRAIN, bool LAST, bool WS>
cudaError_t set_tc_attr() {
  bool& done = g_tc_attr[(TRAIN ? 4 : 0) + (LAST ? 2 : 0) + (WS ? 1 : 0)][dev_slot()];
  if (done) return cudaSuccess;
  const void* fn = WS ? reinterpret_cast<const void*>(k_mp_layer_ws<TRAIN, LAST>)
                      : reinterpret_cast<const void*>(k_mp_layer_tc<TRAIN, LAST>);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, WS ? kWsSmem : kTcSmem);
  if (e != cudaSuccess) return e;
  // the whole unified L1 / shared array as shared memory: three CTAs of ~54 KB per SM (rows), one
  // of ~203 KB (warp-specialised)
  e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  done = true;
  return cudaSuccess;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver
// library); null when the driver does not provide it.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of an activation array H [N][64] BF16 (rows of 128 bytes) with boxes of `box_rows`
// rows x 64 features, written to / read from shared memory in the 128-byte swizzle.
cudaError_t rows_map(CUtensorMap* map, const __nv_bfloat16* H, int N, int box_rows) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  if (reinterpret_cast<uintptr_t>(H) & 15u) return cudaErrorInvalidValue;
  const cuuint64_t dim[2] = {(cuuint64_t)F, (cuuint64_t)N};
  const cuuint64_t stride[1] = {(cuuint64_t)F * 2};
  const cuuint32_t box[2] = {(cuuint32_t)F, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(H), dim, stride, box,
                         elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int enc_grid(int N) {  // one wave of kEncCtasPerSm CTAs per SM at most
  const int sms = g_sms[dev_slot()] > 0 ? g_sms[dev_slot()] : kSMs;
  const int tiles = (N + kEncTile - 1) / kEncTile;
  return std::max(1, std::min(tiles, kEncCtasPerSm * sms));
}

// One wave of the layer kernel: kLayerCtasPerSm CTAs on every SM (rows; the register cap of
// __launch_bounds__ and the shared memory per CTA are sized for it), one (warp-specialised).
int tc_grid(int N, bool ws) {
  const int sms = g_sms[dev_slot()] > 0 ? g_sms[dev_slot()] : kSMs;
  const int tiles = (N + kTile - 1) / kTile;
  return std::max(1, std::min(tiles, (ws ? 1 : kLayerCtasPerSm) * sms));
}

template <bool TRAIN, bool LAST>
cudaError_t launch_layer_t(const MpLayerArgs& a, bool plan, cudaStream_t s) {
  if (!plan) {
    k_mp_layer_tc<TRAIN, LAST><<<tc_grid(a.N, false), kLT, kTcSmem, s>>>(a);
    return cudaSuccess;
  }
  CUtensorMap tin, tout;
  cudaError_t e = rows_map(&tin, a.Hin, a.N, kTile);
  if (e == cudaSuccess) e = rows_map(&tout, a.Hout ? a.Hout : a.Hin, a.N, 32);
  if (e != cudaSuccess) return e;
  k_mp_layer_ws<TRAIN, LAST><<<tc_grid(a.N, true), kWsT, kWsSmem, s>>>(a, tin, tout);
  return cudaSuccess;
}

cudaError_t launch_layer(const MpLayerArgs& a, bool train, bool last, cudaStream_t s) {
  const bool plan = a.plan.hdr != nullptr;
  if (train && last) return launch_layer_t<true, true>(a, plan, s);
  if (train) return launch_layer_t<true, false>(a, plan, s);
  if (last) return launch_layer_t<false, true>(a, plan, s);
  return launch_layer_t<false, false>(a, plan, s);
}

}  // namespace

cudaError_t mpnn_prepare_device() {
  static bool wg_done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !wg_done[dev]) {
    const cudaError_t ew = cudaFuncSetAttribute(k_mp_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem);
    if (ew != cudaSuccess) return ew;
    wg_done[dev] = true;
  }
  if (dev >= 0 && dev < 64 && g_sms[dev] == 0) {
    int sms = 0;
    const cudaError_t es = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (es != cudaSuccess) return es;
    g_sms[dev] = std::max(1, sms);
  }
  cudaError_t e = set_tc_attr<false, false, false>();
  if (e == cudaSuccess) e = set_tc_attr<false, true, false>();
  if (e == cudaSuccess) e = set_tc_attr<true, false, false>();
  if (e == cudaSuccess) e = set_tc_attr<true, true, false>();
  if (e == cudaSuccess) e = set_tc_attr<false, false, true>();
  if (e == cudaSuccess) e = set_tc_attr<false, true, true>();
  if (e == cudaSuccess) e = set_tc_attr<true, false, true>();
  if (e == cudaSuccess) e = set_tc_attr<true, true, true>();
  return e;
}

cudaError_t launch_mp_params(const float* p32, __nv_bfloat16* pb, float* pf, cudaStream_t s) {
  k_mp_convert<<<grid_nodes(kMpParams, 256), 256, 0, s>>>(kMpParams, p32, pb, pf);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_rr(int n, const double* r, MpScratch* sc, cudaStream_t s, const int* skip) {
  if (reinterpret_cast<uintptr_t>(r) & 15u)
    k_mp_rr<false><<<kRedGrid, 256, 0, s>>>(n, r, sc, skip);
  else
    k_mp_rr<true><<<kRedGrid, 256, 0, s>>>(n, r, sc, skip);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_static(int N, const double* invd, const double* xy, const float* mat, double coord_scale,
                             MpScratch* sc, float* sf, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  k_mp_dsum<<<kRedGrid, 256, 0, s>>>(2 * N, invd, sc);
  k_mp_static<<<grid_nodes(N, 256), 256, 0, s>>>(N, invd, xy, mat, sc, coord_scale, sf);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_mp_tile_plan(int N, const int* node_ptr, const int* nbr, int4* hdr, int2* runs, uint4* local,
                                cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  k_mp_tile_plan<<<(N + kTile - 1) / kTile, 256, 0, s>>>(N, node_ptr, nbr, hdr, runs, local);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_smoother_weights(int n, const double* invd, const double* lam, double factor, double* out,
                                       cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_mp_smoother_weights<<<grid_nodes(n, 256), 256, 0, s>>>(n, invd, lam, factor, out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_mp_forward(const MpnnGraph& g, const MpnnParams& P, const double* r, const double* invd,
                              const double* rr, const float* sf, const int* skip, MpnnWork& w, bool train,
                              const double* zbase, double* z, long long spin_limit, int* err, cudaStream_t s) {
  const int N = g.n_nodes;
  if (N <= 0) return cudaSuccess;
  const double inv_n = 1.0 / (2.0 * N);
  if (reinterpret_cast<uintptr_t>(r) & 15u) return cudaErrorInvalidValue;  // the bulk copies' alignment
  const int ge = enc_grid(N);
  if (train)
    k_mp_encode<true><<<ge, kEncT, 0, s>>>(N, r, rr, inv_n, sf, P, skip, w.H[0], w.X, spin_limit, err);
  else
    k_mp_encode<false><<<ge, kEncT, 0, s>>>(N, r, rr, inv_n, sf, P, skip, w.H[0], nullptr, spin_limit, err);
  MpLayerArgs a{};
  a.N = N;
  a.node_ptr = g.node_ptr;
  a.nbr = g.nbr;
  a.plan = g.plan;
  a.P = P;
  a.skip = skip;
  a.r = r;
  a.invd = invd;
  a.rr = rr;
  a.inv_n = inv_n;
  a.zbase = zbase;
  a.z = z;
  a.Yout = train ? w.Y : nullptr;
  a.spin_limit = spin_limit;
  a.err = err;
  for (int l = 0; l < kMpL; ++l) {
    const bool last = l + 1 == kMpL;
    a.layer = l;
    a.Hin = train ? w.H[l] : w.H[l & 1];
    a.Hout = train ? w.H[l + 1] : (last ? nullptr : w.H[(l + 1) & 1]);
    a.Gout = train ? w.G[l] : nullptr;
    a.Aout = train ? w.A[l] : nullptr;
    const cudaError_t e = launch_layer(a, train, last, s);
    if (e != cudaSuccess) return e;
  }
  count_launches(1 + kMpL);
  return cudaGetLastError();
}

cudaError_t launch_mp_stage(const MpnnGraph& g, const MpnnParams& P, int stage, const double* r, const double* invd,
                            const double* rr, const float* sf, MpnnWork& w, double* z, long long spin_limit, int* err,
                            cudaStream_t s) {
  const int N = g.n_nodes;
  if (N <= 0) return cudaSuccess;
  const double inv_n = 1.0 / (2.0 * N);
  if (stage == 0) {
    if (reinterpret_cast<uintptr_t>(r) & 15u) return cudaErrorInvalidValue;
    k_mp_encode<false><<<enc_grid(N), kEncT, 0, s>>>(N, r, rr, inv_n, sf, P, nullptr, w.H[0], nullptr, spin_limit,
                                                      err);
  } else {
    MpLayerArgs a{};
    a.N = N;
    a.node_ptr = g.node_ptr;
    a.nbr = g.nbr;
    a.plan = g.plan;
    a.P = P;
    a.r = r;
    a.invd = invd;
    a.rr = rr;
    a.inv_n = inv_n;
    a.z = z;
    a.spin_limit = spin_limit;
    a.err = err;
    a.layer = stage - 1;
    const bool last = stage == kMpL;
    a.Hin = w.H[(stage - 1) & 1];
    a.Hout = last ? nullptr : w.H[stage & 1];
    const cudaError_t e = launch_layer(a, false, last, s);
    if (e != cudaSuccess) return e;
  }
  count_launches(1);
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

cudaError_t launch_mp_backward(const MpnnGraph& g, const MpnnParams& P, MpnnWork& w, float* grad, long long spin_limit,
                               int* err, cudaStream_t s) {
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
    k_mp_wgrad_tc<<<G, 256, kWgSmem, s>>>(N, w.dU, w.H[l], w.A[l], spin_limit, w.part, err);
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
