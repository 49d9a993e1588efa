// Flexible conjugate gradients with the learned preconditioner z = M(r).
//
// M is a nonlinear map of r (a ReLU network), so the Fletcher-Reeves beta of pcg_iterate
// (solver.cpp:84-99) is replaced by Polak-Ribiere, which keeps the iteration a flexible CG:
//     beta = z_new'(r_new - r_old) / (z_old'r_old) = -alpha z_new'q / (z_old'r_old),   q = A p.
// One iteration: q = A p and alpha = z'r / p'q (the PCG SpMV kernels); x += alpha p,
// r -= alpha q and the convergence test (k_fcg_update); z = M(r) (mpnn.cu); z'r, z'q, r'D^-1 r
// and beta (k_fcg_dots); p = z + beta p (k_fcg_pupdate).
//
// Jacobi is the fallback: when z'r <= 0 (the network returned a non-descent direction) the
// iteration uses z = D^-1 r and restarts; when the residual norm has not halved over a window
// of iterations (stagnation) the network is switched off for the rest of the solve and the
// iteration continues as plain Jacobi-PCG (Fletcher-Reeves beta), restarted once.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {

constexpr int kGrid = kSMs * 4;  // fixed grid: a fixed reduction order

// NV block sums at once: each warp sums its lanes' values, then warp q adds value q over the
// warps (q = w, w + kWarps, ...); two block barriers for any NV. Every thread gets the totals.
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* sm /* NV * (kWarps + 1) */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
  __syncthreads();  // sm may still be read from an earlier call
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[q * kWarps + w] = v[q];
  __syncthreads();
  for (int q = w; q < NV; q += kWarps) {
    double t = lane < kWarps ? sm[q * kWarps + lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) sm[NV * kWarps + q] = t;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = sm[NV * kWarps + q];
}

// Grid reduction in a fixed order: per-block sums into `partials`, the last block to arrive adds
// them (each thread a strided share of every value, all loads in flight together) and returns
// true with the totals.
template <int NV>
__device__ __forceinline__ bool fcg_reduce(const double (&v)[NV], double* partials, unsigned int* ticket,
                                           double (&tot)[NV]) {
  __shared__ double sm[NV * (kWarps + 1)];
  __shared__ bool am_last;
  double b[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) b[q] = v[q];
  block_sums<NV>(b, sm);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[q * gridDim.x + blockIdx.x] = b[q];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NV; ++q) tot[q] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] += __ldcg(&partials[q * gridDim.x + i]);
  block_sums<NV>(tot, sm);
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// x = 0, r = b; ||b|| and the solver state (solver.cpp:42-58). The first p is set by
// k_fcg_dots / k_fcg_pupdate after the first z = M(b) (restart_pending = 1: beta = 0).
__global__ void __launch_bounds__(kThreads) k_fcg_init(int n, const double* __restrict__ b, double* __restrict__ x,
                                                       double* __restrict__ r, double* partials, PcgState* st,
                                                       double rtol, int max_iter) {
  double bb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double bi = b[i];
    x[i] = 0.0;
    r[i] = bi;
    bb = fma(bi, bi, bb);
  }
  const double v[1] = {bb};
  double tot[1];
  if (fcg_reduce<1>(v, partials, &st->ticket[5], tot) && threadIdx.x == 0) {
    st->bnorm = sqrt(tot[0]);
    st->rr = tot[0];
    st->rel = tot[0] > 0.0 ? 1.0 : 0.0;
    st->rtol = rtol;
    st->max_iter = max_iter;
    st->iter = 0;
    st->done = tot[0] > 0.0 ? (max_iter > 0 ? 0 : CSTG_SOLVE_MAX_ITER + 1) : CSTG_SOLVE_ZERO_RHS + 1;
    st->alpha = st->beta = 0.0;
    st->rz = 0.0;
    st->replace_count = 0;
    st->restart_pending = 1;
    st->fallback = 0;
    st->use_jacobi = 0;
    st->mp_skip = st->done != 0;
    st->fb_rr0 = tot[0];
    st->fb_it0 = 0;
    st->true_rel = 0.0;
    st->rmax = st->rel;
    st->reliable_due = 0;
  }
}

// z'r, z'q and r'D^-1 r, r'D^-1 q; the last block picks z (network or Jacobi) and beta.
__global__ void __launch_bounds__(kThreads) k_fcg_dots(int n, const double* __restrict__ z,
                                                       const double* __restrict__ r, const double* __restrict__ q,
                                                       const double* __restrict__ invd, double* partials,
                                                       PcgState* st) {
  if (__ldcg(&st->done)) return;
  double zr = 0.0, zq = 0.0, jr = 0.0, jq = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = r[i], qi = q[i], ji = invd[i] * ri;
    zr = fma(z[i], ri, zr);
    zq = fma(z[i], qi, zq);
    jr = fma(ji, ri, jr);
    jq = fma(ji, qi, jq);
  }
  const double v[4] = {zr, zq, jr, jq};
  double tot[4];
  if (fcg_reduce<4>(v, partials, &st->ticket[6], tot) && threadIdx.x == 0) {
    bool restart = st->restart_pending != 0;
    bool jac = st->fallback != 0;
    if (!jac && !(tot[0] > 0.0)) {  // a non-descent network output: Jacobi this step, restarted
      jac = true;
      restart = true;
    }
    const double rz_new = jac ? tot[2] : tot[0];
    double beta = 0.0;
    if (!restart && st->rz > 0.0) {
      if (st->fallback)
        beta = rz_new / st->rz;  // plain Jacobi-PCG (Fletcher-Reeves), solver.cpp:84-99
      else
        beta = -st->alpha * (jac ? tot[3] : tot[1]) / st->rz;  // Polak-Ribiere
    }
    st->beta = beta;
    st->rz = rz_new;
    st->use_jacobi = jac ? 1 : 0;
    st->restart_pending = 0;
  }
}

// p = z + beta p (z = D^-1 r when use_jacobi)
__global__ void __launch_bounds__(kThreads) k_fcg_pupdate(int n, const double* __restrict__ z,
                                                          const double* __restrict__ r,
                                                          const double* __restrict__ invd, double* __restrict__ p,
                                                          const PcgState* st) {
  if (__ldcg(&st->done)) return;
  const double beta = __ldcg(&st->beta);
  const bool jac = __ldcg(&st->use_jacobi) != 0;
  // pairs of DOFs (16-byte loads); an odd last row on its own
  const int n2 = n >> 1;
  const double2* z2 = reinterpret_cast<const double2*>(z);
  const double2* r2 = reinterpret_cast<const double2*>(r);
  const double2* d2 = reinterpret_cast<const double2*>(invd);
  double2* p2 = reinterpret_cast<double2*>(p);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    double2 zi;
    if (jac) {
      const double2 ri = r2[i], di = d2[i];
      zi = make_double2(di.x * ri.x, di.y * ri.y);
    } else {
      zi = z2[i];
    }
    const double2 pi = p2[i];
    p2[i] = make_double2(fma(beta, pi.x, zi.x), fma(beta, pi.y, zi.y));
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int i = n - 1;
    const double zi = jac ? invd[i] * r[i] : z[i];
    p[i] = fma(beta, p[i], zi);
  }
}

// x += alpha p, r -= alpha q; ||r||, convergence (solver.cpp:72-82), max_iter, stagnation.
__global__ void __launch_bounds__(kThreads) k_fcg_update(int n, double* __restrict__ x, double* __restrict__ r,
                                                         const double* __restrict__ p,
                                                         const double* __restrict__ q, double* partials,
                                                         PcgState* st, int window, double ratio2,
                                                         double reliable_delta) {
  if (__ldcg(&st->done)) return;
  const double alpha = __ldcg(&st->alpha);
  double rr = 0.0;
  // pairs of DOFs (16-byte loads); an odd last row on its own
  const int n2 = n >> 1;
  double2* x2 = reinterpret_cast<double2*>(x);
  double2* r2 = reinterpret_cast<double2*>(r);
  const double2* p2 = reinterpret_cast<const double2*>(p);
  const double2* q2 = reinterpret_cast<const double2*>(q);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    const double2 pi = p2[i], qi = q2[i];
    double2 xi = x2[i], ri = r2[i];
    xi.x = fma(alpha, pi.x, xi.x);
    xi.y = fma(alpha, pi.y, xi.y);
    ri.x = fma(-alpha, qi.x, ri.x);
    ri.y = fma(-alpha, qi.y, ri.y);
    x2[i] = xi;
    r2[i] = ri;
    rr = fma(ri.x, ri.x, fma(ri.y, ri.y, rr));
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const int i = n - 1;
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    rr = fma(ri, ri, rr);
  }
  const double v[1] = {rr};
  double tot[1];
  if (fcg_reduce<1>(v, partials, &st->ticket[7], tot) && threadIdx.x == 0) {
    const int it = st->iter + 1;
    st->iter = it;
    st->rr = tot[0];
    st->rel = st->bnorm > 0.0 ? sqrt(tot[0]) / st->bnorm : 0.0;
    if (st->rel <= st->rtol)
      st->done = CSTG_SOLVE_CONVERGED + 1;
    else if (it >= st->max_iter)
      st->done = CSTG_SOLVE_MAX_ITER + 1;
    if (!st->fallback && window > 0 && it - st->fb_it0 >= window) {
      if (tot[0] > ratio2 * st->fb_rr0) {  // stagnation: the network is switched off
        st->fallback = 1;
        st->restart_pending = 1;
      }
      st->fb_rr0 = tot[0];
      st->fb_it0 = it;
    }
    st->mp_skip = (st->done != 0 || st->fallback != 0) ? 1 : 0;
    if (reliable_delta > 0.0 && st->done == 0) {
      st->rmax = fmax(st->rmax, st->rel);
      if (st->rel < reliable_delta * st->rmax) st->reliable_due = 1;
    }
  }
}

// r = b - A x with the FP64 2x2-block matrix, thread per node, and ||r||; the recursive residual
// becomes the true one (van der Vorst-Ye reliable update, the direction and the ring are kept).
__global__ void __launch_bounds__(kThreads) k_fcg_reliable(int n_nodes, BlockMatrix A, const double* __restrict__ b,
                                                           const double* __restrict__ x, double* __restrict__ r,
                                                           double* partials, PcgState* st) {
  if (__ldcg(&st->done) || !__ldcg(&st->reliable_due)) return;  // uniform
  const double2* x2 = reinterpret_cast<const double2*>(x);
  const double2* b2 = reinterpret_cast<const double2*>(b);
  double2* r2 = reinterpret_cast<double2*>(r);
  const double2* v2 = reinterpret_cast<const double2*>(A.vals);
  double rr = 0.0;
  for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < n_nodes; nd += gridDim.x * blockDim.x) {
    const int k0 = A.node_ptr[nd], d = A.node_ptr[nd + 1] - k0;
    const size_t base = 2 * (size_t)k0;  // node nd's rows start at value 4 k0 (double2 index 2 k0)
    double y0 = 0.0, y1 = 0.0;
    for (int k = 0; k < d; ++k) {
      const double2 xm = x2[A.bnbr[k0 + k]];
      const double2 a0 = v2[base + k], a1 = v2[base + d + k];
      y0 = fma(a0.x, xm.x, fma(a0.y, xm.y, y0));
      y1 = fma(a1.x, xm.x, fma(a1.y, xm.y, y1));
    }
    const double2 bn = b2[nd];
    const double2 rn = make_double2(bn.x - y0, bn.y - y1);
    r2[nd] = rn;
    rr = fma(rn.x, rn.x, fma(rn.y, rn.y, rr));
  }
  const double v[1] = {rr};
  double tot[1];
  if (fcg_reduce<1>(v, partials, &st->ticket[4], tot) && threadIdx.x == 0) {
    st->rr = tot[0];
    st->rel = st->bnorm > 0.0 ? sqrt(tot[0]) / st->bnorm : 0.0;
    st->rmax = st->rel;
    st->reliable_due = 0;
    st->replace_count += 1;
  }
}

// ---- truncated flexible CG (depth H + 1) -----------------------------------------------------------

// Age of ring slot j (0: the most recent push); the slot holds a direction when age < count.
__device__ __forceinline__ int ring_age(const FcgRing* R, int j, int H) { return (R->head - 1 - j + 2 * H) % H; }

// As k_fcg_dots, plus z'q_j (and (D^-1 r)'q_j) for the ring's directions: the last block sets
// beta[0] = -z'q / p'q for the current p and beta[1 + j] = -z'q_j / p_j'q_j for every stored one,
// then registers the push of the current p / q into the ring (not on a restart, which clears it).
template <int H>
__global__ void __launch_bounds__(kThreads) k_fcg_dots_ring(FcgBuffers w) {
  PcgState* st = w.st;
  if (__ldcg(&st->done)) return;
  FcgRing* R = w.ring;
  bool valid[H];
#pragma unroll
  for (int j = 0; j < H; ++j) valid[j] = ring_age(R, j, H) < R->count;
  double zr = 0.0, zq = 0.0, jr = 0.0, jq = 0.0, zqh[H], jqh[H];
#pragma unroll
  for (int j = 0; j < H; ++j) zqh[j] = jqh[j] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n; i += gridDim.x * blockDim.x) {
    const double ri = w.r[i], qi = w.q[i], ji = w.inv_diag[i] * ri, zi = w.z[i];
    zr = fma(zi, ri, zr);
    zq = fma(zi, qi, zq);
    jr = fma(ji, ri, jr);
    jq = fma(ji, qi, jq);
#pragma unroll
    for (int j = 0; j < H; ++j)
      if (valid[j]) {
        const double qj = w.qh[j][i];
        zqh[j] = fma(zi, qj, zqh[j]);
        jqh[j] = fma(ji, qj, jqh[j]);
      }
  }
  double v[4 + 2 * H];
  v[0] = zr;
  v[1] = zq;
  v[2] = jr;
  v[3] = jq;
#pragma unroll
  for (int j = 0; j < H; ++j) {
    v[4 + j] = zqh[j];
    v[4 + H + j] = jqh[j];
  }
  double tot[4 + 2 * H];
  if (fcg_reduce<4 + 2 * H>(v, w.partials, &st->ticket[6], tot) && threadIdx.x == 0) {
    bool restart = st->restart_pending != 0;
    bool jac = st->fallback != 0;
    if (!jac && !(tot[0] > 0.0)) {  // a non-descent network output: Jacobi this step, restarted
      jac = true;
      restart = true;
    }
    const double rz_new = jac ? tot[2] : tot[0];
    double beta = 0.0;
#pragma unroll
    for (int j = 0; j < H; ++j) R->beta[1 + j] = 0.0;
    if (!restart && st->rz > 0.0) {
      if (st->fallback) {
        beta = rz_new / st->rz;  // plain Jacobi-PCG (Fletcher-Reeves), solver.cpp:84-99
      } else {
        beta = -st->alpha * (jac ? tot[3] : tot[1]) / st->rz;  // -z'q / p'q
#pragma unroll
        for (int j = 0; j < H; ++j)
          if (valid[j] && R->pq[j] > 0.0) R->beta[1 + j] = -(jac ? tot[4 + H + j] : tot[4 + j]) / R->pq[j];
      }
    }
    st->beta = beta;
    R->beta[0] = beta;
    if (restart || st->fallback) {
      R->count = 0;
      R->push = 0;
    } else {
      R->push = 1;
      R->push_slot = R->head;
      R->pq[R->head] = st->pAp;
      R->head = (R->head + 1) % H;
      if (R->count < H) R->count += 1;
    }
    st->rz = rz_new;
    st->use_jacobi = jac ? 1 : 0;
    st->restart_pending = 0;
  }
}

// p = z + beta[0] p + sum_j beta[1 + j] p_j (z = D^-1 r when use_jacobi); the old p and q go into
// the ring slot registered by k_fcg_dots_ring (read before they are overwritten, element by element).
template <int H>
__global__ void __launch_bounds__(kThreads) k_fcg_pupdate_ring(FcgBuffers w) {
  const PcgState* st = w.st;
  if (__ldcg(&st->done)) return;
  const FcgRing* R = w.ring;
  const bool jac = __ldcg(&st->use_jacobi) != 0;
  double beta[H + 1];
#pragma unroll
  for (int j = 0; j <= H; ++j) beta[j] = __ldcg(&R->beta[j]);
  const bool push = __ldcg(&R->push) != 0;
  const int slot = __ldcg(&R->push_slot);
  double* ps = push ? w.ph[0] : nullptr;
  double* qs = push ? w.qh[0] : nullptr;
#pragma unroll
  for (int j = 1; j < H; ++j)
    if (push && slot == j) {
      ps = w.ph[j];
      qs = w.qh[j];
    }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n; i += gridDim.x * blockDim.x) {
    const double zi = jac ? w.inv_diag[i] * w.r[i] : w.z[i];
    const double pi = w.p[i];
    double pn = fma(beta[0], pi, zi);
#pragma unroll
    for (int j = 0; j < H; ++j)
      if (beta[1 + j] != 0.0) pn = fma(beta[1 + j], w.ph[j][i], pn);
    if (push) {
      ps[i] = pi;
      qs[i] = w.q[i];
    }
    w.p[i] = pn;
  }
}

}  // namespace

cudaError_t launch_fcg_dots_ring(const FcgBuffers& w, cudaStream_t s) {
  switch (w.hist) {
    case 1:
      k_fcg_dots_ring<1><<<kGrid, kThreads, 0, s>>>(w);
      k_fcg_pupdate_ring<1><<<kGrid, kThreads, 0, s>>>(w);
      break;
    case 2:
      k_fcg_dots_ring<2><<<kGrid, kThreads, 0, s>>>(w);
      k_fcg_pupdate_ring<2><<<kGrid, kThreads, 0, s>>>(w);
      break;
    case 3:
      k_fcg_dots_ring<3><<<kGrid, kThreads, 0, s>>>(w);
      k_fcg_pupdate_ring<3><<<kGrid, kThreads, 0, s>>>(w);
      break;
    case 4:
      k_fcg_dots_ring<4><<<kGrid, kThreads, 0, s>>>(w);
      k_fcg_pupdate_ring<4><<<kGrid, kThreads, 0, s>>>(w);
      break;
    default:
      return launch_fcg_dots(w, s);
  }
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_fcg_init(const FcgBuffers& w, double rtol, int max_iter, int window, cudaStream_t s) {
  (void)window;
  k_fcg_init<<<kGrid, kThreads, 0, s>>>(w.n, w.b, w.x, w.r, w.partials, w.st, rtol, max_iter);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fcg_dots(const FcgBuffers& w, cudaStream_t s) {
  k_fcg_dots<<<kGrid, kThreads, 0, s>>>(w.n, w.z, w.r, w.q, w.inv_diag, w.partials, w.st);
  k_fcg_pupdate<<<kGrid, kThreads, 0, s>>>(w.n, w.z, w.r, w.inv_diag, w.p, w.st);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t launch_fcg_pupdate(const FcgBuffers& w, cudaStream_t s) {
  k_fcg_pupdate<<<kGrid, kThreads, 0, s>>>(w.n, w.z, w.r, w.inv_diag, w.p, w.st);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fcg_update(const FcgBuffers& w, int window, double ratio2, cudaStream_t s,
                              double reliable_delta) {
  k_fcg_update<<<kGrid, kThreads, 0, s>>>(w.n, w.x, w.r, w.p, w.q, w.partials, w.st, window, ratio2,
                                          reliable_delta);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fcg_reliable(const FcgBuffers& w, const BlockMatrix& A, cudaStream_t s) {
  k_fcg_reliable<<<kGrid, kThreads, 0, s>>>(A.n_nodes, A, w.b, w.x, w.r, w.partials, w.st);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
