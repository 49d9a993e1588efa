// Batched Jacobi-PCG: many disjoint systems (plates of uneven size) x up to four right-hand
// sides (load cases) in ONE persistent launch of thread-block clusters.
//
// The batch is one block-diagonal matrix (the plates' meshes concatenated, assembled and
// eliminated by the single-system kernels). Each cluster takes the next plate from a queue
// (largest first), solves all of its load cases together, and takes another plate until the
// queue is empty. Inside a plate the cluster's CTAs split the plate's nodes; the reductions of
// a CG iteration (p'Ap; r'z and r'r; the true-residual norms) are summed per CTA, exchanged
// through distributed shared memory after a cluster barrier, and added in CTA-rank order by
// every CTA, so all CTAs take identical decisions and the results are deterministic for a given
// launch shape. No grid-wide barrier and no global-memory spin: clusters never wait on each
// other.
//
// Per load case the recurrence is pcg_iterate's (solver.cpp:35-105) with the FP32
// difference-form operator of mixed_kernels.cu; x, r, p, Ap and every scalar are FP64. Reliable
// updates replace r by the FP64 true residual b - A x once per decade of residual reduction
// (p is kept); when the recursive residual meets rtol the true residual is checked the same way,
// and a load case stops only when the FP64 true residual meets rtol. A plate whose FP32
// operator stops improving the true residual (or fails more checks than max_refinements)
// switches to the FP64 operator with one restart.
//
// Vectors are interleaved per node: [node][load case][2] doubles, so one neighbour gather
// serves all load cases and every matrix block is read once per iteration for all of them.
#include <cooperative_groups.h>

#include "../../include/cstfem_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace cstg {

namespace {

// Cluster-wide deterministic sum of V values per thread; the totals land in `tot` (all CTAs).
// wsum holds max(T/32, 16) * V doubles.
template <int V, int T>
__device__ __forceinline__ void cluster_sum(const cg::cluster_group& cl, const double (&v)[V],
                                            double* wsum, double* red, int& buf, double* tot) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < V; ++i) {
    const double s = warp_sum(v[i]);
    if (lane == 0) wsum[w * V + i] = s;
  }
  __syncthreads();
  double* mine = red + buf * V;
  if (threadIdx.x < V) {
    double s = 0.0;
#pragma unroll 4
    for (int q = 0; q < T / 32; ++q) s += wsum[q * V + threadIdx.x];
    mine[threadIdx.x] = s;
  }
  cl.sync();  // release/acquire at cluster scope: every CTA's partials (and prior writes) visible
  // Fetch all ranks' partials at once (one remote load per thread), then add them in rank order.
  const unsigned nb = cl.num_blocks();
  if (threadIdx.x < nb * V) wsum[threadIdx.x] = cl.map_shared_rank(mine, threadIdx.x / V)[threadIdx.x % V];
  __syncthreads();
  if (threadIdx.x < V) {
    double s = 0.0;
    for (unsigned q = 0; q < nb; ++q) s += wsum[q * V + threadIdx.x];
    tot[threadIdx.x] = s;
  }
  __syncthreads();
  buf ^= 1;  // the other buffer is next; a cluster barrier separates any two uses of one buffer
}

// Reliable updates: replace r by the FP64 true residual when the recursive r'r has fallen to
// this fraction (0.1^2: one decade of ||r||) of its largest value since the last replacement,
// or after this many iterations without one.
constexpr double kBatchDelta2 = 1e-2;
constexpr int kBatchCycle = 1000;

__device__ __forceinline__ double dot2(double2 a, double2 b, double acc) {
  return fma(a.x, b.x, fma(a.y, b.y, acc));
}

template <int R, int T>
__global__ void __launch_bounds__(T, (T >= 512 ? 1 : 512 / T)) k_batch_pcg(const BatchArgs a) {
  const cg::cluster_group cl = cg::this_cluster();
  const int crank = (int)cl.block_rank(), C = (int)cl.num_blocks();
  constexpr int V = 2 * R;
  __shared__ double wsum[(T / 32 > 16 ? T / 32 : 16) * V];  // warp partials, then <= 16 ranks' partials
  __shared__ double red[2 * V];
  __shared__ double tot[V];
  __shared__ int s_plate;
  int buf = 0;
  const double2* __restrict__ invd2 = reinterpret_cast<const double2*>(a.inv_diag);
  const double2* __restrict__ b2 = reinterpret_cast<const double2*>(a.b);
  double2* __restrict__ x2 = reinterpret_cast<double2*>(a.x);
  double2* __restrict__ r2 = reinterpret_cast<double2*>(a.r);
  double2* p2 = reinterpret_cast<double2*>(a.p);  // read by neighbours: always through L2
  double2* __restrict__ Ap2 = reinterpret_cast<double2*>(a.Ap);
  const double2* __restrict__ v64 = reinterpret_cast<const double2*>(a.A64.vals);
  const double rtol2 = a.rtol * a.rtol;

  for (;;) {
    if (crank == 0 && threadIdx.x == 0) {
      const int q = atomicAdd(a.queue, 1);
      s_plate = q < a.n_sys ? a.order[q] : -1;
    }
    cl.sync();
    const int plate = *cl.map_shared_rank(&s_plate, 0);
    if (plate < 0) break;
    const int n0 = a.sys_node[plate], n1 = a.sys_node[plate + 1];
    const int first = n0 + crank * T + (int)threadIdx.x, stride = C * T;

    // x = 0, r = b, p = D^-1 b; r'z and b'b per load case (solver.cpp:42-58)
    double v[V];
#pragma unroll
    for (int i = 0; i < V; ++i) v[i] = 0.0;
    for (int n = first; n < n1; n += stride) {
      const double2 d = invd2[n];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const size_t k = (size_t)n * R + q;
        const double2 bk = b2[k];
        const double2 z = make_double2(d.x * bk.x, d.y * bk.y);
        x2[k] = make_double2(0.0, 0.0);
        r2[k] = bk;
        __stcg(&p2[k], z);
        v[q] = dot2(bk, z, v[q]);
        v[R + q] = dot2(bk, bk, v[R + q]);
      }
    }
    cluster_sum<V, T>(cl, v, wsum, red, buf, tot);

    double rz[R], bn2[R], alpha[R], beta[R], rel[R], true_rel[R], prev_true[R], rmax[R];
    int it[R], nref[R], nfail[R], last_rep[R], status[R];
    unsigned active = 0;
    bool fp64 = a.start_fp64 != 0;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      rz[q] = tot[q];
      bn2[q] = tot[R + q];
      rmax[q] = bn2[q];
      alpha[q] = beta[q] = 0.0;
      it[q] = nref[q] = nfail[q] = last_rep[q] = 0;
      prev_true[q] = INFINITY;
      true_rel[q] = 0.0;
      rel[q] = bn2[q] > 0.0 ? 1.0 : 0.0;
      status[q] = CSTG_SOLVE_CONVERGED;
      if (bn2[q] > 0.0)
        active |= 1u << q;
      else
        status[q] = CSTG_SOLVE_ZERO_RHS;  // x = 0 is exact
    }

    while (active) {
      // ---- Phase A: Ap = A p and p'Ap (all load cases share the matrix read). Neighbours are
      // taken two at a time so both index loads, then all their p loads, are in flight at once.
#pragma unroll
      for (int i = 0; i < V; ++i) v[i] = 0.0;
      for (int n = first; n < n1; n += stride) {
        double2 pn[R], y[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          pn[q] = __ldcg(&p2[(size_t)n * R + q]);
          y[q] = make_double2(0.0, 0.0);
        }
        if (fp64) {
          const int b0 = __ldg(&a.A64.node_ptr[n]), deg = __ldg(&a.A64.node_ptr[n + 1]) - b0;
          const double2* ra = v64 + 2L * b0;
          const double2* rb = ra + deg;
          for (int k = 0; k < deg; k += 2) {
            const bool two = k + 1 < deg;
            const int m0 = __ldg(&a.A64.bnbr[b0 + k]);
            const int m1 = two ? __ldg(&a.A64.bnbr[b0 + k + 1]) : m0;
            const double2 ka0 = __ldg(ra + k), kb0 = __ldg(rb + k);
            const double2 ka1 = two ? __ldg(ra + k + 1) : make_double2(0.0, 0.0);
            const double2 kb1 = two ? __ldg(rb + k + 1) : make_double2(0.0, 0.0);
            double2 p0[R], p1[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
              p0[q] = __ldcg(&p2[(size_t)m0 * R + q]);
              p1[q] = __ldcg(&p2[(size_t)m1 * R + q]);
            }
#pragma unroll
            for (int q = 0; q < R; ++q) {
              y[q].x = dot2(ka1, p1[q], dot2(ka0, p0[q], y[q].x));
              y[q].y = dot2(kb1, p1[q], dot2(kb0, p0[q], y[q].y));
            }
          }
        } else {
          const int bb = __ldg(&a.A32.node_ptr[n]);
          const int o = bb - n, c = __ldg(&a.A32.node_ptr[n + 1]) - bb - 1;
          for (int k = 0; k < c; k += 2) {
            const bool two = k + 1 < c;
            const int m0 = __ldg(&a.A32.nbr32[o + k]);
            const int m1 = two ? __ldg(&a.A32.nbr32[o + k + 1]) : n;
            const float4 f0 = __ldg(&a.A32.val32[o + k]);
            const float4 f1 = two ? __ldg(&a.A32.val32[o + k + 1]) : make_float4(0.f, 0.f, 0.f, 0.f);
            double2 p0[R], p1[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
              p0[q] = __ldcg(&p2[(size_t)m0 * R + q]);
              p1[q] = __ldcg(&p2[(size_t)m1 * R + q]);
            }
#pragma unroll
            for (int q = 0; q < R; ++q) {
              const double dx0 = p0[q].x - pn[q].x, dy0 = p0[q].y - pn[q].y;
              const double dx1 = p1[q].x - pn[q].x, dy1 = p1[q].y - pn[q].y;
              y[q].x = fma((double)f0.x, dx0, fma((double)f0.y, dy0, y[q].x));
              y[q].y = fma((double)f0.z, dx0, fma((double)f0.w, dy0, y[q].y));
              y[q].x = fma((double)f1.x, dx1, fma((double)f1.y, dy1, y[q].x));
              y[q].y = fma((double)f1.z, dx1, fma((double)f1.w, dy1, y[q].y));
            }
          }
          const double2 sa = __ldg(&a.A32.S64[2 * n]), sb = __ldg(&a.A32.S64[2 * n + 1]);
#pragma unroll
          for (int q = 0; q < R; ++q) {
            y[q].x = dot2(sa, pn[q], y[q].x);
            y[q].y = dot2(sb, pn[q], y[q].y);
          }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
          Ap2[(size_t)n * R + q] = y[q];
          v[q] = dot2(pn[q], y[q], v[q]);
        }
      }
      cluster_sum<V, T>(cl, v, wsum, red, buf, tot);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if (!((active >> q) & 1u)) continue;
        const double pAp = tot[q];
        if (!(pAp > 0.0)) {  // solver.cpp:64-68
          status[q] = CSTG_SOLVE_BREAKDOWN;
          active &= ~(1u << q);
          alpha[q] = 0.0;
        } else {
          alpha[q] = rz[q] / pAp;
        }
      }
      if (!active) break;

      // ---- Phase B: x += alpha p, r -= alpha Ap; r'z and r'r. All loads of a node are issued
      // before any store (stores of finished cases are skipped), so its 4R loads fly together.
#pragma unroll
      for (int i = 0; i < V; ++i) v[i] = 0.0;
#pragma unroll 2
      for (int n = first; n < n1; n += stride) {
        const double2 d = invd2[n];
        double2 pk[R], apk[R], xk[R], rk[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const size_t k = (size_t)n * R + q;
          pk[q] = __ldcg(&p2[k]);
          apk[q] = Ap2[k];
          xk[q] = x2[k];
          rk[q] = r2[k];
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
          xk[q].x = fma(alpha[q], pk[q].x, xk[q].x);
          xk[q].y = fma(alpha[q], pk[q].y, xk[q].y);
          rk[q].x = fma(-alpha[q], apk[q].x, rk[q].x);
          rk[q].y = fma(-alpha[q], apk[q].y, rk[q].y);
          if ((active >> q) & 1u) {
            const size_t k = (size_t)n * R + q;
            x2[k] = xk[q];
            r2[k] = rk[q];
          }
          v[q] = fma(rk[q].x, d.x * rk[q].x, fma(rk[q].y, d.y * rk[q].y, v[q]));
          v[R + q] = dot2(rk[q], rk[q], v[R + q]);
        }
      }
      cluster_sum<V, T>(cl, v, wsum, red, buf, tot);
      // Which load cases need the FP64 true residual now: a convergence check (the recursive
      // residual met rtol, or max_iter), or a reliable update (the recursive residual fell by
      // kBatchDelta2 since the largest one after the last update, or kBatchCycle iterations
      // passed). A reliable update replaces r and keeps p (van der Vorst and Ye's scheme).
      unsigned check = 0, repl = 0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if (!((active >> q) & 1u)) continue;
        ++it[q];
        const double rr = tot[R + q];
        rel[q] = sqrt(rr / bn2[q]);
        rmax[q] = fmax(rmax[q], rr);
        if (rr <= rtol2 * bn2[q] || it[q] >= a.max_iter) {
          check |= 1u << q;
        } else if (rr <= kBatchDelta2 * rmax[q] || it[q] - last_rep[q] >= kBatchCycle) {
          repl |= 1u << q;
        } else {
          beta[q] = tot[q] / rz[q];
          rz[q] = tot[q];
        }
      }
      repl |= check;

      if (repl) {
        // ---- Phase R: FP64 true residual r = b - A x for the replaced load cases
#pragma unroll
        for (int i = 0; i < V; ++i) v[i] = 0.0;
        for (int n = first; n < n1; n += stride) {
          const double2 d = invd2[n];
          const int b0 = __ldg(&a.A64.node_ptr[n]), deg = __ldg(&a.A64.node_ptr[n + 1]) - b0;
          const double2* ra = v64 + 2L * b0;
          const double2* rb = ra + deg;
          double2 t[R];
#pragma unroll
          for (int q = 0; q < R; ++q) t[q] = make_double2(0.0, 0.0);
          for (int k = 0; k < deg; ++k) {
            const int m = __ldg(&a.A64.bnbr[b0 + k]);
            const double2 ka = __ldg(ra + k), kb = __ldg(rb + k);
#pragma unroll
            for (int q = 0; q < R; ++q) {
              if (!((repl >> q) & 1u)) continue;
              const double2 xm = __ldcg(&x2[(size_t)m * R + q]);
              t[q].x = dot2(ka, xm, t[q].x);
              t[q].y = dot2(kb, xm, t[q].y);
            }
          }
#pragma unroll
          for (int q = 0; q < R; ++q) {
            if (!((repl >> q) & 1u)) continue;
            const size_t k = (size_t)n * R + q;
            const double2 bk = b2[k];
            const double2 rk = make_double2(bk.x - t[q].x, bk.y - t[q].y);
            r2[k] = rk;
            v[q] = dot2(rk, rk, v[q]);
            v[R + q] = fma(rk.x, d.x * rk.x, fma(rk.y, d.y * rk.y, v[R + q]));
          }
        }
        cluster_sum<V, T>(cl, v, wsum, red, buf, tot);
        bool restart = false;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          if (!((repl >> q) & 1u)) continue;
          const double rr = tot[q], tr = sqrt(rr / bn2[q]);
          true_rel[q] = tr;
          const bool is_check = (check >> q) & 1u;
          if (is_check && rr <= rtol2 * bn2[q]) {
            status[q] = CSTG_SOLVE_CONVERGED;
            active &= ~(1u << q);
            continue;
          }
          if (it[q] >= a.max_iter) {
            status[q] = CSTG_SOLVE_MAX_ITER;
            active &= ~(1u << q);
            continue;
          }
          ++nref[q];
          last_rep[q] = it[q];
          rmax[q] = rr;
          rel[q] = tr;
          if (is_check) {  // the recursive residual met rtol but the true one did not
            ++nfail[q];
            if (!fp64 && (nfail[q] > a.max_refine || tr > 0.5 * prev_true[q])) {
              fp64 = true;  // the FP32 operator's accuracy floor: FP64 from here, restarted
              restart = true;
            }
            prev_true[q] = tr;
          }
          beta[q] = tot[R + q] / rz[q];
          rz[q] = tot[R + q];
        }
        if (restart)
#pragma unroll
          for (int q = 0; q < R; ++q) beta[q] = 0.0;
      }

      // ---- Phase C: p = D^-1 r + beta p
      if (active) {
#pragma unroll 2
        for (int n = first; n < n1; n += stride) {
          const double2 d = invd2[n];
          double2 rk[R], pk[R];
#pragma unroll
          for (int q = 0; q < R; ++q) {
            const size_t k = (size_t)n * R + q;
            rk[q] = r2[k];
            pk[q] = __ldcg(&p2[k]);
          }
#pragma unroll
          for (int q = 0; q < R; ++q)
            if ((active >> q) & 1u)
              __stcg(&p2[(size_t)n * R + q], make_double2(fma(beta[q], pk[q].x, d.x * rk[q].x),
                                                          fma(beta[q], pk[q].y, d.y * rk[q].y)));
        }
      }
      cl.sync();  // Phase C's p visible to the neighbours' CTAs before the next SpMV
    }

    if (crank == 0 && threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        BatchResultDev o;
        o.iterations = it[q];
        o.status = status[q];
        o.refinements = nref[q];
        o.fp64 = fp64 ? 1 : 0;
        o.rel = rel[q];
        o.true_rel = true_rel[q];
        a.res[(size_t)plate * a.res_stride + a.res_offset + q] = o;
      }
    }
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// [rhs][2N] (ld doubles apart) <-> [node][R][2] for load cases q0 .. q0 + R - 1
__global__ void k_batch_pack(int N, int R, int q0, long long ld, const double* __restrict__ src,
                             double2* __restrict__ dst) {
  const long long total = (long long)N * R;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(i / R), q = (int)(i - (long long)n * R);
    const double* s = src + (q0 + q) * ld + 2LL * n;
    dst[i] = make_double2(s[0], s[1]);
  }
}

__global__ void k_batch_unpack(int N, int R, int q0, long long ld, const double2* __restrict__ src,
                               double* __restrict__ dst) {
  const long long total = (long long)N * R;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(i / R), q = (int)(i - (long long)n * R);
    const double2 v = src[i];
    double* d = dst + (q0 + q) * ld + 2LL * n;
    d[0] = v.x;
    d[1] = v.y;
  }
}

// Every node's neighbours must lie in the node's own plate: the smallest offending node is
// recorded (a coupled batch would be solved wrongly, since plates never synchronise).
__global__ void k_batch_check(int N, int n_sys, const int* __restrict__ sys_node,
                              const int* __restrict__ node_ptr, const int* __restrict__ bnbr, int* err) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  int lo = 0, hi = n_sys;  // plate s with sys_node[s] <= n < sys_node[s + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (sys_node[mid] <= n)
      lo = mid;
    else
      hi = mid;
  }
  const int a = sys_node[lo], b = sys_node[lo + 1];
  for (int k = node_ptr[n]; k < node_ptr[n + 1]; ++k) {
    const int m = bnbr[k];
    if (m < a || m >= b) {
      atomicMin(&err[kErrBatch], n);
      return;
    }
  }
}

int grid_for(long long work) {
  const long long g = (work + 255) / 256;
  return (int)std::min<long long>(std::max<long long>(g, 1), 148LL * 8);
}

template <int R, int T>
cudaError_t launch_shape(const BatchArgs* a, int cluster, int n_clusters, int* max_clusters,
                         cudaStream_t s) {
  auto kern = k_batch_pcg<R, T>;
  if (cluster > 8 && max_clusters) {  // the shape query always precedes a launch (never in a capture)
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (max_clusters) {
    cfg.gridDim = dim3((unsigned)cluster);
    *max_clusters = 0;
    return cudaOccupancyMaxActiveClusters(max_clusters, (void*)kern, &cfg);
  }
  cfg.gridDim = dim3((unsigned)(n_clusters * cluster));
  return cudaLaunchKernelEx(&cfg, kern, *a);
}

template <int R>
cudaError_t launch_r(const BatchArgs* a, int cluster, int threads, int n_clusters, int* max_clusters,
                     cudaStream_t s) {
  switch (threads) {
    case 256: return launch_shape<R, 256>(a, cluster, n_clusters, max_clusters, s);
    case 512: return launch_shape<R, 512>(a, cluster, n_clusters, max_clusters, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t dispatch(const BatchArgs* a, int R, int cluster, int threads, int n_clusters, int* max_clusters,
                     cudaStream_t s) {
  if (cluster < 1 || cluster > 16) return cudaErrorInvalidValue;
  switch (R) {
    case 1: return launch_r<1>(a, cluster, threads, n_clusters, max_clusters, s);
    case 2: return launch_r<2>(a, cluster, threads, n_clusters, max_clusters, s);
    case 3: return launch_r<3>(a, cluster, threads, n_clusters, max_clusters, s);
    case 4: return launch_r<4>(a, cluster, threads, n_clusters, max_clusters, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t batch_max_clusters(int R, int cluster, int threads, int* n) {
  return dispatch(nullptr, R, cluster, threads, 0, n, nullptr);
}

cudaError_t launch_batch_pcg(const BatchArgs& a, int R, int cluster, int threads, int n_clusters,
                             cudaStream_t s) {
  const cudaError_t e = dispatch(&a, R, cluster, threads, n_clusters, nullptr, s);
  if (e == cudaSuccess) count_launches(1);
  return e;
}

cudaError_t launch_batch_pack(int N, int R, int q0, long long ld, const double* src, double* dst,
                              cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  k_batch_pack<<<grid_for((long long)N * R), 256, 0, s>>>(N, R, q0, ld, src, reinterpret_cast<double2*>(dst));
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_batch_unpack(int N, int R, int q0, long long ld, const double* src, double* dst,
                                cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  k_batch_unpack<<<grid_for((long long)N * R), 256, 0, s>>>(N, R, q0, ld, reinterpret_cast<const double2*>(src),
                                                             dst);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_batch_check(int N, int n_sys, const int* sys_node, const int* node_ptr, const int* bnbr,
                               int* err, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  k_batch_check<<<(N + 255) / 256, 256, 0, s>>>(N, n_sys, sys_node, node_ptr, bnbr, err);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace cstg
