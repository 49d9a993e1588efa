// Mesh-side kernels: node->element incidence, stiffness pattern + element slot map,
// bit-exact CST assembly, Dirichlet elimination, Jacobi diagonal, element stresses.
//
// HBM layout (node-block CSR, which IS the reference's row-owner CSR):
//   node_ptr[N+1]  first 2x2 block of node n's block row (prefix sum of neighbour counts)
//   bnbr[nb]       neighbour node of each block, ascending per node (self included)
//   row_ptr[2N+1]  row_ptr[2n] = 4 node_ptr[n], row_ptr[2n+1] = 4 node_ptr[n] + 2 deg(n)
//   cols[nnz]      row 2n and 2n+1 both list 2m, 2m+1 for every neighbour m
//   vals[nnz]      so node n's two rows are one contiguous run of 4 deg(n) doubles
//   ne_ptr[N+1], ne[3E]  incidences (element * 3 + corner), ascending element per node
//   slot[3 * 3E]   for incidence q of node n: global block index of each corner node of the
//                  element inside node n's block row (the element slot map)
#include <cuda_runtime.h>

#include <atomic>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

static std::atomic<long long> g_launches{0};
void count_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launches_total() { return g_launches.load(std::memory_order_relaxed); }

// ---------------------------------------------------------------------------------------
// exclusive scan of int32 counts: out[0..n] (out[n] = total). Three passes, 2048 items per
// block. Used for incidence and pattern offsets.
constexpr int kScanItems = 8;
constexpr int kScanChunk = kThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) k_scan_reduce(const int* __restrict__ in, int n,
                                                          int* __restrict__ block_sums) {
  __shared__ int sm[kWarps];
  const long base = (long)blockIdx.x * kScanChunk;
  int s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    const long i = base + (long)k * kThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kWarps; ++w) t += sm[w];
    block_sums[blockIdx.x] = t;
  }
}

// Single block: exclusive scan of block_sums in place (nb entries), sequential per thread.
__global__ void __launch_bounds__(1024) k_scan_blocks(int* block_sums, int nb) {
  __shared__ int part[1024];
  const int per = (nb + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(nb, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += block_sums[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int t = 0; t < 1024; ++t) {
      const int v = part[t];
      part[t] = acc;
      acc += v;
    }
  }
  __syncthreads();
  int acc = part[threadIdx.x];
  for (int i = lo; i < hi; ++i) {
    const int v = block_sums[i];
    block_sums[i] = acc;
    acc += v;
  }
}

__global__ void __launch_bounds__(kThreads) k_scan_apply(const int* __restrict__ in, int n,
                                                         const int* __restrict__ block_offs,
                                                         int* __restrict__ out) {
  __shared__ int sm[kThreads * kScanItems];
  __shared__ int wsum[kWarps];
  const long base = (long)blockIdx.x * kScanChunk;
  for (int k = 0; k < kScanItems; ++k) {
    const long i = base + (long)k * kThreads + threadIdx.x;
    sm[k * kThreads + threadIdx.x] = i < n ? in[i] : 0;
  }
  __syncthreads();
  // thread t owns items [t*I, t*I+I) of the chunk
  int loc[kScanItems];
  int s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    loc[k] = s;
    s += sm[threadIdx.x * kScanItems + k];
  }
  // exclusive scan of the per-thread totals across the block
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int q = 0; q < kWarps; ++q) {
      const int v = wsum[q];
      wsum[q] = acc;
      acc += v;
    }
  }
  __syncthreads();
  const int excl = incl - s + wsum[w] + block_offs[blockIdx.x];
  __syncthreads();
  for (int k = 0; k < kScanItems; ++k) sm[threadIdx.x * kScanItems + k] = excl + loc[k];
  __syncthreads();
  for (int k = 0; k < kScanItems; ++k) {
    const long i = base + (long)k * kThreads + threadIdx.x;
    if (i < n) out[i] = sm[k * kThreads + threadIdx.x];
  }
}

// out[n] = total: the last element's exclusive offset plus its count
__global__ void k_scan_total(const int* in, int n, int* out) {
  out[n] = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

cudaError_t scan_exclusive(const int* in, int n, int* out, int* tmp, cudaStream_t s) {
  const int nb = (n + kScanChunk - 1) / kScanChunk;
  if (nb > 0) {
    k_scan_reduce<<<nb, kThreads, 0, s>>>(in, n, tmp);
    k_scan_blocks<<<1, 1024, 0, s>>>(tmp, nb);
    k_scan_apply<<<nb, kThreads, 0, s>>>(in, n, tmp, out);
  }
  k_scan_total<<<1, 1, 0, s>>>(in, n, out);
  count_launches(nb > 0 ? 4 : 1);
  return cudaGetLastError();
}

int scan_tmp_ints(int n) { return (n + kScanChunk - 1) / kScanChunk + 1; }

// ---------------------------------------------------------------------------------------
// node -> element incidence (the inverse of the triangle list)

__global__ void k_count_incidence(int n_tri, const int* __restrict__ tri, int n_nodes,
                                  int* __restrict__ cnt, int* err) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3L * n_tri) return;
  const int v = tri[i];
  if (v < 0 || v >= n_nodes) {
    atomicMin(&err[kErrMesh], (int)(i / 3));
    return;
  }
  atomicAdd(&cnt[v], 1);
}

__global__ void k_fill_incidence(int n_tri, const int* __restrict__ tri, int n_nodes,
                                 const int* __restrict__ ne_ptr, int* __restrict__ cursor,
                                 int* __restrict__ ne) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3L * n_tri) return;
  const int v = tri[i];
  if (v < 0 || v >= n_nodes) return;  // reported by k_count_incidence
  const int pos = ne_ptr[v] + atomicAdd(&cursor[v], 1);
  ne[pos] = (int)i;  // element * 3 + corner
}

// Per node: insertion sort of its incidences (ascending element = ascending e*3+corner).
__global__ void k_sort_incidence(int n_nodes, const int* __restrict__ ne_ptr, int* __restrict__ ne) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  const int lo = ne_ptr[n], hi = ne_ptr[n + 1];
  for (int i = lo + 1; i < hi; ++i) {
    const int v = ne[i];
    int j = i - 1;
    while (j >= lo && ne[j] > v) {
      ne[j + 1] = ne[j];
      --j;
    }
    ne[j + 1] = v;
  }
}

// Sorted unique neighbour set of node n (self included), assembly.cpp:11-21.
// Returns the count, or -1 when it exceeds kMaxNeighbours.
__device__ int neighbour_set(int n, const int* __restrict__ ne_ptr, const int* __restrict__ ne,
                             const int* __restrict__ tri, int* list) {
  int cnt = 1;
  list[0] = n;
  for (int q = ne_ptr[n]; q < ne_ptr[n + 1]; ++q) {
    const int e = ne[q] / 3;
    for (int c = 0; c < 3; ++c) {
      const int m = tri[3 * e + c];
      // insert m into the sorted list[0..cnt)
      int pos = cnt;
      while (pos > 0 && list[pos - 1] > m) --pos;
      if (pos > 0 && list[pos - 1] == m) continue;
      if (cnt == kMaxNeighbours) return -1;
      for (int k = cnt; k > pos; --k) list[k] = list[k - 1];
      list[pos] = m;
      ++cnt;
    }
  }
  return cnt;
}

__global__ void __launch_bounds__(128) k_pattern_count(int n_nodes, const int* __restrict__ ne_ptr,
                                                       const int* __restrict__ ne,
                                                       const int* __restrict__ tri,
                                                       int* __restrict__ deg, int* err) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  int list[kMaxNeighbours];
  const int c = neighbour_set(n, ne_ptr, ne, tri, list);
  if (c < 0) {
    atomicMin(&err[kErrNeighbours], n);
    deg[n] = 0;
    return;
  }
  deg[n] = c;
}

__global__ void __launch_bounds__(128) k_pattern_fill(
    int n_nodes, const int* __restrict__ ne_ptr, const int* __restrict__ ne,
    const int* __restrict__ tri, const int* __restrict__ node_ptr, int* __restrict__ bnbr,
    int* __restrict__ slot, int* __restrict__ row_ptr, int* __restrict__ cols) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  int list[kMaxNeighbours];
  const int c = neighbour_set(n, ne_ptr, ne, tri, list);
  const int b0 = node_ptr[n];
  const long v0 = 4L * b0;
  row_ptr[2 * n] = (int)v0;
  row_ptr[2 * n + 1] = (int)(v0 + 2 * c);
  for (int k = 0; k < c; ++k) {
    const int m = list[k];
    bnbr[b0 + k] = m;
    cols[v0 + 2 * k] = 2 * m;
    cols[v0 + 2 * k + 1] = 2 * m + 1;
    cols[v0 + 2 * c + 2 * k] = 2 * m;
    cols[v0 + 2 * c + 2 * k + 1] = 2 * m + 1;
  }
  // element slot map: block of each corner node of every incident element
  for (int q = ne_ptr[n]; q < ne_ptr[n + 1]; ++q) {
    const int e = ne[q] / 3;
    for (int b = 0; b < 3; ++b) {
      const int m = tri[3 * e + b];
      int lo = 0, hi = c;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (list[mid] < m)
          lo = mid + 1;
        else
          hi = mid;
      }
      slot[3 * q + b] = b0 + lo;
    }
  }
  if (n == n_nodes - 1) row_ptr[2 * n_nodes] = (int)(4L * node_ptr[n_nodes]);
}

// ---------------------------------------------------------------------------------------
// CST element (element.cpp:17-55), FP64 with explicit round-to-nearest operations so that no
// multiply-add is contracted: the same operations, in the same order, as the reference.

struct CstB {
  double B[18];  // 3x6 row-major
  double DB[18];
  double scale;  // t |A|
};

__device__ __forceinline__ double signed_area(double x1, double y1, double x2, double y2,
                                              double x3, double y3) {
  // 0.5 * ((x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1))
  return __dmul_rn(0.5, __dsub_rn(__dmul_rn(__dsub_rn(x2, x1), __dsub_rn(y3, y1)),
                                  __dmul_rn(__dsub_rn(x3, x1), __dsub_rn(y2, y1))));
}

__device__ __forceinline__ void cst_B(const double* xy, double* B) {
  const double x1 = xy[0], y1 = xy[1], x2 = xy[2], y2 = xy[3], x3 = xy[4], y3 = xy[5];
  const double b[3] = {__dsub_rn(y2, y3), __dsub_rn(y3, y1), __dsub_rn(y1, y2)};
  const double c[3] = {__dsub_rn(x3, x2), __dsub_rn(x1, x3), __dsub_rn(x2, x1)};
  const double inv2A = __ddiv_rn(1.0, __dmul_rn(2.0, signed_area(x1, y1, x2, y2, x3, y3)));
#pragma unroll
  for (int k = 0; k < 18; ++k) B[k] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    B[0 * 6 + 2 * i] = __dmul_rn(b[i], inv2A);
    B[1 * 6 + 2 * i + 1] = __dmul_rn(c[i], inv2A);
    B[2 * 6 + 2 * i] = __dmul_rn(c[i], inv2A);
    B[2 * 6 + 2 * i + 1] = __dmul_rn(b[i], inv2A);
  }
}

__device__ __forceinline__ void cst_element(const double* xy, const double* D, double t, CstB& o) {
  cst_B(xy, o.B);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s = __dadd_rn(s, __dmul_rn(D[i * 3 + k], o.B[k * 6 + j]));
      o.DB[i * 6 + j] = s;
    }
  o.scale = __dmul_rn(t, fabs(signed_area(xy[0], xy[1], xy[2], xy[3], xy[4], xy[5])));
}

// Ke(i, j) = scale * sum_k B(k, min) DB(k, max): the upper-triangle value the reference
// mirrors to the lower triangle.
__device__ __forceinline__ double ke_entry(const CstB& o, int i, int j) {
  const int p = i < j ? i : j, q = i < j ? j : i;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) s = __dadd_rn(s, __dmul_rn(o.B[k * 6 + p], o.DB[k * 6 + q]));
  return __dmul_rn(o.scale, s);
}

// Rows 2A, 2A+1 of an element's Ke added into a node's two CSR rows (ra, rb) at the slots of
// the element's three corners. A is a template parameter so that every index into B and DB is
// known at compile time.
template <int A>
__device__ __forceinline__ void add_corner_rows(const CstB& o, const int* __restrict__ slot3, int b0, double* ra,
                                                double* rb) {
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const int k = slot3[b] - b0;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      ra[2 * k + c] = __dadd_rn(ra[2 * k + c], ke_entry(o, 2 * A, 2 * b + c));
      rb[2 * k + c] = __dadd_rn(rb[2 * k + c], ke_entry(o, 2 * A + 1, 2 * b + c));
    }
  }
}

// One thread per node: the node's two rows are zeroed, then every incident element (in
// ascending element order) adds its 2 x 6 slice of Ke. Each CSR entry therefore receives
// its contributions in the reference's order (assembly.cpp:56-72), starting from 0.0.
// With a material table (`mat` non-null: element e uses D = Dtab[9 mat[e] ..], t = ttab[mat[e]]),
// disjoint plates of different materials assemble in one launch; each plate's entries are then
// exactly what assemble_stiffness gives for that plate alone.
__global__ void __launch_bounds__(128) k_assemble(
    int n_nodes, const double* __restrict__ xy, const int* __restrict__ tri,
    const int* __restrict__ ne_ptr, const int* __restrict__ ne, const int* __restrict__ slot,
    const int* __restrict__ node_ptr, const Mat3 Dm, double thickness,
    const int* __restrict__ mat, const double* __restrict__ Dtab, const double* __restrict__ ttab,
    double* __restrict__ vals) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  const int b0 = node_ptr[n], deg = node_ptr[n + 1] - b0;
  double* ra = vals + 4L * b0;
  double* rb = ra + 2 * deg;
  for (int k = 0; k < 4 * deg; ++k) ra[k] = 0.0;
  for (int q = ne_ptr[n]; q < ne_ptr[n + 1]; ++q) {
    const int code = ne[q], e = code / 3, a = code - 3 * e;
    double exy[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int v = tri[3 * e + c];
      exy[2 * c] = xy[2 * v];
      exy[2 * c + 1] = xy[2 * v + 1];
    }
    CstB o;
    if (mat) {
      const int mi = mat[e];
      cst_element(exy, Dtab + 9 * mi, ttab[mi], o);
    } else {
      cst_element(exy, Dm.v, thickness, o);
    }
    // the corner's rows with compile-time indices (B and DB stay in registers)
    if (a == 0)
      add_corner_rows<0>(o, slot + 3 * q, b0, ra, rb);
    else if (a == 1)
      add_corner_rows<1>(o, slot + 3 * q, b0, ra, rb);
    else
      add_corner_rows<2>(o, slot + 3 * q, b0, ra, rb);
  }
}

// ---------------------------------------------------------------------------------------
// Dirichlet elimination (bc.cpp:137-166)

__global__ void k_dir_scatter(int n_fixed, const int* __restrict__ dofs,
                              const double* __restrict__ values, int n_rows,
                              unsigned char* __restrict__ fixed, double* __restrict__ ubar, int* err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_fixed) return;
  const int d = dofs[q];
  if (d < 0 || d >= n_rows) {
    atomicMin(&err[kErrRange], q);
    return;
  }
  fixed[d] = 1;
  ubar[d] = values[q];
}

// A DOF listed twice with different values is a conflict (DirichletDofs::add). After the
// scatter one of the values is stored; any entry that differs from it reveals the conflict.
__global__ void k_dir_verify(int n_fixed, const int* __restrict__ dofs,
                             const double* __restrict__ values, int n_rows,
                             const double* __restrict__ ubar, int* err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_fixed) return;
  const int d = dofs[q];
  if (d < 0 || d >= n_rows) return;
  const double u = ubar[d], v = values[q];
  if (u != v && __double_as_longlong(u) != __double_as_longlong(v)) atomicMin(&err[kErrConflict], d);
}

__device__ __forceinline__ int find_col(const int* __restrict__ cols, int lo, int hi, int col) {
  const int end = hi;
  while (lo < hi) {
    const int mid = lo + ((hi - lo) >> 1);
    if (cols[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo != end && cols[lo] == col) ? lo : -1;
}

// One thread per row; the row's entries are visited in ascending position, so b_i receives
// its corrections in the reference's order.
// Several load vectors sharing K (n_rhs vectors, `ld` doubles apart) are eliminated in one
// pass: each b receives exactly the corrections a separate apply_dirichlet would give it, and
// K is zeroed once, after every vector has read the entries.
__global__ void k_dir_apply(int n_rows, const int* __restrict__ row_ptr,
                            const int* __restrict__ cols, double* __restrict__ vals,
                            const unsigned char* __restrict__ fixed,
                            const double* __restrict__ ubar, double* __restrict__ b, int n_rhs,
                            long long ld, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rows) return;
  const int lo = row_ptr[i], hi = row_ptr[i + 1];
  if (fixed[i]) {
    const int kd = find_col(cols, lo, hi, i);
    const double diag = kd >= 0 ? vals[kd] : 0.0;
    if (!(diag > 0.0)) {
      atomicMin(&err[kErrDiag], i);
      return;
    }
    for (int k = lo; k < hi; ++k)
      if (cols[k] != i) vals[k] = 0.0;
    for (int q = 0; q < n_rhs; ++q) b[q * ld + i] = __dmul_rn(diag, ubar[i]);
  } else {
    for (int q = 0; q < n_rhs; ++q) {
      double bi = b[q * ld + i];
      for (int k = lo; k < hi; ++k) {
        const int c = cols[k];
        if (fixed[c]) bi = __dsub_rn(bi, __dmul_rn(vals[k], ubar[c]));
      }
      b[q * ld + i] = bi;
    }
    for (int k = lo; k < hi; ++k)
      if (fixed[cols[k]]) vals[k] = 0.0;
  }
}

// CgJacobiSolver::setup (solver.cpp:133-148)
__global__ void k_inv_diag(int n_rows, const int* __restrict__ row_ptr,
                           const int* __restrict__ cols, const double* __restrict__ vals,
                           double* __restrict__ inv_diag, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rows) return;
  const int kd = find_col(cols, row_ptr[i], row_ptr[i + 1], i);
  const double d = kd >= 0 ? vals[kd] : 0.0;
  if (!(d > 0.0)) {
    atomicMin(&err[kErrDiag], i);
    inv_diag[i] = 0.0;
    return;
  }
  inv_diag[i] = __ddiv_rn(1.0, d);
}

// ---------------------------------------------------------------------------------------
// compute_element_stresses (postprocess.cpp:35-60, element.cpp:57-81)
__global__ void k_element_stresses(int n_tri, const double* __restrict__ xy,
                                   const int* __restrict__ tri, const double* __restrict__ u,
                                   const Mat3 Dm, double nu, int plane_strain,
                                   double* __restrict__ out) {
  const double* Dg = Dm.v;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_tri) return;
  double exy[6], ue[6], B[18];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int v = tri[3 * e + c];
    exy[2 * c] = xy[2 * v];
    exy[2 * c + 1] = xy[2 * v + 1];
    ue[2 * c] = u[2 * v];
    ue[2 * c + 1] = u[2 * v + 1];
  }
  cst_B(exy, B);
  double eps[3], sig[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) s = __dadd_rn(s, __dmul_rn(B[i * 6 + j], ue[j]));
    eps[i] = s;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) s = __dadd_rn(s, __dmul_rn(Dg[i * 3 + j], eps[j]));
    sig[i] = s;
  }
  const double sx = sig[0], sy = sig[1], txy = sig[2];
  const double sz = plane_strain ? __dmul_rn(nu, __dadd_rn(sx, sy)) : 0.0;
  const double d1 = __dsub_rn(sx, sy), d2 = __dsub_rn(sy, sz), d3 = __dsub_rn(sz, sx);
  const double j2x2 = __dadd_rn(__dadd_rn(__dmul_rn(d1, d1), __dmul_rn(d2, d2)), __dmul_rn(d3, d3));
  const double vm = sqrt(__dadd_rn(__dmul_rn(0.5, j2x2), __dmul_rn(__dmul_rn(3.0, txy), txy)));
  const long ne = n_tri;
  out[0 * ne + e] = sx;
  out[1 * ne + e] = sy;
  out[2 * ne + e] = txy;
  out[3 * ne + e] = vm;
  out[4 * ne + e] = sz;
  out[5 * ne + e] = __ddiv_rn(__dadd_rn(__dadd_rn(exy[0], exy[2]), exy[4]), 3.0);
  out[6 * ne + e] = __ddiv_rn(__dadd_rn(__dadd_rn(exy[1], exy[3]), exy[5]), 3.0);
  out[7 * ne + e] = fabs(signed_area(exy[0], exy[1], exy[2], exy[3], exy[4], exy[5]));
}

// ---------------------------------------------------------------------------------------
// host launchers

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

cudaError_t launch_incidence(const MeshDev& m, int* cnt, int* cursor, int* ne_ptr, int* ne,
                             int* scan_tmp, int* err, cudaStream_t s) {
  cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)m.n_nodes, s);
  cudaMemsetAsync(cursor, 0, sizeof(int) * (size_t)m.n_nodes, s);
  const long ninc = 3L * m.n_tri;
  if (ninc) k_count_incidence<<<nblk(ninc, 256), 256, 0, s>>>(m.n_tri, m.tri, m.n_nodes, cnt, err);
  scan_exclusive(cnt, m.n_nodes, ne_ptr, scan_tmp, s);
  if (ninc) k_fill_incidence<<<nblk(ninc, 256), 256, 0, s>>>(m.n_tri, m.tri, m.n_nodes, ne_ptr, cursor, ne);
  if (m.n_nodes) k_sort_incidence<<<nblk(m.n_nodes, 128), 128, 0, s>>>(m.n_nodes, ne_ptr, ne);
  count_launches((ninc ? 2 : 0) + (m.n_nodes ? 1 : 0));
  return cudaGetLastError();
}

cudaError_t launch_pattern_count(const MeshDev& m, const int* ne_ptr, const int* ne, int* deg,
                                 int* node_ptr, int* scan_tmp, int* err, cudaStream_t s) {
  if (m.n_nodes)
    k_pattern_count<<<nblk(m.n_nodes, 128), 128, 0, s>>>(m.n_nodes, ne_ptr, ne, m.tri, deg, err);
  count_launches(m.n_nodes ? 1 : 0);
  return scan_exclusive(deg, m.n_nodes, node_ptr, scan_tmp, s);
}

cudaError_t launch_pattern_fill(const MeshDev& m, const int* ne_ptr, const int* ne,
                                const int* node_ptr, int* bnbr, int* slot, int* row_ptr,
                                int* cols, cudaStream_t s) {
  k_pattern_fill<<<nblk(m.n_nodes, 128), 128, 0, s>>>(m.n_nodes, ne_ptr, ne, m.tri, node_ptr, bnbr,
                                                      slot, row_ptr, cols);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const MeshDev& m, const int* ne_ptr, const int* ne, const int* slot,
                            const int* node_ptr, const Mat3& D, double t, const int* mat,
                            const double* Dtab, const double* ttab, double* vals, cudaStream_t s) {
  k_assemble<<<nblk(m.n_nodes, 128), 128, 0, s>>>(m.n_nodes, m.xy, m.tri, ne_ptr, ne, slot, node_ptr,
                                                  D, t, mat, Dtab, ttab, vals);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_dirichlet(int n_rows, const int* row_ptr, const int* cols, double* vals,
                             int n_fixed, const int* dofs, const double* values,
                             unsigned char* fixed, double* ubar, double* b, int n_rhs,
                             int* err, cudaStream_t s, bool apply) {
  if (!apply) {
    cudaMemsetAsync(fixed, 0, (size_t)n_rows, s);
    if (n_fixed) {
      k_dir_scatter<<<nblk(n_fixed, 256), 256, 0, s>>>(n_fixed, dofs, values, n_rows, fixed, ubar, err);
      k_dir_verify<<<nblk(n_fixed, 256), 256, 0, s>>>(n_fixed, dofs, values, n_rows, ubar, err);
      count_launches(2);
    }
  } else {
    if (n_rows)
      k_dir_apply<<<nblk(n_rows, 128), 128, 0, s>>>(n_rows, row_ptr, cols, vals, fixed, ubar, b, n_rhs,
                                                    (long long)n_rows, err);
    count_launches(n_rows ? 1 : 0);
  }
  return cudaGetLastError();
}

cudaError_t launch_inv_diag(int n_rows, const int* row_ptr, const int* cols, const double* vals,
                            double* inv_diag, int* err, cudaStream_t s) {
  k_inv_diag<<<nblk(n_rows, 256), 256, 0, s>>>(n_rows, row_ptr, cols, vals, inv_diag, err);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_element_stresses(const MeshDev& m, const double* u, const Mat3& D, double nu,
                                    int plane_strain, double* out, cudaStream_t s) {
  if (m.n_tri)
    k_element_stresses<<<nblk(m.n_tri, 128), 128, 0, s>>>(m.n_tri, m.xy, m.tri, u, D, nu,
                                                           plane_strain, out);
  count_launches(m.n_tri ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace cstg
