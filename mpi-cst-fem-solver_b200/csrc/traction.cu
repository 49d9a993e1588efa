// add_traction on the GPU (bc.cpp:190-253): consistent nodal forces of a traction on line
// edges, 2-point Gauss rule, outward normal from the adjacent triangle.
//
// Per edge (one thread): the adjacent triangle and its opposite node (from the node ->
// triangle incidence of the pattern builder), the length, the outward normal and the four
// contributions (node a and node b, both Gauss points) with the reference's operations in the
// reference's order (explicit round-to-nearest intrinsics: no FMA contraction). Per node (one
// thread): f[2n], f[2n+1] receive their contributions in ascending edge order, Gauss point
// -1/sqrt(3) before +1/sqrt(3), exactly the sequence of additions of the reference's loop, so a
// constant traction gives bit-identical loads. The analytic Kirsch traction (kirsch.cpp:40-45)
// uses CUDA's atan2 / sin / cos, which are not bit-identical to the host library's.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace cstg {

namespace {

// sqrt(x^2 + y^2) rounded to nearest: h = sqrt(fl(x^2 + y^2)) is corrected by one Newton step
// e / (2h), with e = x^2 + y^2 - h^2 evaluated exactly from the fma residues of the three
// squares (x_sq - h_sq is exact: x <= h <= sqrt(2) x). This is the correction scheme of
// C. F. Borges, "An improved algorithm for hypot(a, b)" (2019). Mesh coordinates need no
// rescaling (no overflow or underflow of the squares).
__device__ __forceinline__ double hypot_rn(double x, double y) {
  x = fabs(x);
  y = fabs(y);
  if (x < y) {
    const double t = x;
    x = y;
    y = t;
  }
  if (y == 0.0) return x;
  const double y_sq = __dmul_rn(y, y);
  const double h = __dsqrt_rn(__fma_rn(x, x, y_sq));
  const double h_sq = __dmul_rn(h, h), x_sq = __dmul_rn(x, x);
  const double h_err = __fma_rn(h, h, -h_sq), x_err = __fma_rn(x, x, -x_sq), y_err = __fma_rn(y, y, -y_sq);
  const double e = __dadd_rn(__dadd_rn(__dsub_rn(x_sq, h_sq), y_sq), __dsub_rn(__dadd_rn(x_err, y_err), h_err));
  return __dadd_rn(h, __ddiv_rn(e, __dmul_rn(2.0, h)));
}

// Kirsch field's traction sigma . n at (x, y) (kirsch.cpp:7-45)
__device__ void kirsch_traction(double a, double s, double x, double y, double nx, double ny, double& t0,
                                double& t1) {
  const double r = hypot(x, y), th = atan2(y, x);
  const double q2 = (a * a) / (r * r), q4 = q2 * q2;
  const double c2 = cos(2.0 * th), s2 = sin(2.0 * th);
  const double rr = 0.5 * s * (1.0 - q2) + 0.5 * s * (1.0 - 4.0 * q2 + 3.0 * q4) * c2;
  const double tt = 0.5 * s * (1.0 + q2) - 0.5 * s * (1.0 + 3.0 * q4) * c2;
  const double rt = -0.5 * s * (1.0 + 2.0 * q2 - 3.0 * q4) * s2;
  const double c = cos(th), n = sin(th);
  const double sxx = rr * c * c + tt * n * n - 2.0 * rt * n * c;
  const double syy = rr * n * n + tt * c * c + 2.0 * rt * n * c;
  const double sxy = (rr - tt) * n * c + rt * (c * c - n * n);
  t0 = sxx * nx + sxy * ny;
  t1 = sxy * nx + syy * ny;
}

// Contributions of edge q: con[8q ..] = (a: q1x, q1y, q2x, q2y, b: q1x, q1y, q2x, q2y)
__global__ void k_trac_edges(int n_edges, const int* __restrict__ edges, int n_nodes, const double* __restrict__ xy,
                             const int* __restrict__ tri, const int* __restrict__ ne_ptr,
                             const int* __restrict__ ne, double thickness, int kind, double p0, double p1, double g,
                             double* __restrict__ con, int* __restrict__ cnt, int* err) {
  // cnt[n]: the number of (valid) edges touching node n
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_edges) return;
  const int a = edges[2 * q], b = edges[2 * q + 1];
  if (a < 0 || a >= n_nodes || b < 0 || b >= n_nodes) {
    atomicMin(&err[kErrRange], q);
    return;
  }
  int count = 0, c = -1;
  for (int k = ne_ptr[a]; k < ne_ptr[a + 1]; ++k) {
    const int e = ne[k] / 3;
    const int* t = tri + 3 * (size_t)e;
    for (int s = 0; s < 3; ++s) {
      const int u = t[s], v = t[(s + 1) % 3];
      if ((u == a && v == b) || (u == b && v == a)) {
        ++count;
        c = t[(s + 2) % 3];
      }
    }
  }
  if (count != 1) {
    atomicMin(&err[kErrEdge], q);
    return;
  }
  atomicAdd(&cnt[a], 1);
  atomicAdd(&cnt[b], 1);
  const double xa = xy[2 * a], ya = xy[2 * a + 1], xb = xy[2 * b], yb = xy[2 * b + 1];
  const double dx = __dsub_rn(xb, xa), dy = __dsub_rn(yb, ya);
  const double len = hypot_rn(dx, dy);
  double nx = __ddiv_rn(dy, len), ny = __ddiv_rn(-dx, len);
  if (__dadd_rn(__dmul_rn(nx, __dsub_rn(xy[2 * c], xa)), __dmul_rn(ny, __dsub_rn(xy[2 * c + 1], ya))) > 0.0) {
    nx = -nx;
    ny = -ny;
  }
  const double w = __dmul_rn(__dmul_rn(thickness, 0.5), len);
  double* o = con + 8 * (size_t)q;
  for (int i = 0; i < 2; ++i) {
    const double xi = i == 0 ? -g : g;
    const double Na = __dmul_rn(0.5, __dsub_rn(1.0, xi)), Nb = __dmul_rn(0.5, __dadd_rn(1.0, xi));
    double t0 = p0, t1 = p1;
    if (kind == CSTG_TRACTION_STRESS) {  // sigma . n of the uniform stress diag(p0, p1)
      t0 = __dmul_rn(p0, nx);
      t1 = __dmul_rn(p1, ny);
    } else if (kind == CSTG_TRACTION_KIRSCH) {
      const double x = __dadd_rn(__dmul_rn(Na, xa), __dmul_rn(Nb, xb));
      const double y = __dadd_rn(__dmul_rn(Na, ya), __dmul_rn(Nb, yb));
      kirsch_traction(p0, p1, x, y, nx, ny, t0, t1);
    }
    const double wa = __dmul_rn(w, Na), wb = __dmul_rn(w, Nb);
    o[2 * i] = __dmul_rn(wa, t0);
    o[2 * i + 1] = __dmul_rn(wa, t1);
    o[4 + 2 * i] = __dmul_rn(wb, t0);
    o[4 + 2 * i + 1] = __dmul_rn(wb, t1);
  }
}

// records (edge << 1 | role) per node, then sorted ascending per node
__global__ void k_trac_fill(int n_edges, const int* __restrict__ edges, const int* __restrict__ ptr,
                            int* __restrict__ cur, int* __restrict__ rec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_edges) return;
  const int a = edges[2 * q], b = edges[2 * q + 1];
  rec[ptr[a] + atomicAdd(&cur[a], 1)] = 2 * q;
  rec[ptr[b] + atomicAdd(&cur[b], 1)] = 2 * q + 1;
}

__global__ void k_trac_gather(int n_nodes, const int* __restrict__ ptr, int* __restrict__ rec,
                              const double* __restrict__ con, double* __restrict__ f) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  const int lo = ptr[n], hi = ptr[n + 1];
  if (lo == hi) return;
  for (int i = lo + 1; i < hi; ++i) {  // few records per node: insertion sort
    const int v = rec[i];
    int j = i - 1;
    while (j >= lo && rec[j] > v) {
      rec[j + 1] = rec[j];
      --j;
    }
    rec[j + 1] = v;
  }
  double fx = f[2 * n], fy = f[2 * n + 1];
  for (int i = lo; i < hi; ++i) {
    const int q = rec[i] >> 1, role = rec[i] & 1;
    const double* o = con + 8 * (size_t)q + 4 * role;
    fx = __dadd_rn(fx, o[0]);
    fy = __dadd_rn(fy, o[1]);
    fx = __dadd_rn(fx, o[2]);
    fy = __dadd_rn(fy, o[3]);
  }
  f[2 * n] = fx;
  f[2 * n + 1] = fy;
}

// Host-array tractions move only the loaded nodes' entries: dir = 0 scatters the compact values
// (2 per node, in `nodes` order) into f, dir = 1 gathers them back.
__global__ void k_trac_compact(int m, const int* __restrict__ nodes, double* __restrict__ fc, double* __restrict__ f,
                               int dir) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int n = nodes[i];
  if (dir == 0) {
    f[2 * (size_t)n] = fc[2 * i];
    f[2 * (size_t)n + 1] = fc[2 * i + 1];
  } else {
    fc[2 * i] = f[2 * (size_t)n];
    fc[2 * i + 1] = f[2 * (size_t)n + 1];
  }
}

}  // namespace

cudaError_t launch_traction_compact(int m, const int* nodes, double* fc, double* f, int dir, cudaStream_t s) {
  if (m <= 0) return cudaSuccess;
  k_trac_compact<<<(m + 255) / 256, 256, 0, s>>>(m, nodes, fc, f, dir);
  count_launches(1);
  return cudaGetLastError();
}

// Phase 1: per-edge contributions and per-node record counts (the caller checks the error word
// before phase 2; a failed edge leaves f untouched).
cudaError_t launch_traction_edges(int n_edges, const int* edges, const MeshDev& m, const int* ne_ptr, const int* ne,
                                  double thickness, int kind, double p0, double p1, double* con, int* cnt, int* err,
                                  cudaStream_t s) {
  const int N = m.n_nodes;
  if (n_edges <= 0 || N <= 0) return cudaSuccess;
  const double g = 1.0 / sqrt(3.0);  // 2-point Gauss abscissa (bc.cpp:213)
  cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)N, s);
  k_trac_edges<<<(n_edges + 127) / 128, 128, 0, s>>>(n_edges, edges, N, m.xy, m.tri, ne_ptr, ne, thickness, kind, p0,
                                                     p1, g, con, cnt, err);
  count_launches(1);
  return cudaGetLastError();
}

// Phase 2: per-node records sorted by edge, then f += contributions in the reference's order.
cudaError_t launch_traction_apply(int n_edges, const int* edges, int n_nodes, const double* con, const int* cnt,
                                  int* ptr, int* cur, int* rec, int* scan_tmp, double* f, cudaStream_t s) {
  if (n_edges <= 0 || n_nodes <= 0) return cudaSuccess;
  cudaError_t e = scan_exclusive(cnt, n_nodes, ptr, scan_tmp, s);
  if (e != cudaSuccess) return e;
  cudaMemsetAsync(cur, 0, sizeof(int) * (size_t)n_nodes, s);
  k_trac_fill<<<(n_edges + 127) / 128, 128, 0, s>>>(n_edges, edges, ptr, cur, rec);
  k_trac_gather<<<(n_nodes + 255) / 256, 256, 0, s>>>(n_nodes, ptr, rec, con, f);
  count_launches(2);
  return cudaGetLastError();
}

}  // namespace cstg
