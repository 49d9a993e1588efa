/*
 * CPU oracle for the CST assembly -> Dirichlet elimination -> Jacobi-PCG path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C restatement of the reference
 * (FreddyJuka/mpi-cst-fem-solver) serial core. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it, and only as the checker. The GPU library never
 * links or calls it.
 *
 * Every function repeats the reference's floating-point operations in the reference's
 * order, with no FMA contraction (the Makefile passes -ffp-contract=off; x86-64 g++ -O3
 * without -march does not contract either). Results are therefore bit-identical to the
 * reference for the same inputs. Each function names the reference lines it follows.
 *
 * Parity is pinned in tests/test_oracle.py: against the reference's own known answers
 * (tests/test_element.cpp:60-84, tests/test_bc.cpp:169-184, tests/test_pcg.cpp:58-102)
 * and bit-for-bit against the reference compiled from source (oracle/_ref), through the
 * golden fixtures under tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OR_OK 0
#define OR_ERR_ARG 1
#define OR_ERR_BAD_DIAGONAL 3
#define OR_ERR_PATTERN 7
#define OR_ERR_EDGE 11

static char g_msg[512];
const char* or_last_message(void) { return g_msg; }

/* ---- element: include/cstfem/element.hpp, src/element.cpp ------------------------------ */

/* element.cpp:7-15 */
void or_constitutive(double E, double nu, int plane_strain, double D[9]) {
  if (!plane_strain) {
    const double c = E / (1.0 - nu * nu);
    const double v[9] = {c, c * nu, 0.0, c * nu, c, 0.0, 0.0, 0.0, c * (1.0 - nu) / 2.0};
    memcpy(D, v, sizeof v);
  } else {
    const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double v[9] = {c * (1.0 - nu), c * nu, 0.0, c * nu, c * (1.0 - nu), 0.0,
                         0.0, 0.0, c * (1.0 - 2.0 * nu) / 2.0};
    memcpy(D, v, sizeof v);
  }
}

/* element.cpp:17-19 (xy = x1,y1,x2,y2,x3,y3) */
double or_signed_area(const double xy[6]) {
  return 0.5 * ((xy[2] - xy[0]) * (xy[5] - xy[1]) - (xy[4] - xy[0]) * (xy[3] - xy[1]));
}

/* element.cpp:21-35: B is 3x6 row-major */
void or_cst_B(const double xy[6], double B[18]) {
  const double x1 = xy[0], y1 = xy[1], x2 = xy[2], y2 = xy[3], x3 = xy[4], y3 = xy[5];
  const double b[3] = {y2 - y3, y3 - y1, y1 - y2};
  const double c[3] = {x3 - x2, x1 - x3, x2 - x1};
  const double inv2A = 1.0 / (2.0 * or_signed_area(xy));
  memset(B, 0, 18 * sizeof(double));
  for (int i = 0; i < 3; ++i) {
    B[0 * 6 + 2 * i] = b[i] * inv2A;
    B[1 * 6 + 2 * i + 1] = c[i] * inv2A;
    B[2 * 6 + 2 * i] = c[i] * inv2A;
    B[2 * 6 + 2 * i + 1] = b[i] * inv2A;
  }
}

/* element.cpp:37-55: upper triangle computed, mirrored to the lower one */
void or_cst_stiffness(const double xy[6], const double D[9], double thickness, double K[36]) {
  double B[18], DB[18];
  or_cst_B(xy, B);
  memset(DB, 0, sizeof DB);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 6; ++j)
      for (int k = 0; k < 3; ++k) DB[i * 6 + j] += D[i * 3 + k] * B[k * 6 + j];
  const double scale = thickness * fabs(or_signed_area(xy));
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += B[k * 6 + i] * DB[k * 6 + j];
      K[i * 6 + j] = K[j * 6 + i] = scale * s;
    }
}

/* element.cpp:57-81 (strain, stress, sigma_zz, von Mises) */
void or_element_stress(const double xy[6], const double ue[6], const double D[9], double nu,
                       int plane_strain, double out[5] /* sxx syy txy szz vm */) {
  double B[18], e[3] = {0, 0, 0}, s[3] = {0, 0, 0};
  or_cst_B(xy, B);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 6; ++j) e[i] += B[i * 6 + j] * ue[j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s[i] += D[i * 3 + j] * e[j];
  const double sz = plane_strain ? nu * (s[0] + s[1]) : 0.0;
  const double sx = s[0], sy = s[1], txy = s[2];
  const double j2x2 = (sx - sy) * (sx - sy) + (sy - sz) * (sy - sz) + (sz - sx) * (sz - sx);
  out[0] = sx;
  out[1] = sy;
  out[2] = txy;
  out[3] = sz;
  out[4] = sqrt(0.5 * j2x2 + 3.0 * txy * txy);
}

/* ---- pattern and assembly: src/assembly.cpp, src/csr.cpp ------------------------------- */

static int cmp_int(const void* a, const void* b) {
  const int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/*
 * assembly.cpp:9-42. Node adjacency through triangles (self included), sorted and unique;
 * rows 2n and 2n+1 both list (2m, 2m+1) for every neighbour m in ascending order.
 * Call with cols == NULL to get the row pointer (and nnz) only; then again with cols.
 * Returns nnz, or -1 on a node index out of range.
 */
long long or_build_pattern(int n_nodes, int n_tri, const int* tri, int* row_ptr, int* cols) {
  int* cnt = (int*)calloc((size_t)n_nodes + 1, sizeof(int));
  for (int n = 0; n < n_nodes; ++n) cnt[n + 1] = 1; /* self */
  for (long e = 0; e < n_tri; ++e)
    for (int a = 0; a < 3; ++a) {
      const int v = tri[3 * e + a];
      if (v < 0 || v >= n_nodes) {
        free(cnt);
        snprintf(g_msg, sizeof g_msg, "triangle %ld: node %d out of range", e, v);
        return -1;
      }
      cnt[v + 1] += 2;
    }
  for (int n = 0; n < n_nodes; ++n) cnt[n + 1] += cnt[n];
  int* adj = (int*)malloc(sizeof(int) * (size_t)(cnt[n_nodes] > 0 ? cnt[n_nodes] : 1));
  int* fill = (int*)malloc(sizeof(int) * (size_t)(n_nodes > 0 ? n_nodes : 1));
  for (int n = 0; n < n_nodes; ++n) {
    adj[cnt[n]] = n;
    fill[n] = cnt[n] + 1;
  }
  for (long e = 0; e < n_tri; ++e) {
    const int* t = &tri[3 * e];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (a != b) adj[fill[t[a]]++] = t[b];
  }
  long long nnz = 0;
  int* len = fill; /* reuse: unique length per node */
  for (int n = 0; n < n_nodes; ++n) {
    int* a = adj + cnt[n];
    const int m = cnt[n + 1] - cnt[n];
    qsort(a, (size_t)m, sizeof(int), cmp_int);
    int u = 0;
    for (int k = 0; k < m; ++k)
      if (k == 0 || a[k] != a[u - 1]) a[u++] = a[k];
    len[n] = u;
    if (row_ptr) {
      row_ptr[2 * n] = (int)nnz;
      row_ptr[2 * n + 1] = (int)(nnz + 2 * u);
    }
    nnz += 4LL * u;
  }
  if (row_ptr) row_ptr[2 * n_nodes] = (int)nnz;
  if (cols) {
    long long k = 0;
    for (int n = 0; n < n_nodes; ++n)
      for (int c = 0; c < 2; ++c)
        for (int q = 0; q < len[n]; ++q) {
          cols[k++] = 2 * adj[cnt[n] + q];
          cols[k++] = 2 * adj[cnt[n] + q] + 1;
        }
  }
  free(adj);
  free(fill);
  free(cnt);
  return nnz;
}

/* csr.cpp:7-12: lower_bound in the sorted row */
static int csr_find(const int* row_ptr, const int* cols, int row, int col) {
  int lo = row_ptr[row], hi = row_ptr[row + 1];
  const int end = hi;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (cols[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo != end && cols[lo] == col) ? lo : -1;
}

/* assembly.cpp:44-74: zero, then add Ke of every triangle in element order */
int or_assemble(int n_nodes, const double* xy, int n_tri, const int* tri, const double D[9],
                double thickness, const int* row_ptr, const int* cols, double* vals) {
  const long long nnz = row_ptr[2 * n_nodes];
  for (long long k = 0; k < nnz; ++k) vals[k] = 0.0;
  for (long e = 0; e < n_tri; ++e) {
    double exy[6], Ke[36];
    int dofs[6];
    for (int k = 0; k < 3; ++k) {
      const int n = tri[3 * e + k];
      exy[2 * k] = xy[2 * n];
      exy[2 * k + 1] = xy[2 * n + 1];
      dofs[2 * k] = 2 * n;
      dofs[2 * k + 1] = 2 * n + 1;
    }
    or_cst_stiffness(exy, D, thickness, Ke);
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        const int pos = csr_find(row_ptr, cols, dofs[i], dofs[j]);
        if (pos < 0) {
          snprintf(g_msg, sizeof g_msg, "assemble_stiffness: entry (%d, %d) missing from the pattern",
                   dofs[i], dofs[j]);
          return OR_ERR_PATTERN;
        }
        vals[pos] += Ke[i * 6 + j];
      }
  }
  return OR_OK;
}

/* csr.cpp:19-26 */
void or_spmv(int n_rows, const int* row_ptr, const int* cols, const double* vals, const double* x,
             double* y) {
  for (int i = 0; i < n_rows; ++i) {
    double s = 0.0;
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += vals[k] * x[cols[k]];
    y[i] = s;
  }
}

/* ---- Dirichlet: src/bc.cpp:137-166 ----------------------------------------------------- */

int or_apply_dirichlet(int n_rows, const int* row_ptr, const int* cols, double* vals, int n_fixed,
                       const int* dofs, const double* values, double* b) {
  char* fixed = (char*)calloc((size_t)n_rows, 1);
  double* ubar = (double*)calloc((size_t)n_rows, sizeof(double));
  for (int q = 0; q < n_fixed; ++q) {
    if (dofs[q] < 0 || dofs[q] >= n_rows) {
      snprintf(g_msg, sizeof g_msg, "apply_dirichlet: DOF %d out of range", dofs[q]);
      free(fixed);
      free(ubar);
      return OR_ERR_ARG;
    }
    fixed[dofs[q]] = 1;
    ubar[dofs[q]] = values[q];
  }
  int rc = OR_OK;
  for (int i = 0; i < n_rows; ++i) {
    if (fixed[i]) {
      const int kd = csr_find(row_ptr, cols, i, i);
      const double diag = kd >= 0 ? vals[kd] : 0.0;
      if (!(diag > 0.0)) {
        snprintf(g_msg, sizeof g_msg, "apply_dirichlet: non-positive diagonal at DOF %d", i);
        rc = OR_ERR_BAD_DIAGONAL;
        break;
      }
      for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        if (cols[k] != i) vals[k] = 0.0;
      b[i] = diag * ubar[i];
    } else {
      for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
        if (fixed[cols[k]]) {
          b[i] -= vals[k] * ubar[cols[k]];
          vals[k] = 0.0;
        }
    }
  }
  free(fixed);
  free(ubar);
  return rc;
}

/* ---- traction loads: src/bc.cpp:190-253 (constant traction) ----------------------------- */

typedef struct {
  uint64_t key;
  int opposite;
} edge_rec;

static uint64_t edge_key(int a, int b) {
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}

static int cmp_edge(const void* a, const void* b) {
  const uint64_t x = ((const edge_rec*)a)->key, y = ((const edge_rec*)b)->key;
  return (x > y) - (x < y);
}

/*
 * Consistent nodal forces of a constant traction (tx, ty) on the given edges, 2-point Gauss,
 * outward normal from the single adjacent triangle. Edges are visited in the given order,
 * so the additions to f happen in the reference's order.
 */
int or_add_traction(int n_nodes, const double* xy, int n_tri, const int* tri, int n_edges,
                    const int* edges, double thickness, double tx, double ty, double* f) {
  (void)n_nodes;
  edge_rec* all = (edge_rec*)malloc(sizeof(edge_rec) * (size_t)(3 * (long)n_tri + 1));
  for (long t = 0; t < n_tri; ++t)
    for (int k = 0; k < 3; ++k) {
      all[3 * t + k].key = edge_key(tri[3 * t + k], tri[3 * t + (k + 1) % 3]);
      all[3 * t + k].opposite = tri[3 * t + (k + 2) % 3];
    }
  qsort(all, (size_t)(3 * (long)n_tri), sizeof(edge_rec), cmp_edge);
  const double g = 1.0 / sqrt(3.0);
  const double xi[2] = {-g, g};
  int rc = OR_OK;
  for (int q = 0; q < n_edges && rc == OR_OK; ++q) {
    const int a = edges[2 * q], b = edges[2 * q + 1];
    const uint64_t key = edge_key(a, b);
    long lo = 0, hi = 3 * (long)n_tri;
    while (lo < hi) {
      const long mid = lo + (hi - lo) / 2;
      if (all[mid].key < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    int count = 0, c = -1;
    for (long k = lo; k < 3 * (long)n_tri && all[k].key == key; ++k) {
      ++count;
      c = all[k].opposite;
    }
    if (count != 1) {
      snprintf(g_msg, sizeof g_msg, "traction edge (%d, %d) is adjacent to %d triangles (expected 1)",
               a, b, count);
      rc = OR_ERR_EDGE;
      break;
    }
    const double xa = xy[2 * a], ya = xy[2 * a + 1];
    const double xb = xy[2 * b], yb = xy[2 * b + 1];
    const double len = hypot(xb - xa, yb - ya);
    double nx = (yb - ya) / len, ny = -(xb - xa) / len;
    if (nx * (xy[2 * c] - xa) + ny * (xy[2 * c + 1] - ya) > 0.0) {
      nx = -nx;
      ny = -ny;
    }
    (void)nx;
    (void)ny;
    for (int p = 0; p < 2; ++p) {
      const double Na = 0.5 * (1.0 - xi[p]), Nb = 0.5 * (1.0 + xi[p]);
      const double w = thickness * 0.5 * len;
      f[2 * a] += w * Na * tx;
      f[2 * a + 1] += w * Na * ty;
      f[2 * b] += w * Nb * tx;
      f[2 * b + 1] += w * Nb * ty;
    }
  }
  free(all);
  return rc;
}

/* ---- Jacobi-PCG: src/solver.cpp:35-148 ------------------------------------------------ */

typedef struct {
  int iterations;
  int converged;
  int breakdown;
  double rel_residual;
  double true_rel_residual;
} or_stats;

static double dot(long n, const double* a, const double* b) {
  double s = 0.0; /* solver.cpp:24-31: sequential order */
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/*
 * CgJacobiSolver::setup (solver.cpp:133-148) + pcg_jacobi (solver.cpp:109-131, 35-105).
 * history (optional, max_iter + 1 entries) receives ||r_k|| / ||b||.
 * Returns OR_ERR_BAD_DIAGONAL (with the row in the message) like setup() throws.
 */
int or_pcg_jacobi(int n, const int* row_ptr, const int* cols, const double* vals, const double* b,
                  double* x, double rtol, int max_iter, double* history, or_stats* st) {
  memset(st, 0, sizeof *st);
  double* inv_diag = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) {
    const int kd = csr_find(row_ptr, cols, i, i);
    const double d = kd >= 0 ? vals[kd] : 0.0;
    if (!(d > 0.0)) {
      snprintf(g_msg, sizeof g_msg, "cg_jacobi: non-positive diagonal at row %d", i);
      free(inv_diag);
      return OR_ERR_BAD_DIAGONAL;
    }
    inv_diag[i] = 1.0 / d;
  }
  for (int i = 0; i < n; ++i) x[i] = 0.0;
  const double bnorm = sqrt(dot(n, b, b));
  if (bnorm == 0.0) {
    st->converged = 1;
    if (history) history[0] = 0.0;
    free(inv_diag);
    snprintf(g_msg, sizeof g_msg, "zero right-hand side, x = 0");
    return OR_OK;
  }
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* Ap = (double*)malloc(sizeof(double) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    r[i] = b[i];
    z[i] = inv_diag[i] * r[i];
    p[i] = z[i];
  }
  double rz = dot(n, r, z);
  st->rel_residual = 1.0;
  if (history) history[0] = 1.0;
  int done = 0;
  for (int k = 1; k <= max_iter; ++k) {
    or_spmv(n, row_ptr, cols, vals, p, Ap);
    const double pAp = dot(n, p, Ap);
    if (!(pAp > 0.0)) {
      st->breakdown = 1;
      snprintf(g_msg, sizeof g_msg, "CG breakdown at iteration %d: p'Ap = %g (matrix not SPD?)", k,
               pAp);
      done = 2;
      break;
    }
    const double alpha = rz / pAp;
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    st->iterations = k;
    st->rel_residual = sqrt(dot(n, r, r)) / bnorm;
    if (history) history[k] = st->rel_residual;
    if (st->rel_residual < rtol) {
      st->converged = 1;
      snprintf(g_msg, sizeof g_msg, "converged in %d iterations, relative residual %g", k,
               st->rel_residual);
      done = 1;
      break;
    }
    for (int i = 0; i < n; ++i) z[i] = inv_diag[i] * r[i];
    const double rz_new = dot(n, r, z);
    const double beta = rz_new / rz;
    rz = rz_new;
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  if (!done)
    snprintf(g_msg, sizeof g_msg, "NOT converged: reached max_iter = %d, relative residual %g (rtol %g)",
             max_iter, st->rel_residual, rtol);
  /* solver.cpp:117-122: true residual */
  or_spmv(n, row_ptr, cols, vals, x, r);
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  st->true_rel_residual = sqrt(dot(n, r, r)) / bnorm;
  free(r);
  free(z);
  free(p);
  free(Ap);
  free(inv_diag);
  return OR_OK;
}
