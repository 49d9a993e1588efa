// C-ABI shim over the reference's own serial core, compiled from its sources by
// oracle/Makefile into oracle/_ref/libcstfem_ref.so.
//
// TEST INFRASTRUCTURE ONLY: tests/golden/make_golden.py uses it to pin the oracle
// restatement (oracle/cst_oracle.c) bit-for-bit, and bench.py's reference arm and CPU-baseline
// leg time the reference's CPU path through it. The GPU library never links it.
//
// Every entry point catches the reference's exceptions and returns a nonzero code; the
// message is kept for ref_last_message().
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "cstfem/assembly.hpp"
#include "cstfem/bc.hpp"
#include "cstfem/element.hpp"
#include "cstfem/mesh.hpp"
#include "cstfem/postprocess.hpp"
#include "cstfem/solver.hpp"

using namespace cstfem;

namespace {
thread_local std::string g_msg;

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_msg = e.what();
    return 1;
  }
}
}  // namespace

extern "C" {

const char* ref_last_message() { return g_msg.c_str(); }

// ---- mesh -------------------------------------------------------------------------------
void* ref_mesh_create(int n_nodes, const double* xy, int n_tri, const int32_t* tri) {
  auto* m = new Mesh;
  m->xy.assign(xy, xy + 2 * static_cast<std::size_t>(n_nodes));
  m->node_tags.resize(n_nodes);
  for (int i = 0; i < n_nodes; ++i) m->node_tags[i] = static_cast<std::size_t>(i) + 1;
  m->triangles.assign(tri, tri + 3 * static_cast<std::size_t>(n_tri));
  return m;
}

void ref_mesh_add_group(void* mesh, const char* name, int n_edges, const int32_t* edges) {
  auto& v = static_cast<Mesh*>(mesh)->boundary_edges[name];
  for (int i = 0; i < n_edges; ++i) v.push_back({edges[2 * i], edges[2 * i + 1]});
}

void* ref_mesh_read(const char* path) {
  Mesh* out = nullptr;
  if (guarded([&] { out = new Mesh(read_gmsh(std::string(path))); })) return nullptr;
  return out;
}

void ref_mesh_info(void* mesh, int* n_nodes, int* n_tri, int* flipped) {
  auto* m = static_cast<Mesh*>(mesh);
  *n_nodes = static_cast<int>(m->num_nodes());
  *n_tri = static_cast<int>(m->num_triangles());
  *flipped = m->flipped_triangles;
}

void ref_mesh_get(void* mesh, double* xy, int32_t* tri) {
  auto* m = static_cast<Mesh*>(mesh);
  std::memcpy(xy, m->xy.data(), m->xy.size() * sizeof(double));
  for (std::size_t i = 0; i < m->triangles.size(); ++i) tri[i] = m->triangles[i];
}

// Number of edges of group `name`, or -1 if the group does not exist; fills `edges` if given.
int ref_mesh_group(void* mesh, const char* name, int32_t* edges) {
  auto* m = static_cast<Mesh*>(mesh);
  const auto it = m->boundary_edges.find(name);
  if (it == m->boundary_edges.end()) return -1;
  if (edges)
    for (std::size_t i = 0; i < it->second.size(); ++i) {
      edges[2 * i] = it->second[i][0];
      edges[2 * i + 1] = it->second[i][1];
    }
  return static_cast<int>(it->second.size());
}

void ref_mesh_destroy(void* mesh) { delete static_cast<Mesh*>(mesh); }

// ---- element ------------------------------------------------------------------------------
void ref_constitutive(double E, double nu, int plane_strain, double* D) {
  const Mat3 d = constitutive_matrix(E, nu, plane_strain ? PlaneCondition::Strain
                                                         : PlaneCondition::Stress);
  std::memcpy(D, d.data(), sizeof(double) * 9);
}

void ref_cst_stiffness(const double* xy, const double* D, double t, double* K) {
  TriCoords c;
  Mat3 d;
  std::memcpy(c.data(), xy, sizeof(double) * 6);
  std::memcpy(d.data(), D, sizeof(double) * 9);
  const Mat6 k = cst_stiffness(c, d, t);
  std::memcpy(K, k.data(), sizeof(double) * 36);
}

// ---- CSR: build_stiffness_pattern, assemble_stiffness, apply_dirichlet ---------------------
void* ref_pattern(void* mesh) { return new CsrMatrix(build_stiffness_pattern(*static_cast<Mesh*>(mesh))); }

void* ref_csr_create(int n, const int32_t* row_ptr, const int32_t* cols, const double* vals) {
  auto* K = new CsrMatrix;
  K->num_rows = K->num_cols = n;
  K->row_ptr.assign(row_ptr, row_ptr + n + 1);
  K->cols.assign(cols, cols + row_ptr[n]);
  K->vals.assign(vals, vals + row_ptr[n]);
  return K;
}

long long ref_csr_nnz(void* K) { return static_cast<long long>(static_cast<CsrMatrix*>(K)->nnz()); }
int ref_csr_rows(void* K) { return static_cast<CsrMatrix*>(K)->num_rows; }

void ref_csr_get(void* Kp, int32_t* row_ptr, int32_t* cols, double* vals) {
  auto* K = static_cast<CsrMatrix*>(Kp);
  if (row_ptr)
    for (std::size_t i = 0; i < K->row_ptr.size(); ++i) row_ptr[i] = K->row_ptr[i];
  if (cols)
    for (std::size_t i = 0; i < K->cols.size(); ++i) cols[i] = K->cols[i];
  if (vals) std::memcpy(vals, K->vals.data(), K->vals.size() * sizeof(double));
}

void ref_csr_destroy(void* K) { delete static_cast<CsrMatrix*>(K); }

int ref_assemble(void* mesh, const double* D, double t, void* K) {
  Mat3 d;
  std::memcpy(d.data(), D, sizeof(double) * 9);
  return guarded([&] { assemble_stiffness(*static_cast<Mesh*>(mesh), d, t, *static_cast<CsrMatrix*>(K)); });
}

int ref_spmv(void* Kp, const double* x, double* y) {
  auto* K = static_cast<CsrMatrix*>(Kp);
  std::vector<double> xv(x, x + K->num_cols), yv;
  K->multiply(xv, yv);
  std::memcpy(y, yv.data(), yv.size() * sizeof(double));
  return 0;
}

int ref_add_traction(void* mesh, const char* group, double t, double tx, double ty, double* f) {
  auto* m = static_cast<Mesh*>(mesh);
  std::vector<double> fv(f, f + 2 * m->num_nodes());
  const int rc = guarded([&] { add_traction(*m, group, t, tx, ty, fv); });
  if (rc == 0) std::memcpy(f, fv.data(), fv.size() * sizeof(double));
  return rc;
}

// Adds component (0 = ux, 1 = uy) = value on every node of group `group` (bc.cpp:118-135).
// dofs/values receive the sorted DOF map (DirichletDofs::values order); returns its size,
// or -1 on error (unknown group, conflicting values).
int ref_dirichlet_dofs(void* mesh, int n_specs, const char* const* groups, const int* comps,
                       const double* vals, int32_t* dofs_out, double* values_out) {
  auto* m = static_cast<Mesh*>(mesh);
  DirichletDofs d;
  if (guarded([&] {
        for (int s = 0; s < n_specs; ++s) add_dirichlet_group(*m, groups[s], comps[s], vals[s], d);
      }))
    return -1;
  int k = 0;
  for (const auto& [dof, v] : d.values()) {
    if (dofs_out) dofs_out[k] = dof;
    if (values_out) values_out[k] = v;
    ++k;
  }
  return k;
}

int ref_apply_dirichlet(void* Kp, int n_fixed, const int32_t* dofs, const double* values, double* b) {
  auto* K = static_cast<CsrMatrix*>(Kp);
  return guarded([&] {
    DirichletDofs d;
    for (int i = 0; i < n_fixed; ++i) d.add(dofs[i], values[i]);
    std::vector<double> bv(b, b + K->num_rows);
    apply_dirichlet(d, *K, bv);
    std::memcpy(b, bv.data(), bv.size() * sizeof(double));
  });
}

// ---- solver: CgJacobiSolver::setup + solve ------------------------------------------------
struct RefStats {
  int iterations;
  int converged;
  double rel_residual;
  double true_rel_residual;
  double t_setup;
  double t_solve;
  double t_spmv;
  double t_dot;
  double t_vec;
};

// Runs CgJacobiSolver (setup + solve) with SolveBreakdown on. history: max_iter + 1 doubles or
// NULL. msg/warn (256 chars each) receive the stats message and warning.
int ref_pcg(void* Kp, const double* b, double* x, double rtol, int max_iter, double* history,
            RefStats* st, char* msg, char* warn) {
  auto* K = static_cast<CsrMatrix*>(Kp);
  return guarded([&] {
    SolverOptions opt;
    opt.rtol = rtol;
    opt.max_iter = max_iter;
    opt.record_history = history != nullptr;
    CgJacobiSolver solver(opt);
    SolveBreakdown bd;
    bd.clock = steady_seconds;
    solver.set_breakdown(&bd);
    const double t0 = steady_seconds();
    solver.setup(*K);
    const double t1 = steady_seconds();
    std::vector<double> bv(b, b + K->num_rows), xv;
    const SolverStats s = solver.solve(bv, xv);
    const double t2 = steady_seconds();
    std::memcpy(x, xv.data(), xv.size() * sizeof(double));
    if (history)
      std::memcpy(history, s.residual_history.data(), s.residual_history.size() * sizeof(double));
    st->iterations = s.iterations;
    st->converged = s.converged ? 1 : 0;
    st->rel_residual = s.rel_residual;
    st->true_rel_residual = s.true_rel_residual;
    st->t_setup = t1 - t0;
    st->t_solve = t2 - t1;
    st->t_spmv = bd.spmv_local;
    st->t_dot = bd.dot_local;
    st->t_vec = bd.vector_ops;
    if (msg) {
      std::strncpy(msg, s.message.c_str(), 255);
      msg[255] = 0;
    }
    if (warn) {
      std::strncpy(warn, s.warning.c_str(), 255);
      warn[255] = 0;
    }
  });
}

// ---- post-processing ------------------------------------------------------------------------
// Element stresses (postprocess.cpp:35-60): out has 8 arrays of n_tri doubles
// (sxx, syy, txy, von_mises, szz, cx, cy, area).
int ref_element_stresses(void* mesh, const double* u, double E, double nu, int plane_strain,
                         double* out) {
  auto* m = static_cast<Mesh*>(mesh);
  return guarded([&] {
    const PlaneCondition pc = plane_strain ? PlaneCondition::Strain : PlaneCondition::Stress;
    std::vector<double> uv(u, u + 2 * m->num_nodes());
    const ElementStresses s = compute_element_stresses(*m, uv, constitutive_matrix(E, nu, pc), nu, pc);
    const std::size_t ne = m->num_triangles();
    const std::vector<double>* arrs[8] = {&s.sxx, &s.syy, &s.txy, &s.von_mises,
                                          &s.szz, &s.cx,  &s.cy,  &s.area};
    for (int a = 0; a < 8; ++a) std::memcpy(out + a * ne, arrs[a]->data(), ne * sizeof(double));
  });
}

}  // extern "C"
