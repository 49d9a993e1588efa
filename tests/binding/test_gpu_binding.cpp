// The reference-side GPU backend (gpu_backend.hpp) compiled against the reference's own headers
// and linked with the reference's serial core (oracle/_ref/libcstfem_ref.so) and this library.
// It runs the reference's PCG test cases (tests/test_pcg.cpp: random SPD systems against
// Cholesky, zero right-hand side, max_iter, the true-residual warning through the LinearOperator
// seam, a non-positive diagonal) through the GPU classes, and the driver flow of
// run_serial_case (src/driver.cpp:164-188) on a Kirsch mesh: the reference's reader, GPU
// assembly, the reference's loads, GPU elimination, the GPU solver, the reference's stresses.
//
// Usage: test_gpu_binding <kirsch mesh .msh>; exit status 0 when every check holds.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>

#include "cstfem/element.hpp"
#include "cstfem/mesh.hpp"
#include "cstfem/postprocess.hpp"
#include "gpu_backend.hpp"

using namespace cstfem;
using cstfem_gpu::CgJacobiGpuSolver;
using cstfem_gpu::GpuOperator;
using cstfem_gpu::GpuStiffness;

namespace {

int g_checks = 0, g_failed = 0;

#define EXPECT(cond)                                                            \
  do {                                                                          \
    ++g_checks;                                                                 \
    if (!(cond)) {                                                              \
      ++g_failed;                                                               \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);             \
    }                                                                           \
  } while (0)

using Dense = std::vector<double>;

CsrMatrix to_csr(const Dense& A, int n) {
  CsrMatrix K;
  K.num_rows = K.num_cols = n;
  K.row_ptr.push_back(0);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j)
      if (A[(size_t)i * n + j] != 0.0) {
        K.cols.push_back(j);
        K.vals.push_back(A[(size_t)i * n + j]);
      }
    K.row_ptr.push_back((int)K.cols.size());
  }
  return K;
}

// A = M'M + n I scaled by D A D with d_i = 10^(3 (u + 1) / 2): SPD with a spread diagonal
Dense spd(int n, std::mt19937& gen) {
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  Dense M((size_t)n * n), A((size_t)n * n, 0.0);
  for (double& v : M) v = u(gen);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += M[(size_t)k * n + i] * M[(size_t)k * n + j];
      A[(size_t)i * n + j] = s + (i == j ? n : 0.0);
    }
  std::vector<double> d(n);
  for (double& v : d) v = std::pow(10.0, 3.0 * (u(gen) + 1.0) / 2.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[(size_t)i * n + j] *= d[i] * d[j];
  return A;
}

// dense Cholesky solve (the check's exact solution)
std::vector<double> chol_solve(Dense A, int n, std::vector<double> b) {
  for (int j = 0; j < n; ++j) {
    for (int k = 0; k < j; ++k) A[(size_t)j * n + j] -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
    A[(size_t)j * n + j] = std::sqrt(A[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i) {
      for (int k = 0; k < j; ++k) A[(size_t)i * n + j] -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
      A[(size_t)i * n + j] /= A[(size_t)j * n + j];
    }
  }
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < i; ++k) b[i] -= A[(size_t)i * n + k] * b[k];
    b[i] /= A[(size_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    for (int k = i + 1; k < n; ++k) b[i] -= A[(size_t)k * n + i] * b[k];
    b[i] /= A[(size_t)i * n + i];
  }
  return b;
}

double max_rel(const std::vector<double>& x, const std::vector<double>& y) {
  double e = 0.0, r = 0.0;
  for (size_t i = 0; i < x.size(); ++i) {
    e = std::max(e, std::abs(x[i] - y[i]));
    r = std::max(r, std::abs(y[i]));
  }
  return r > 0.0 ? e / r : e;
}

void random_spd_systems() {
  std::mt19937 gen(2026);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (int n : {5, 40, 120}) {
    const Dense A = spd(n, gen);
    std::vector<double> b(n);
    for (double& v : b) v = u(gen);
    const auto x_exact = chol_solve(A, n, b);
    const CsrMatrix K = to_csr(A, n);
    CgJacobiGpuSolver gpu({1e-12, 1000, true});
    gpu.setup(K);
    std::vector<double> x;
    const SolverStats st = gpu.solve(b, x);
    CgJacobiSolver cpu({1e-12, 1000, true});
    cpu.setup(K);
    std::vector<double> xc;
    const SolverStats sc = cpu.solve(b, xc);
    std::printf("  n = %3d: GPU %d iterations (CPU %d), rel. residual %.2e, max rel. error vs Cholesky %.2e\n", n,
                st.iterations, sc.iterations, st.rel_residual, max_rel(x, x_exact));
    EXPECT(st.converged);
    EXPECT(st.rel_residual < 1e-12);
    EXPECT(max_rel(x, x_exact) < 1e-9);
    EXPECT(std::abs(st.iterations - sc.iterations) <= 2);
    EXPECT(st.residual_history.size() == (size_t)st.iterations + 1);
    EXPECT(st.residual_history.front() == 1.0 && st.residual_history.back() < 1e-12);
    EXPECT(st.message.find("converged in") == 0);
  }
}

void zero_rhs_and_max_iter() {
  std::mt19937 gen(1);
  const CsrMatrix K = to_csr(spd(6, gen), 6);
  CgJacobiGpuSolver s;
  s.setup(K);
  std::vector<double> x(6, 123.0);
  const SolverStats st = s.solve(std::vector<double>(6, 0.0), x);
  EXPECT(st.converged && st.iterations == 0);
  EXPECT(std::all_of(x.begin(), x.end(), [](double v) { return v == 0.0; }));

  std::mt19937 gen3(3);
  const CsrMatrix K30 = to_csr(spd(30, gen3), 30);
  CgJacobiGpuSolver s2({1e-14, 2, false});
  s2.setup(K30);
  std::vector<double> x2;
  const SolverStats sn = s2.solve(std::vector<double>(30, 1.0), x2);
  std::printf("  max_iter = 2: %s\n", sn.message.c_str());
  EXPECT(!sn.converged && sn.iterations == 2);
  EXPECT(sn.message.find("NOT converged") != std::string::npos);
  EXPECT(!s2.stats().converged);
}

// The reference's pcg_jacobi driving the GPU SpMV through the LinearOperator seam; the operator
// scales its result by 1.01 after `switch_after` applications.
class SwitchingGpuOperator : public LinearOperator {
 public:
  SwitchingGpuOperator(const CsrMatrix& A, int switch_after) : gpu_(A), switch_after_(switch_after) {}
  void apply(const std::vector<double>& x, std::vector<double>& y) const override {
    gpu_.apply(x, y);
    if (++calls_ > switch_after_)
      for (double& v : y) v *= 1.01;
  }
  int calls() const { return calls_; }

 private:
  GpuOperator gpu_;
  int switch_after_;
  mutable int calls_ = 0;
};

void true_residual_warning() {
  std::mt19937 gen(11);
  const int n = 40;
  const CsrMatrix K = to_csr(spd(n, gen), n);
  std::vector<double> b(n, 1.0), inv_diag(n), x;
  for (int i = 0; i < n; ++i) inv_diag[i] = 1.0 / K.diagonal(i);
  const SolverOptions opt{1e-10, 1000, false};
  SwitchingGpuOperator good(K, 1 << 30);
  const SolverStats st = pcg_jacobi(good, inv_diag, SerialReduction(), b, x, opt);
  std::printf("  consistent GPU operator: %d iterations, recursive %.2e, true %.2e\n", st.iterations, st.rel_residual,
              st.true_rel_residual);
  EXPECT(st.converged && st.true_rel_residual < 10 * opt.rtol && st.warning.empty());
  EXPECT(good.calls() == st.iterations + 1);
  // the CPU operator gives the same solve (the GPU rows sum in another order: the same count
  // within two iterations, the same solution within the parity tolerance)
  CsrOperator cpu(K);
  std::vector<double> xc;
  const SolverStats sc = pcg_jacobi(cpu, inv_diag, SerialReduction(), b, xc, opt);
  EXPECT(std::abs(sc.iterations - st.iterations) <= 2 && max_rel(x, xc) < 1e-8);
  SwitchingGpuOperator bad(K, st.iterations);
  const SolverStats sb = pcg_jacobi(bad, inv_diag, SerialReduction(), b, x, opt);
  std::printf("  operator changed for the true residual: %s\n", sb.warning.c_str());
  EXPECT(sb.converged && sb.true_rel_residual > 10 * opt.rtol);
  EXPECT(sb.warning.find("WARNING") != std::string::npos && sb.warning.find("true residual") != std::string::npos);
}

void bad_diagonal() {
  const CsrMatrix K = to_csr({2.0, 1.0, 1.0, -1.0}, 2);
  CgJacobiGpuSolver s;
  bool threw = false;
  try {
    s.setup(K);
  } catch (const std::runtime_error& e) {
    threw = std::string(e.what()).find("non-positive diagonal") != std::string::npos;
  }
  EXPECT(threw);
}

// run_serial_case's flow with the GPU classes on a Kirsch mesh, against the CPU path
void driver_flow(const std::string& msh) {
  const Mesh m = read_gmsh(msh);
  const Mat3 D = constitutive_matrix(210e9, 0.3, PlaneCondition::Stress);
  const double t = 0.01;
  GpuStiffness gk;
  gk.build(m, D, t);
  CsrMatrix Kc = build_stiffness_pattern(m);
  assemble_stiffness(m, D, t, Kc);
  const CsrMatrix Kg = gk.download();
  EXPECT(Kg.row_ptr == Kc.row_ptr && Kg.cols == Kc.cols && Kg.vals == Kc.vals);  // bit for bit
  std::vector<double> f(m.xy.size(), 0.0);
  add_traction(m, "right", t, 100e6, 0.0, f);
  DirichletDofs dofs;
  add_dirichlet(m, parse_dirichlet("left_sym:ux=0 ; bottom_sym:uy=0"), dofs);
  std::vector<double> bg = f, bc = f;
  gk.apply_dirichlet(dofs, bg);
  apply_dirichlet(dofs, Kc, bc);
  EXPECT(bg == bc);
  EXPECT(gk.download().vals == Kc.vals);
  SolveBreakdown bd;
  bd.clock = steady_seconds;
  CgJacobiGpuSolver gs({1e-12, 20000, false}, &gk);
  gs.set_breakdown(&bd);
  gs.setup(Kc);  // (the matrix already lives in gk's context)
  std::vector<double> ug;
  const SolverStats sg = gs.solve(bg, ug);
  CgJacobiSolver cs({1e-12, 20000, false});
  cs.setup(Kc);
  std::vector<double> uc;
  const SolverStats sc = cs.solve(bc, uc);
  std::printf("  kirsch driver flow: GPU %d iterations (CPU %d), max rel. difference %.2e, solve %.4f s\n",
              sg.iterations, sc.iterations, max_rel(ug, uc), bd.total);
  EXPECT(sg.converged && sc.converged);
  EXPECT(std::abs(sg.iterations - sc.iterations) <= std::max(2, sc.iterations / 50));
  EXPECT(max_rel(ug, uc) < 1e-8);
  EXPECT(bd.total > 0.0 && bd.spmv_calls == sg.iterations + 1);
  const ElementStresses es = compute_element_stresses(m, ug, D, 0.3, PlaneCondition::Stress);
  const ElementStresses ec = compute_element_stresses(m, uc, D, 0.3, PlaneCondition::Stress);
  double ds = 0.0, rs = 0.0;
  for (size_t e = 0; e < es.sxx.size(); ++e) {
    ds = std::max(ds, std::abs(es.sxx[e] - ec.sxx[e]));
    rs = std::max(rs, std::abs(ec.sxx[e]));
  }
  EXPECT(ds / rs < 1e-7);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::printf("usage: %s kirsch.msh\n", argv[0]);
    return 2;
  }
  try {
    random_spd_systems();
    zero_rhs_and_max_iter();
    true_residual_warning();
    bad_diagonal();
    driver_flow(argv[1]);
  } catch (const std::exception& e) {
    std::printf("FAILED: exception %s\n", e.what());
    return 1;
  }
  std::printf("%d checks, %d failed\n", g_checks, g_failed);
  return g_failed ? 1 : 0;
}
