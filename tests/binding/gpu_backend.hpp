// The GPU backend a maintainer of the reference would add to its tree: the C ABI of
// include/cstfem_b200.h behind the reference's own interfaces.
//
//   GpuStiffness       build_stiffness_pattern + assemble_stiffness (include/cstfem/assembly.hpp:15,22)
//                      and apply_dirichlet (include/cstfem/bc.hpp:53) on the GPU; download() gives
//                      the reference's CsrMatrix
//   GpuOperator        a cstfem::LinearOperator (include/cstfem/solver.hpp:60-64) whose apply() is the
//                      GPU SpMV, so the reference's pcg_jacobi (solver.hpp:115-118) can drive it
//   CgJacobiGpuSolver  a cstfem::LinearSolver (solver.hpp:120-128): CgJacobiSolver on the GPU, with
//                      the reference's SolverStats and, when a SolveBreakdown is given, the solve
//                      time under its `total` field
//
// Errors of the C ABI become the reference's exceptions: std::logic_error for call order and
// pattern errors, std::runtime_error otherwise (the reference's message text).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "cstfem/assembly.hpp"
#include "cstfem/bc.hpp"
#include "cstfem/solver.hpp"
#include "cstfem_b200.h"

namespace cstfem_gpu {

inline void check(cstg_ctx* c, int rc) {
  if (rc == CSTG_OK) return;
  const std::string msg = c ? cstg_last_error(c) : "cstfem_b200: status " + std::to_string(rc);
  if (rc == CSTG_ERR_STATE || rc == CSTG_ERR_PATTERN) throw std::logic_error(msg);
  throw std::runtime_error(msg);
}

class Context {
 public:
  explicit Context(int device = 0) {
    int st = 0;
    ctx_ = cstg_create(device, &st);
    if (!ctx_) throw std::runtime_error("cstg_create failed with status " + std::to_string(st));
  }
  ~Context() { cstg_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  cstg_ctx* get() const { return ctx_; }

 private:
  cstg_ctx* ctx_ = nullptr;
};

class GpuStiffness {
 public:
  explicit GpuStiffness(int device = 0) : ctx_(device) {}
  void build(const cstfem::Mesh& m, const cstfem::Mat3& D, double t) {
    check(ctx_.get(), cstg_set_mesh(ctx_.get(), (int)(m.xy.size() / 2), m.xy.data(), (int)(m.triangles.size() / 3),
                                    m.triangles.data()));
    check(ctx_.get(), cstg_build_pattern(ctx_.get(), nullptr));
    check(ctx_.get(), cstg_assemble(ctx_.get(), D.data(), t));
  }
  void apply_dirichlet(const cstfem::DirichletDofs& d, std::vector<double>& b) {
    std::vector<int32_t> dofs;
    std::vector<double> vals;
    for (const auto& kv : d.values()) {
      dofs.push_back(kv.first);
      vals.push_back(kv.second);
    }
    check(ctx_.get(), cstg_apply_dirichlet(ctx_.get(), (int)dofs.size(), dofs.data(), vals.data(), b.data()));
  }
  cstfem::CsrMatrix download() const {
    int n = 0;
    int64_t nnz = 0;
    check(ctx_.get(), cstg_matrix_size(ctx_.get(), &n, &nnz));
    cstfem::CsrMatrix K;
    K.num_rows = K.num_cols = n;
    K.row_ptr.resize((size_t)n + 1);
    K.cols.resize((size_t)nnz);
    K.vals.resize((size_t)nnz);
    check(ctx_.get(), cstg_get_csr(ctx_.get(), K.row_ptr.data(), K.cols.data(), K.vals.data()));
    return K;
  }
  cstg_ctx* ctx() const { return ctx_.get(); }

 private:
  Context ctx_;
};

// y = A x on the GPU for any CsrMatrix (uploaded once) or the matrix of a GpuStiffness.
class GpuOperator : public cstfem::LinearOperator {
 public:
  explicit GpuOperator(const cstfem::CsrMatrix& A, int device = 0) : own_(new Context(device)) {
    check(own_->get(), cstg_set_csr(own_->get(), A.num_rows, A.row_ptr.data(), A.cols.data(), A.vals.data()));
  }
  explicit GpuOperator(const GpuStiffness& K) : ext_(K.ctx()) {}
  ~GpuOperator() override { delete own_; }
  void apply(const std::vector<double>& x, std::vector<double>& y) const override {
    y.resize(x.size());
    check(ctx(), cstg_multiply(ctx(), x.data(), y.data()));
  }

 private:
  cstg_ctx* ctx() const { return own_ ? own_->get() : ext_; }
  Context* own_ = nullptr;
  cstg_ctx* ext_ = nullptr;
};

class CgJacobiGpuSolver : public cstfem::LinearSolver {
 public:
  explicit CgJacobiGpuSolver(cstfem::SolverOptions o = {}, GpuStiffness* on_device = nullptr)
      : o_(o), dev_(on_device) {
    if (!dev_) own_ = new Context(0);
  }
  ~CgJacobiGpuSolver() override { delete own_; }
  void set_breakdown(cstfem::SolveBreakdown* bd) { bd_ = bd; }
  void setup(const cstfem::CsrMatrix& A) override {
    cstg_ctx* c = ctx();
    if (own_) check(c, cstg_set_csr(c, A.num_rows, A.row_ptr.data(), A.cols.data(), A.vals.data()));
    check(c, cstg_pcg_setup(c));  // throws on a non-positive diagonal, like CgJacobiSolver::setup
  }
  cstfem::SolverStats solve(const std::vector<double>& b, std::vector<double>& x) override {
    cstg_solver_options opt;
    cstg_default_options(&opt);
    opt.rtol = o_.rtol;
    opt.max_iter = o_.max_iter;
    opt.record_history = o_.record_history ? 1 : 0;
    std::vector<double> hist(o_.record_history ? (size_t)o_.max_iter + 1 : 0);
    cstg_stats s{};
    x.resize(b.size());
    const double t0 = bd_ && bd_->clock ? bd_->clock() : 0.0;
    check(ctx(), cstg_pcg_solve(ctx(), b.data(), x.data(), &opt, &s, o_.record_history ? hist.data() : nullptr));
    if (bd_ && bd_->clock) {
      bd_->total += bd_->clock() - t0;
      bd_->spmv_calls += s.spmv_calls;
    }
    stats_ = cstfem::SolverStats{};
    stats_.iterations = s.iterations;
    stats_.rel_residual = s.rel_residual;
    stats_.true_rel_residual = s.true_rel_residual;
    stats_.converged = s.converged != 0;
    stats_.message = s.message;
    stats_.warning = s.warning;
    if (o_.record_history) {
      const size_t cnt = s.status == CSTG_SOLVE_ZERO_RHS ? 1 : (size_t)s.iterations + 1;
      stats_.residual_history.assign(hist.begin(), hist.begin() + (long)cnt);
    }
    return stats_;
  }
  const cstfem::SolverStats& stats() const override { return stats_; }

 private:
  cstg_ctx* ctx() const { return dev_ ? dev_->ctx() : own_->get(); }
  cstfem::SolverOptions o_;
  GpuStiffness* dev_ = nullptr;
  Context* own_ = nullptr;
  cstfem::SolveBreakdown* bd_ = nullptr;
  cstfem::SolverStats stats_;
};

}  // namespace cstfem_gpu
