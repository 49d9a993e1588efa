// C-ABI layer (include/cstfem_b200.h): the context, argument checks, device buffers, error
// reporting with the reference's messages, and the host side of the PCG driver (chunks of
// iterations captured once in a CUDA graph, a host check of the device state between
// chunks).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

using namespace cstg;


extern "C" {

int cstg_version(void) { return 1; }

long long cstg_kernel_launches(void) { return launches_total(); }

void cstg_default_options(cstg_solver_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->rtol = 1e-10;
  o->max_iter = 20000;
  o->precision = CSTG_PRECISION_FP64;
  o->true_residual_stop = 0;
  o->max_refinements = 16;
  o->check_interval = 0;
}

cstg_ctx* cstg_create(int device, int* status) {
  auto set = [&](int s) {
    if (status) *status = s;
  };
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set(CSTG_ERR_CUDA);
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    set(CSTG_ERR_CUDA);
    return nullptr;
  }
  auto* ctx = new cstg_ctx;
  ctx->device = device;
  const char* gather = std::getenv("CSTG_MP_GATHER");
  ctx->lp_plan_on = !(gather && std::strcmp(gather, "rows") == 0);
  bool ok = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&ctx->ev0) == cudaSuccess && cudaEventCreate(&ctx->ev1) == cudaSuccess &&
            cudaMallocHost(&ctx->h_err, sizeof(int) * kErrSlots) == cudaSuccess &&
            cudaMallocHost(&ctx->h_state, sizeof(PcgState)) == cudaSuccess;
  ctx->stream = ctx->own;
  ok = ok && ensure(ctx, ctx->err_word, sizeof(int) * kErrSlots) == 0 &&
       ensure(ctx, ctx->state, sizeof(PcgState)) == 0 &&
       ensure(ctx, ctx->partials, sizeof(double) * 4 * kMaxGrid) == 0 &&
       cudaMemsetAsync(ctx->state.p, 0, sizeof(PcgState), ctx->stream) == cudaSuccess &&
       cudaStreamSynchronize(ctx->stream) == cudaSuccess;
  if (!ok) {
    cstg_destroy(ctx);
    set(CSTG_ERR_CUDA);
    return nullptr;
  }
  set(CSTG_OK);
  return ctx;
}

void cstg_destroy(cstg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  if (ctx->bat_graph) cudaGraphExecDestroy(ctx->bat_graph);
  if (ctx->fcg_graph) cudaGraphExecDestroy(ctx->fcg_graph);
  amg_free(ctx);
  DevBuf* all[] = {&ctx->xy,      &ctx->tri,    &ctx->cnt,      &ctx->cursor,   &ctx->ne_ptr,
                   &ctx->ne,      &ctx->scan_tmp, &ctx->deg,    &ctx->node_ptr, &ctx->bnbr,
                   &ctx->slot,    &ctx->row_ptr, &ctx->cols,    &ctx->vals,     &ctx->fixed,
                   &ctx->ubar,    &ctx->dofs,   &ctx->dvals,    &ctx->b_in,     &ctx->x,
                   &ctx->r,       &ctx->p,      &ctx->Ap,       &ctx->inv_diag, &ctx->partials,
                   &ctx->state,   &ctx->err_word, &ctx->hist,   &ctx->vec_in,   &ctx->vec_out,
                   &ctx->stress,    &ctx->val32,  &ctx->nbr32,    &ctx->S32,      &ctx->mat,
                   &ctx->mat_tab, &ctx->bat_sys, &ctx->bat_order, &ctx->bat_queue, &ctx->bat_b,
                   &ctx->bat_x,   &ctx->bat_r,  &ctx->bat_p,    &ctx->bat_Ap,   &ctx->bat_stats,
                   &ctx->bat_in,  &ctx->bat_out, &ctx->lp_p32, &ctx->lp_pb,   &ctx->lp_pf,
                   &ctx->lp_sf,   &ctx->lp_h0,  &ctx->lp_h1,    &ctx->lp_sc,    &ctx->lp_z,
                   &ctx->tr_con,  &ctx->tr_cnt, &ctx->tr_ptr,   &ctx->tr_cur,   &ctx->tr_rec,
                   &ctx->lm_winvd, &ctx->fcg_ring, &ctx->lp_mat, &ctx->lp_plan_hdr, &ctx->lp_plan_runs,
                   &ctx->lp_plan_local, &ctx->tr_edges, &ctx->tr_f};
  for (DevBuf* b : all) free_buf(*b);
  for (int j = 0; j < kFcgMaxHist; ++j) {
    free_buf(ctx->fcg_ph[j]);
    free_buf(ctx->fcg_qh[j]);
  }
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  if (ctx->h_state) cudaFreeHost(ctx->h_state);
  for (cudaEvent_t e : ctx->bd_ev) cudaEventDestroy(e);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
}

const char* cstg_last_error(const cstg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int cstg_set_stream(cstg_ctx* ctx, void* s) {
  BEGIN(ctx);
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stream = s ? static_cast<cudaStream_t>(s) : ctx->own;
  return CSTG_OK;
}

int cstg_binary_version(int device, int* version) {
  if (!version) return CSTG_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return CSTG_ERR_CUDA;
  return kernel_binary_version(version) == cudaSuccess ? CSTG_OK : CSTG_ERR_CUDA;
}

int cstg_solve_breakdown(cstg_ctx* ctx, cstg_breakdown* out) {
  BEGIN(ctx);
  if (!out) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "solve_breakdown: null output");
  if (!ctx->bd.valid)
    return fail(ctx, CSTG_ERR_STATE, "solve_breakdown: no instrumented solve since the last cstg_pcg_setup");
  *out = ctx->bd;
  return CSTG_OK;
}

int cstg_get_stream(cstg_ctx* ctx, void** stream) {
  BEGIN(ctx);
  if (!stream) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "get_stream: null output");
  *stream = static_cast<void*>(ctx->stream);
  return CSTG_OK;
}

// ---- mesh --------------------------------------------------------------------------------

static int set_mesh_common(cstg_ctx* ctx, int n_nodes, int n_tri) {
  if (n_nodes < 0 || n_tri < 0)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_mesh: negative size (%d nodes, %d triangles)",
                n_nodes, n_tri);
  if ((long long)n_nodes * 2 > INT_MAX - 1)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_mesh: %d nodes exceed the int32 DOF range",
                n_nodes);
  ENSURE(ctx->xy, sizeof(double) * 2 * (size_t)n_nodes);
  ENSURE(ctx->tri, sizeof(int) * 3 * (size_t)n_tri);
  ctx->n_nodes = n_nodes;
  ctx->n_tri = n_tri;
  ctx->has_mesh = true;
  ctx->kind = 0;
  ctx->has_values = ctx->setup_done = false;
  ctx->h_ne_ptr.clear();
  ctx->h_ne.clear();
  return CSTG_OK;
}

int cstg_set_mesh(cstg_ctx* ctx, int n_nodes, const double* xy, int n_tri, const int32_t* tri) {
  BEGIN(ctx);
  if ((n_nodes > 0 && !xy) || (n_tri > 0 && !tri))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_mesh: null array");
  const int rc = set_mesh_common(ctx, n_nodes, n_tri);
  if (rc) return rc;
  // the host copy of the mesh (the host traction path's input) is read back from the device when
  // first needed, not copied here
  ctx->h_xy.clear();
  ctx->h_tri.clear();
  ctx->host_mesh = true;
  if (n_nodes)
    CK(cudaMemcpyAsync(ctx->xy.p, xy, sizeof(double) * 2 * (size_t)n_nodes, cudaMemcpyHostToDevice,
                       ctx->stream));
  if (n_tri)
    CK(cudaMemcpyAsync(ctx->tri.p, tri, sizeof(int) * 3 * (size_t)n_tri, cudaMemcpyHostToDevice,
                       ctx->stream));
  return CSTG_OK;
}

int cstg_set_mesh_device(cstg_ctx* ctx, int n_nodes, const double* d_xy, int n_tri,
                         const int32_t* d_tri) {
  BEGIN(ctx);
  if ((n_nodes > 0 && !d_xy) || (n_tri > 0 && !d_tri))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_mesh_device: null array");
  const int rc = set_mesh_common(ctx, n_nodes, n_tri);
  if (rc) return rc;
  ctx->host_mesh = false;
  ctx->h_xy.clear();
  ctx->h_tri.clear();
  if (n_nodes)
    CK(cudaMemcpyAsync(ctx->xy.p, d_xy, sizeof(double) * 2 * (size_t)n_nodes,
                       cudaMemcpyDeviceToDevice, ctx->stream));
  if (n_tri)
    CK(cudaMemcpyAsync(ctx->tri.p, d_tri, sizeof(int) * 3 * (size_t)n_tri,
                       cudaMemcpyDeviceToDevice, ctx->stream));
  return CSTG_OK;
}

// ---- build_stiffness_pattern ----------------------------------------------------------------

int cstg_build_pattern(cstg_ctx* ctx, int64_t* nnz_out) {
  BEGIN(ctx);
  if (!ctx->has_mesh) return fail(ctx, CSTG_ERR_STATE, "build_pattern: no mesh (call cstg_set_mesh)");
  const int N = ctx->n_nodes, E = ctx->n_tri;
  ENSURE(ctx->cnt, sizeof(int) * (size_t)N);
  ENSURE(ctx->cursor, sizeof(int) * (size_t)N);
  ENSURE(ctx->ne_ptr, sizeof(int) * ((size_t)N + 1));
  ENSURE(ctx->ne, sizeof(int) * 3 * (size_t)E);
  ENSURE(ctx->scan_tmp, sizeof(int) * (size_t)scan_tmp_ints(std::max(N, 1)));
  ENSURE(ctx->deg, sizeof(int) * (size_t)N);
  ENSURE(ctx->node_ptr, sizeof(int) * ((size_t)N + 1));
  MeshDev m;
  m.n_nodes = N;
  m.n_tri = E;
  m.xy = buf_ptr<double>(ctx->xy);
  m.tri = buf_ptr<int>(ctx->tri);
  RESET_ERR();
  int* err = buf_ptr<int>(ctx->err_word);
  CK(launch_incidence(m, buf_ptr<int>(ctx->cnt), buf_ptr<int>(ctx->cursor), buf_ptr<int>(ctx->ne_ptr),
                      buf_ptr<int>(ctx->ne), buf_ptr<int>(ctx->scan_tmp), err, ctx->stream));
  CK(launch_pattern_count(m, buf_ptr<int>(ctx->ne_ptr), buf_ptr<int>(ctx->ne), buf_ptr<int>(ctx->deg),
                          buf_ptr<int>(ctx->node_ptr), buf_ptr<int>(ctx->scan_tmp), err, ctx->stream));
  CK(cudaMemcpyAsync(&ctx->h_err[kErrSlots - 1], buf_ptr<int>(ctx->node_ptr) + N, sizeof(int),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->h_err, ctx->err_word.p, sizeof(int) * (kErrSlots - 1),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_err[kErrMesh] != kErrNone)
    return fail(ctx, CSTG_ERR_MESH, "build_pattern: triangle %d has a node index outside [0, %d)",
                ctx->h_err[kErrMesh], N);
  if (ctx->h_err[kErrNeighbours] != kErrNone)
    return fail(ctx, CSTG_ERR_MESH, "build_pattern: node %d has more than %d neighbours",
                ctx->h_err[kErrNeighbours], kMaxNeighbours - 1);
  const long long nb = (unsigned)ctx->h_err[kErrSlots - 1];
  if (4 * nb > INT_MAX)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "build_pattern: nnz = %lld exceeds the int32 range",
                4 * nb);
  ENSURE(ctx->bnbr, sizeof(int) * (size_t)nb);
  ENSURE(ctx->slot, sizeof(int) * 9 * (size_t)E);
  ENSURE(ctx->row_ptr, sizeof(int) * (2 * (size_t)N + 1));
  ENSURE(ctx->cols, sizeof(int) * 4 * (size_t)nb);
  ENSURE(ctx->vals, sizeof(double) * 4 * (size_t)nb);
  if (N)
    CK(launch_pattern_fill(m, buf_ptr<int>(ctx->ne_ptr), buf_ptr<int>(ctx->ne),
                           buf_ptr<int>(ctx->node_ptr), buf_ptr<int>(ctx->bnbr), buf_ptr<int>(ctx->slot),
                           buf_ptr<int>(ctx->row_ptr), buf_ptr<int>(ctx->cols), ctx->stream));
  else
    CK(cudaMemsetAsync(ctx->row_ptr.p, 0, sizeof(int), ctx->stream));
  ctx->kind = 1;
  ctx->pattern_count++;
  ctx->n_rows = 2 * N;
  ctx->nnz = 4 * nb;
  ctx->has_values = ctx->setup_done = false;
  if (nnz_out) *nnz_out = ctx->nnz;
  return CSTG_OK;
}

// ---- assemble_stiffness ---------------------------------------------------------------------

int cstg_assemble(cstg_ctx* ctx, const double D[9], double thickness) {
  BEGIN(ctx);
  if (!D) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "assemble: null D");
  if (ctx->kind != 1)
    return fail(ctx, CSTG_ERR_STATE, "assemble: no mesh pattern (call cstg_build_pattern)");
  MeshDev m;
  m.n_nodes = ctx->n_nodes;
  m.n_tri = ctx->n_tri;
  m.xy = buf_ptr<double>(ctx->xy);
  m.tri = buf_ptr<int>(ctx->tri);
  Mat3 d;
  std::memcpy(d.v, D, sizeof d.v);
  if (ctx->n_nodes)
    CK(launch_assemble(m, buf_ptr<int>(ctx->ne_ptr), buf_ptr<int>(ctx->ne), buf_ptr<int>(ctx->slot),
                       buf_ptr<int>(ctx->node_ptr), d, thickness, nullptr, nullptr, nullptr,
                       buf_ptr<double>(ctx->vals), ctx->stream));
  ctx->has_values = true;
  ctx->setup_done = false;
  return CSTG_OK;
}

int cstg_assemble_materials(cstg_ctx* ctx, int n_materials, const double* D, const double* thickness,
                            const int32_t* material_of_element) {
  BEGIN(ctx);
  if (n_materials < 1 || !D || !thickness || (ctx->n_tri > 0 && !material_of_element))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "assemble: bad material table");
  if (ctx->kind != 1)
    return fail(ctx, CSTG_ERR_STATE, "assemble: no mesh pattern (call cstg_build_pattern)");
  for (int e = 0; e < ctx->n_tri; ++e)
    if (material_of_element[e] < 0 || material_of_element[e] >= n_materials)
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "assemble: element %d has material %d of %d", e,
                  material_of_element[e], n_materials);
  ENSURE(ctx->mat, sizeof(int) * (size_t)ctx->n_tri);
  ENSURE(ctx->mat_tab, sizeof(double) * 10 * (size_t)n_materials);
  double* tab = buf_ptr<double>(ctx->mat_tab);
  if (ctx->n_tri)
    CK(cudaMemcpyAsync(ctx->mat.p, material_of_element, sizeof(int) * (size_t)ctx->n_tri,
                       cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(tab, D, sizeof(double) * 9 * (size_t)n_materials, cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemcpyAsync(tab + 9 * (size_t)n_materials, thickness, sizeof(double) * (size_t)n_materials,
                     cudaMemcpyHostToDevice, ctx->stream));
  MeshDev m;
  m.n_nodes = ctx->n_nodes;
  m.n_tri = ctx->n_tri;
  m.xy = buf_ptr<double>(ctx->xy);
  m.tri = buf_ptr<int>(ctx->tri);
  Mat3 d{};
  if (ctx->n_nodes)
    CK(launch_assemble(m, buf_ptr<int>(ctx->ne_ptr), buf_ptr<int>(ctx->ne), buf_ptr<int>(ctx->slot),
                       buf_ptr<int>(ctx->node_ptr), d, 0.0, buf_ptr<int>(ctx->mat), tab,
                       tab + 9 * (size_t)n_materials, buf_ptr<double>(ctx->vals), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));  // the host tables may go out of scope
  ctx->has_values = true;
  ctx->setup_done = false;
  return CSTG_OK;
}

// ---- CSR access -------------------------------------------------------------------------------

int cstg_matrix_size(cstg_ctx* ctx, int* n_rows, int64_t* nnz) {
  BEGIN(ctx);
  if (!ctx->kind) return fail(ctx, CSTG_ERR_STATE, "matrix_size: no matrix");
  if (n_rows) *n_rows = ctx->n_rows;
  if (nnz) *nnz = ctx->nnz;
  return CSTG_OK;
}

int cstg_get_csr(cstg_ctx* ctx, int32_t* row_ptr, int32_t* cols, double* vals) {
  BEGIN(ctx);
  if (!ctx->kind) return fail(ctx, CSTG_ERR_STATE, "get_csr: no matrix");
  if (row_ptr)
    CK(cudaMemcpyAsync(row_ptr, ctx->row_ptr.p, sizeof(int) * ((size_t)ctx->n_rows + 1),
                       cudaMemcpyDeviceToHost, ctx->stream));
  if (cols && ctx->nnz)
    CK(cudaMemcpyAsync(cols, ctx->cols.p, sizeof(int) * (size_t)ctx->nnz, cudaMemcpyDeviceToHost,
                       ctx->stream));
  if (vals && ctx->nnz) {
    if (!ctx->has_values) return fail(ctx, CSTG_ERR_STATE, "get_csr: values not assembled");
    CK(cudaMemcpyAsync(vals, ctx->vals.p, sizeof(double) * (size_t)ctx->nnz, cudaMemcpyDeviceToHost,
                       ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

int cstg_set_csr(cstg_ctx* ctx, int n, const int32_t* row_ptr, const int32_t* cols,
                 const double* vals) {
  BEGIN(ctx);
  if (n < 0 || !row_ptr || (n > 0 && (!cols || !vals)))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_csr: bad arguments");
  if (row_ptr[0] != 0) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_csr: row_ptr[0] != 0");
  for (int i = 0; i < n; ++i)
    if (row_ptr[i + 1] < row_ptr[i])
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_csr: row_ptr decreases at row %d", i);
  const long long nnz = row_ptr[n];
  for (long long k = 0; k < nnz; ++k)
    if (cols[k] < 0 || cols[k] >= n)
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "set_csr: column %d out of range at entry %lld",
                  cols[k], k);
  ENSURE(ctx->row_ptr, sizeof(int) * ((size_t)n + 1));
  ENSURE(ctx->cols, sizeof(int) * (size_t)nnz);
  ENSURE(ctx->vals, sizeof(double) * (size_t)nnz);
  CK(cudaMemcpyAsync(ctx->row_ptr.p, row_ptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice,
                     ctx->stream));
  if (nnz) {
    CK(cudaMemcpyAsync(ctx->cols.p, cols, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemcpyAsync(ctx->vals.p, vals, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice,
                       ctx->stream));
  }
  const double avg = n ? (double)nnz / n : 1.0;
  int sub = 1;
  while (sub < 32 && sub < avg) sub <<= 1;
  ctx->csr_sub = sub;
  ctx->kind = 2;
  ctx->n_rows = n;
  ctx->nnz = nnz;
  ctx->has_values = true;
  ctx->setup_done = false;
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

// ---- apply_dirichlet -------------------------------------------------------------------------

static int dirichlet_device(cstg_ctx* ctx, int n_fixed, const int32_t* d_dofs, const double* d_values,
                            int n_rhs, double* d_b) {
  if (!ctx->kind || !ctx->has_values)
    return fail(ctx, CSTG_ERR_STATE, "apply_dirichlet: no assembled matrix");
  if (n_fixed < 0 || n_rhs < 1 || (n_fixed > 0 && (!d_dofs || !d_values)) || (ctx->n_rows > 0 && !d_b))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "apply_dirichlet: bad arguments");
  const int n = ctx->n_rows;
  ENSURE(ctx->fixed, (size_t)n);
  ENSURE(ctx->ubar, sizeof(double) * (size_t)n);
  int* err = buf_ptr<int>(ctx->err_word);
  RESET_ERR();
  CK(launch_dirichlet(n, nullptr, nullptr, nullptr, n_fixed, d_dofs, d_values,
                      buf_ptr<unsigned char>(ctx->fixed), buf_ptr<double>(ctx->ubar), nullptr, 0, err,
                      ctx->stream, false));
  READ_ERR();
  if (ctx->h_err[kErrRange] != kErrNone) {
    int dof = 0;
    CK(cudaMemcpy(&dof, d_dofs + ctx->h_err[kErrRange], sizeof(int), cudaMemcpyDeviceToHost));
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "apply_dirichlet: DOF %d out of range", dof);
  }
  if (ctx->h_err[kErrConflict] != kErrNone) {
    const int dof = ctx->h_err[kErrConflict];
    return fail(ctx, CSTG_ERR_DIRICHLET_CONFLICT,
                "conflicting Dirichlet values for node %d (0-based) component %s", dof / 2,
                dof % 2 == 0 ? "ux" : "uy");
  }
  CK(launch_dirichlet(n, buf_ptr<int>(ctx->row_ptr), buf_ptr<int>(ctx->cols),
                      buf_ptr<double>(ctx->vals), n_fixed, d_dofs, d_values,
                      buf_ptr<unsigned char>(ctx->fixed), buf_ptr<double>(ctx->ubar), d_b, n_rhs, err,
                      ctx->stream, true));
  ctx->setup_done = false;
  READ_ERR();
  if (ctx->h_err[kErrDiag] != kErrNone)
    return fail(ctx, CSTG_ERR_NONPOSITIVE_DIAGONAL,
                "apply_dirichlet: non-positive diagonal at DOF %d", ctx->h_err[kErrDiag]);
  return CSTG_OK;
}

int cstg_apply_dirichlet_device(cstg_ctx* ctx, int n_fixed, const int32_t* d_dofs,
                                const double* d_values, double* d_b) {
  BEGIN(ctx);
  return dirichlet_device(ctx, n_fixed, d_dofs, d_values, 1, d_b);
}

int cstg_apply_dirichlet_multi_device(cstg_ctx* ctx, int n_fixed, const int32_t* d_dofs,
                                      const double* d_values, int n_rhs, double* d_b) {
  BEGIN(ctx);
  return dirichlet_device(ctx, n_fixed, d_dofs, d_values, n_rhs, d_b);
}

static int dirichlet_host(cstg_ctx* ctx, int n_fixed, const int32_t* dofs, const double* values,
                          int n_rhs, double* b) {
  if (!ctx->kind) return fail(ctx, CSTG_ERR_STATE, "apply_dirichlet: no assembled matrix");
  if (n_fixed < 0 || n_rhs < 1 || (n_fixed > 0 && (!dofs || !values)) || (ctx->n_rows > 0 && !b))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "apply_dirichlet: bad arguments");
  const size_t n = (size_t)ctx->n_rows * (size_t)n_rhs;
  ENSURE(ctx->dofs, sizeof(int) * (size_t)n_fixed);
  ENSURE(ctx->dvals, sizeof(double) * (size_t)n_fixed);
  ENSURE(ctx->b_in, sizeof(double) * n);
  if (n_fixed) {
    CK(cudaMemcpyAsync(ctx->dofs.p, dofs, sizeof(int) * (size_t)n_fixed, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemcpyAsync(ctx->dvals.p, values, sizeof(double) * (size_t)n_fixed,
                       cudaMemcpyHostToDevice, ctx->stream));
  }
  if (n) CK(cudaMemcpyAsync(ctx->b_in.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  const int rc = dirichlet_device(ctx, n_fixed, buf_ptr<int>(ctx->dofs), buf_ptr<double>(ctx->dvals),
                                  n_rhs, buf_ptr<double>(ctx->b_in));
  if (rc) {
    if (rc == CSTG_ERR_INVALID_ARGUMENT && ctx->err.find("out of range") != std::string::npos) {
      // report the DOF value from the host array
      for (int q = 0; q < n_fixed; ++q)
        if (dofs[q] < 0 || dofs[q] >= ctx->n_rows)
          return fail(ctx, rc, "apply_dirichlet: DOF %d out of range", dofs[q]);
    }
    return rc;
  }
  if (n) CK(cudaMemcpyAsync(b, ctx->b_in.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

int cstg_apply_dirichlet(cstg_ctx* ctx, int n_fixed, const int32_t* dofs, const double* values,
                         double* b) {
  BEGIN(ctx);
  return dirichlet_host(ctx, n_fixed, dofs, values, 1, b);
}

int cstg_apply_dirichlet_multi(cstg_ctx* ctx, int n_fixed, const int32_t* dofs, const double* values,
                               int n_rhs, double* b) {
  BEGIN(ctx);
  return dirichlet_host(ctx, n_fixed, dofs, values, n_rhs, b);
}

// ---- multiply -----------------------------------------------------------------------------------

int cstg_multiply_device(cstg_ctx* ctx, const double* d_x, double* d_y) {
  BEGIN(ctx);
  if (!ctx->kind || !ctx->has_values) return fail(ctx, CSTG_ERR_STATE, "multiply: no matrix");
  if (ctx->n_rows && (!d_x || !d_y))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "multiply: null vector");
  if (!aligned16(d_x) || !aligned16(d_y))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "multiply: device vectors must be 16-byte aligned");
  return spmv(ctx, d_x, d_y);  // asynchronous: ordered on the context's stream
}

int cstg_multiply(cstg_ctx* ctx, const double* x, double* y) {
  BEGIN(ctx);
  if (!ctx->kind || !ctx->has_values) return fail(ctx, CSTG_ERR_STATE, "multiply: no matrix");
  const size_t n = (size_t)ctx->n_rows;
  if (n && (!x || !y)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "multiply: null vector");
  ENSURE(ctx->vec_in, sizeof(double) * n);
  ENSURE(ctx->vec_out, sizeof(double) * n);
  if (n) CK(cudaMemcpyAsync(ctx->vec_in.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  const int rc = spmv(ctx, buf_ptr<double>(ctx->vec_in), buf_ptr<double>(ctx->vec_out));
  if (rc) return rc;
  if (n) CK(cudaMemcpyAsync(y, ctx->vec_out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

// ---- CgJacobiSolver::setup ----------------------------------------------------------------------

int cstg_pcg_setup(cstg_ctx* ctx) {
  BEGIN(ctx);
  if (!ctx->kind || !ctx->has_values) return fail(ctx, CSTG_ERR_STATE, "pcg_setup: no matrix");
  const int n = ctx->n_rows;
  ENSURE(ctx->inv_diag, sizeof(double) * (size_t)n);
  RESET_ERR();
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (n)
    CK(launch_inv_diag(n, buf_ptr<int>(ctx->row_ptr), buf_ptr<int>(ctx->cols), buf_ptr<double>(ctx->vals),
                       buf_ptr<double>(ctx->inv_diag), buf_ptr<int>(ctx->err_word), ctx->stream));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  READ_ERR();
  {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->bd = cstg_breakdown{};
    ctx->bd.setup = ms * 1e-3;  // the Jacobi setup of the next solves' breakdown
  }
  if (ctx->h_err[kErrDiag] != kErrNone) {
    ctx->setup_done = false;
    return fail(ctx, CSTG_ERR_NONPOSITIVE_DIAGONAL, "cg_jacobi: non-positive diagonal at row %d",
                ctx->h_err[kErrDiag]);
  }
  ctx->setup_done = true;
  ctx->setup_count++;
  ctx->mixed_ready = false;  // the FP32 operator is rebuilt from this matrix on first use
  return CSTG_OK;
}

// ---- CgJacobiSolver::solve / pcg_jacobi ------------------------------------------------------------

static int snapshot(cstg_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->h_state, ctx->state.p, sizeof(PcgState), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

}  // extern "C"

// The FP32 difference-form operator of the current matrix (built once per setup).
int cstg_host::ensure_mixed(cstg_ctx* ctx) {
  const int N = ctx->n_nodes;
  const size_t noff = (size_t)(ctx->nnz / 4) - (size_t)N;
  ENSURE(ctx->val32, sizeof(float4) * noff);
  ENSURE(ctx->nbr32, sizeof(int) * noff);
  ENSURE(ctx->S32, sizeof(double2) * 2 * (size_t)N);
  if (!ctx->mixed_ready) {
    CK(launch_make_mixed(N, buf_ptr<int>(ctx->node_ptr), buf_ptr<int>(ctx->bnbr), buf_ptr<double>(ctx->vals),
                         buf_ptr<float4>(ctx->val32), buf_ptr<int>(ctx->nbr32), buf_ptr<double2>(ctx->S32),
                         ctx->stream));
    ctx->mixed_ready = true;
  }
  return CSTG_OK;
}

MixedMatrix cstg_host::mixed_view(cstg_ctx* ctx) {
  MixedMatrix mm;
  mm.n_nodes = ctx->n_nodes;
  mm.node_ptr = buf_ptr<int>(ctx->node_ptr);
  mm.nbr32 = buf_ptr<int>(ctx->nbr32);
  mm.val32 = buf_ptr<float4>(ctx->val32);
  mm.S64 = buf_ptr<double2>(ctx->S32);
  return mm;
}

extern "C" {

int cstg_multiply_mixed_device(cstg_ctx* ctx, const double* d_x, double* d_y) {
  BEGIN(ctx);
  if (ctx->kind != 1 || !ctx->setup_done)
    return fail(ctx, CSTG_ERR_STATE, "multiply_mixed: needs the mesh pattern and cstg_pcg_setup");
  if (ctx->n_rows && (!d_x || !d_y)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "multiply_mixed: null vector");
  if (!aligned16(d_x) || !aligned16(d_y))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "multiply_mixed: device vectors must be 16-byte aligned");
  const int rc = ensure_mixed(ctx);
  if (rc) return rc;
  CK(launch_spmv_mixed(mixed_view(ctx), d_x, d_y, ctx->stream));
  return CSTG_OK;
}

// Snapshots of the iterate (training data of the learned preconditioner): every `every`
// iterations x is copied to snap[k * n], k < max; the graph path runs with chunks of `every`.
struct Snapshots {
  double* x = nullptr;
  int every = 0, max = 0, count = 0;
};

static int run_solve(cstg_ctx* ctx, const double* d_b, double* d_x, const cstg_solver_options& o,
                     cstg_stats* stats, double* d_hist, bool hist_host, Snapshots* snap = nullptr) {
  const int n = ctx->n_rows;
  ENSURE(ctx->x, sizeof(double) * (size_t)n);
  ENSURE(ctx->r, sizeof(double) * (size_t)n);
  ENSURE(ctx->p, sizeof(double) * (size_t)n);
  ENSURE(ctx->Ap, sizeof(double) * (size_t)n);
  const bool hist = o.record_history != 0;
  if (hist) ENSURE(ctx->hist, sizeof(double) * ((size_t)o.max_iter + 1));

  PcgBuffers w;
  w.n = n;
  w.x = buf_ptr<double>(ctx->x);
  w.r = buf_ptr<double>(ctx->r);
  w.p = buf_ptr<double>(ctx->p);
  w.Ap = buf_ptr<double>(ctx->Ap);
  w.inv_diag = buf_ptr<double>(ctx->inv_diag);
  w.b = d_b;
  w.partials = buf_ptr<double>(ctx->partials);
  w.history = hist ? buf_ptr<double>(ctx->hist) : nullptr;
  w.st = buf_ptr<PcgState>(ctx->state);
  w.err = buf_ptr<int>(ctx->err_word);
  const BlockMatrix bm = block_view(ctx);
  const CsrMatrixDev cm = csr_view(ctx);
  const BlockMatrix* pbm = ctx->kind == 1 ? &bm : nullptr;
  const CsrMatrixDev* pcm = ctx->kind == 1 ? nullptr : &cm;

  // mixed precision: FP32 difference-form operator built once per matrix (after setup)
  const bool mixed = o.precision == CSTG_PRECISION_MIXED;
  MixedBuffers mw;
  MixedMatrix mm;
  if (mixed) {
    const int N = ctx->n_nodes;
    const int rcm = ensure_mixed(ctx);
    if (rcm) return rcm;
    mm = mixed_view(ctx);
    mw.n_nodes = N;
    mw.x = w.x;
    mw.b = d_b;
    mw.inv_diag = w.inv_diag;
    mw.r = w.r;
    mw.p = w.p;
    mw.Ap = w.Ap;
    mw.partials = w.partials;
    mw.history = w.history;
    mw.st = w.st;
  }
  const long long per_iter = mixed ? 4 : 3;

  // Mesh-pattern matrices run as one persistent cooperative kernel per solve (unless the
  // caller asks for the graph path); caller CSR matrices use the graph path.
  const bool instrumented = o.launch_mode == CSTG_LAUNCH_INSTRUMENTED;
  if (instrumented && mixed)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: the instrumented launch mode runs FP64 Jacobi-PCG only");
  const bool persist = ctx->kind == 1 && o.launch_mode != CSTG_LAUNCH_GRAPH && !instrumented && !snap;
  const int chunk = snap ? snap->every : persist ? o.max_iter + 1 : instrumented ? kBdChunk
                                                                  : (o.check_interval > 0 ? o.check_interval : 50);
  // (Re)capture the chunk graph when a buffer, the shape or the method changed. The mixed
  // graph reads b (reliable updates), so it is also tied to the right-hand-side pointer.
  if (!persist && !instrumented && (!ctx->graph || ctx->graph_gen != ctx->generation || ctx->graph_chunk != chunk ||
      ctx->graph_hist != (hist ? 1 : 0) || ctx->graph_kind != ctx->kind || ctx->graph_n != n ||
      ctx->graph_prec != o.precision || ctx->graph_refs != o.max_refinements ||
      (mixed && ctx->graph_b != d_b))) {
    if (ctx->graph) {
      cudaGraphExecDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) {
      if (mixed)
        launch_mixed_iteration(mw, mm, bm, o.max_refinements, ctx->stream);
      else
        launch_pcg_iteration(w, pbm, pcm, ctx->stream);
    }
    CK(cudaStreamEndCapture(ctx->stream, &g));
    count_launches(-per_iter * chunk);  // captured, not run: counted per graph launch below
    const cudaError_t ie = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    ctx->graph_gen = ctx->generation;
    ctx->graph_chunk = chunk;
    ctx->graph_hist = hist ? 1 : 0;
    ctx->graph_kind = ctx->kind;
    ctx->graph_n = n;
    ctx->graph_prec = o.precision;
    ctx->graph_refs = o.max_refinements;
    ctx->graph_b = d_b;
  }

  // instrumented: events around the phases of every iteration (kBdChunk iterations per batch)
  double bd_spmv = 0.0, bd_vec = 0.0;
  if (instrumented && ctx->bd_ev.empty()) {
    ctx->bd_ev.resize(2 * kBdChunk + 1);
    for (cudaEvent_t& e : ctx->bd_ev) CK(cudaEventCreate(&e));
  }
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (mixed)
    CK(launch_mixed_init(mw, o.rtol, o.max_iter, hist, kReliableDelta, ctx->stream));
  else
    CK(launch_pcg_init(w, o.rtol, o.max_iter, hist, ctx->stream));
  long long spmv_calls = 0;
  int rc = snapshot(ctx);
  if (rc) return rc;
  const long long max_chunks = (long long)o.max_iter / chunk + 2 + (long long)o.max_refinements * 4;
  long long chunks = 0;
  bool true_done = false;
  while (ctx->h_state->done != CSTG_SOLVE_ZERO_RHS + 1) {
    while (ctx->h_state->done == 0) {
      if (++chunks > max_chunks)
        return fail(ctx, CSTG_ERR_TIMEOUT, "pcg_solve: the device state did not finish after %lld chunks",
                    chunks);
      const int it0 = ctx->h_state->iter;
      if (persist) {
        CK(launch_pcg_persistent(w, bm, mixed ? &mm : nullptr, o.max_refinements, ctx->barrier_spin, ctx->stream));
      } else if (instrumented) {
        // SpMV (with its fused p'Ap partials), then the vector phase (x, r, p updates with their
        // fused dots), an event after each; the elapsed times are summed after the batch
        CK(cudaEventRecord(ctx->bd_ev[0], ctx->stream));
        for (int k = 0; k < kBdChunk; ++k) {
          CK(launch_spmv_phase(w, pbm, pcm, ctx->stream));
          CK(cudaEventRecord(ctx->bd_ev[2 * k + 1], ctx->stream));
          CK(launch_vector_phase(w, ctx->stream));
          CK(cudaEventRecord(ctx->bd_ev[2 * k + 2], ctx->stream));
        }
        CK(cudaEventSynchronize(ctx->bd_ev[2 * kBdChunk]));
        for (int k = 0; k < kBdChunk; ++k) {
          float a_ms = 0.f, b_ms = 0.f;
          CK(cudaEventElapsedTime(&a_ms, ctx->bd_ev[2 * k], ctx->bd_ev[2 * k + 1]));
          CK(cudaEventElapsedTime(&b_ms, ctx->bd_ev[2 * k + 1], ctx->bd_ev[2 * k + 2]));
          bd_spmv += a_ms * 1e-3;
          bd_vec += b_ms * 1e-3;
        }
      } else {
        CK(cudaGraphLaunch(ctx->graph, ctx->stream));
        count_launches(per_iter * chunk);
        if (snap && snap->count < snap->max && n)
          CK(cudaMemcpyAsync(snap->x + (size_t)snap->count++ * n, w.x, sizeof(double) * (size_t)n,
                             cudaMemcpyDeviceToDevice, ctx->stream));
      }
      rc = snapshot(ctx);
      if (rc) return rc;
      if (ctx->h_state->done == CSTG_SOLVE_TIMEOUT + 1) {
        if (stats) {
          std::memset(stats, 0, sizeof *stats);
          stats->status = CSTG_SOLVE_TIMEOUT;
          stats->iterations = ctx->h_state->iter;
          g_fmt(stats->message, sizeof stats->message, "a grid barrier of the persistent solve timed out");
        }
        return fail(ctx, CSTG_ERR_TIMEOUT, "pcg_solve: a grid barrier of the persistent solve timed out");
      }
      spmv_calls += ctx->h_state->iter - it0 + (ctx->h_state->done == CSTG_SOLVE_BREAKDOWN + 1);
    }
    // true residual (solver.cpp:117-122); with true_residual_stop it may re-open the solve
    if (instrumented) CK(cudaEventRecord(ctx->bd_ev[0], ctx->stream));
    rc = spmv(ctx, w.x, w.Ap);
    if (rc) return rc;
    ++spmv_calls;
    if (instrumented) CK(cudaEventRecord(ctx->bd_ev[1], ctx->stream));
    // (the mixed method confirms convergence on the FP64 true residual itself)
    CK(launch_true_residual(w, !mixed && o.true_residual_stop != 0, o.max_refinements, ctx->stream));
    if (instrumented) {
      CK(cudaEventRecord(ctx->bd_ev[2], ctx->stream));
      CK(cudaEventSynchronize(ctx->bd_ev[2]));
      float a_ms = 0.f, b_ms = 0.f;
      CK(cudaEventElapsedTime(&a_ms, ctx->bd_ev[0], ctx->bd_ev[1]));
      CK(cudaEventElapsedTime(&b_ms, ctx->bd_ev[1], ctx->bd_ev[2]));
      bd_spmv += a_ms * 1e-3;
      bd_vec += b_ms * 1e-3;
    }
    rc = snapshot(ctx);
    if (rc) return rc;
    true_done = true;
    if (ctx->h_state->done != 0) break;
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  if (n) CK(cudaMemcpyAsync(d_x, w.x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
  const PcgState s = *ctx->h_state;
  if (hist && d_hist) {
    const int cnt = s.done == CSTG_SOLVE_ZERO_RHS + 1 ? 1 : s.iter + 1;
    CK(cudaMemcpyAsync(d_hist, w.history, sizeof(double) * (size_t)cnt,
                       hist_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (instrumented) {
    cstg_breakdown& bd = ctx->bd;
    bd.spmv_local = bd_spmv;
    bd.vector_ops = bd_vec;
    bd.dot_local = 0.0;  // fused into the SpMV and vector kernels (counted there)
    bd.total = bd.setup + ms * 1e-3;
    bd.spmv_calls = spmv_calls;
    bd.reductions = 2LL * s.iter + 1;
    bd.valid = 1;
  }

  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->iterations = s.iter;
    stats->status = s.done - 1;
    stats->converged = (s.done == CSTG_SOLVE_CONVERGED + 1 || s.done == CSTG_SOLVE_ZERO_RHS + 1);
    stats->refinements = s.replace_count;
    stats->rel_residual = s.rel;
    stats->true_rel_residual = true_done ? s.true_rel : 0.0;
    stats->solve_seconds = ms * 1e-3;
    stats->spmv_calls = spmv_calls + (o.precision == CSTG_PRECISION_MIXED ? s.replace_count : 0);
    switch (s.done - 1) {
      case CSTG_SOLVE_ZERO_RHS:
        g_fmt(stats->message, sizeof stats->message, "zero right-hand side, x = 0");
        break;
      case CSTG_SOLVE_CONVERGED:
        if (mixed && s.fp64_mode)
          g_fmt(stats->message, sizeof stats->message,
                "converged in %d iterations, relative residual %g (FP64 true residual; %d reliable "
                "updates; FP32 operator to iteration %d, then FP64)",
                s.iter, s.rel, s.replace_count, s.fp64_switch_iter);
        else if (mixed)
          g_fmt(stats->message, sizeof stats->message,
                "converged in %d iterations, relative residual %g (FP64 true residual; %d reliable "
                "updates; FP32 operator throughout)",
                s.iter, s.rel, s.replace_count);
        else
          g_fmt(stats->message, sizeof stats->message, "converged in %d iterations, relative residual %g",
                s.iter, s.rel);
        break;
      case CSTG_SOLVE_BREAKDOWN:
        g_fmt(stats->message, sizeof stats->message,
              "CG breakdown at iteration %d: p'Ap = %g (matrix not SPD?)", s.iter + 1, s.pAp);
        break;
      default:
        g_fmt(stats->message, sizeof stats->message,
              "NOT converged: reached max_iter = %d, relative residual %g (rtol %g)", o.max_iter, s.rel,
              o.rtol);
        break;
    }
    if (stats->converged && s.done != CSTG_SOLVE_ZERO_RHS + 1 && stats->true_rel_residual > 10.0 * o.rtol)
      g_fmt(stats->warning, sizeof stats->warning,
            "WARNING: CG recursive residual converged (%g) but the true residual ||b - Ax|| / ||b|| = %g "
            "exceeds 10 * rtol = %g",
            s.rel, stats->true_rel_residual, 10.0 * o.rtol);
  }
  return CSTG_OK;
}

static int check_solve_args(cstg_ctx* ctx, const cstg_solver_options* opt, cstg_solver_options& o) {
  if (opt)
    o = *opt;
  else
    cstg_default_options(&o);
  if (!ctx->setup_done)
    return fail(ctx, CSTG_ERR_STATE, "cg_jacobi: solve() called before setup()");
  if (!(o.rtol >= 0.0) || o.max_iter < 0 || o.max_refinements < 0 || o.check_interval < 0)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: bad options");
  if (o.precision != CSTG_PRECISION_FP64 && o.precision != CSTG_PRECISION_MIXED)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: precision %d not available", o.precision);
  if (o.precision == CSTG_PRECISION_MIXED && ctx->kind != 1)
    return fail(ctx, CSTG_ERR_UNSUPPORTED,
                "pcg_solve: mixed precision needs the mesh (2x2-block) pattern of cstg_build_pattern");
  if (o.fcg_depth < 0 || o.fcg_depth > kFcgMaxHist + 1)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: fcg_depth %d outside 0..%d", o.fcg_depth,
                kFcgMaxHist + 1);
  if (o.preconditioner != CSTG_PRECOND_JACOBI && o.preconditioner != CSTG_PRECOND_LEARNED &&
      o.preconditioner != CSTG_PRECOND_AMG && o.preconditioner != CSTG_PRECOND_LEARNED_MG)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: unknown preconditioner %d", o.preconditioner);
  if (o.preconditioner == CSTG_PRECOND_AMG) {
    if (ctx->kind != 1)
      return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: the multigrid preconditioner needs the mesh pattern");
    if (o.record_history)
      return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: no residual history with the multigrid preconditioner");
  }
  if (o.preconditioner == CSTG_PRECOND_LEARNED || o.preconditioner == CSTG_PRECOND_LEARNED_MG) {
    if (ctx->kind != 1)
      return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: the learned preconditioner needs the mesh pattern");
    if (!ctx->learned_ready || ctx->learned_setup != ctx->setup_count)
      return fail(ctx, CSTG_ERR_STATE, "pcg_solve: call cstg_learned_setup after cstg_pcg_setup");
    if (o.record_history)
      return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_solve: no residual history with the learned preconditioner");
  }
  return CSTG_OK;
}

int cstg_pcg_solve_device(cstg_ctx* ctx, const double* d_b, double* d_x, const cstg_solver_options* opt,
                          cstg_stats* stats, double* d_history) {
  BEGIN(ctx);
  cstg_solver_options o;
  int rc = check_solve_args(ctx, opt, o);
  if (rc) return rc;
  if (ctx->n_rows && (!d_b || !d_x)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: null vector");
  if (!aligned16(d_b) || !aligned16(d_x))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: device vectors must be 16-byte aligned");
  if (o.preconditioner != CSTG_PRECOND_JACOBI) return run_fcg(ctx, d_b, d_x, o, stats);
  return run_solve(ctx, d_b, d_x, o, stats, d_history, false);
}

int cstg_pcg_iterates_device(cstg_ctx* ctx, const double* d_b, int every, int max_snapshots, double* d_X,
                             int* n_snapshots, const cstg_solver_options* opt, cstg_stats* stats) {
  BEGIN(ctx);
  cstg_solver_options o;
  int rc = check_solve_args(ctx, opt, o);
  if (rc) return rc;
  if (every < 1 || max_snapshots < 0 || (max_snapshots > 0 && !d_X) || (ctx->n_rows && !d_b))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_iterates: bad arguments");
  if (o.precision != CSTG_PRECISION_FP64 || o.preconditioner != CSTG_PRECOND_JACOBI || o.record_history)
    return fail(ctx, CSTG_ERR_UNSUPPORTED, "pcg_iterates: plain FP64 Jacobi-PCG only");
  const size_t n = (size_t)ctx->n_rows;
  ENSURE(ctx->vec_out, sizeof(double) * n);
  Snapshots sn;
  sn.x = d_X;
  sn.every = every;
  sn.max = max_snapshots;
  rc = run_solve(ctx, d_b, buf_ptr<double>(ctx->vec_out), o, stats, nullptr, false, &sn);
  if (n_snapshots) *n_snapshots = sn.count;
  return rc;
}

int cstg_pcg_solve(cstg_ctx* ctx, const double* b, double* x, const cstg_solver_options* opt,
                   cstg_stats* stats, double* history) {
  BEGIN(ctx);
  cstg_solver_options o;
  int rc = check_solve_args(ctx, opt, o);
  if (rc) return rc;
  const size_t n = (size_t)ctx->n_rows;
  if (n && (!b || !x)) return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "pcg_solve: null vector");
  ENSURE(ctx->b_in, sizeof(double) * n);
  ENSURE(ctx->vec_out, sizeof(double) * n);
  if (n) CK(cudaMemcpyAsync(ctx->b_in.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  rc = o.preconditioner != CSTG_PRECOND_JACOBI
           ? run_fcg(ctx, buf_ptr<double>(ctx->b_in), buf_ptr<double>(ctx->vec_out), o, stats)
           : run_solve(ctx, buf_ptr<double>(ctx->b_in), buf_ptr<double>(ctx->vec_out), o, stats, history, true);
  if (rc) return rc;
  if (n) CK(cudaMemcpyAsync(x, ctx->vec_out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

// ---- compute_element_stresses -----------------------------------------------------------------

int cstg_element_stresses(cstg_ctx* ctx, const double* u, double E, double nu, int plane_strain,
                          double* out) {
  BEGIN(ctx);
  if (!ctx->has_mesh) return fail(ctx, CSTG_ERR_STATE, "element_stresses: no mesh");
  if ((ctx->n_nodes && !u) || (ctx->n_tri && !out))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "element_stresses: null array");
  const size_t nd = 2 * (size_t)ctx->n_nodes, ne = (size_t)ctx->n_tri;
  ENSURE(ctx->vec_in, sizeof(double) * nd);
  ENSURE(ctx->stress, sizeof(double) * 8 * ne);
  if (nd) CK(cudaMemcpyAsync(ctx->vec_in.p, u, sizeof(double) * nd, cudaMemcpyHostToDevice, ctx->stream));
  Mat3 D;
  constitutive(E, nu, plane_strain, D.v);
  MeshDev m;
  m.n_nodes = ctx->n_nodes;
  m.n_tri = ctx->n_tri;
  m.xy = buf_ptr<double>(ctx->xy);
  m.tri = buf_ptr<int>(ctx->tri);
  CK(launch_element_stresses(m, buf_ptr<double>(ctx->vec_in), D, nu, plane_strain,
                             buf_ptr<double>(ctx->stress), ctx->stream));
  if (ne)
    CK(cudaMemcpyAsync(out, ctx->stress.p, sizeof(double) * 8 * ne, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return CSTG_OK;
}

// ---- add_traction (host) -------------------------------------------------------------------------

int cstg_add_traction(cstg_ctx* ctx, int n_edges, const int32_t* edges, double thickness, double tx,
                      double ty, double* f) {
  if (!ctx) return CSTG_ERR_INVALID_ARGUMENT;
  ctx->err.clear();
  if (n_edges < 0 || (n_edges > 0 && (!edges || !f)))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: bad arguments");
  if (ctx->kind == 1 && n_edges > 0) {
    BEGIN(ctx);
    // with the pattern built, the device path (the pattern's node incidence, the same bits): the
    // loaded nodes' entries of f go up, the loads are added on the GPU, the entries come back.
    // An edge error is reported by the host path below (the reference's message).
    const int N = ctx->n_nodes;
    std::vector<int32_t> nodes(edges, edges + 2 * (size_t)n_edges);
    for (int q = 0; q < 2 * n_edges; ++q)
      if (nodes[q] < 0 || nodes[q] >= N)
        return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: edge %d has a node out of range", q / 2);
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    const int m = (int)nodes.size();
    std::vector<double> fc(2 * (size_t)m);
    for (int i = 0; i < m; ++i) {
      fc[2 * (size_t)i] = f[2 * (size_t)nodes[i]];
      fc[2 * (size_t)i + 1] = f[2 * (size_t)nodes[i] + 1];
    }
    ENSURE(ctx->tr_edges, sizeof(int32_t) * (2 * (size_t)n_edges + (size_t)m));
    ENSURE(ctx->tr_f, sizeof(double) * (std::max<size_t>((size_t)ctx->n_rows, 1) + 2 * (size_t)m));
    int32_t* d_edges = buf_ptr<int32_t>(ctx->tr_edges);
    int32_t* d_nodes = d_edges + 2 * (size_t)n_edges;
    double* d_f = buf_ptr<double>(ctx->tr_f);
    double* d_fc = d_f + (size_t)ctx->n_rows;
    CK(cudaMemcpyAsync(d_edges, edges, sizeof(int32_t) * 2 * (size_t)n_edges, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_nodes, nodes.data(), sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_fc, fc.data(), sizeof(double) * 2 * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_traction_compact(m, d_nodes, d_fc, d_f, 0, ctx->stream));
    const int rc = cstg_add_traction_device(ctx, n_edges, d_edges, thickness, CSTG_TRACTION_CONSTANT, tx, ty, d_f);
    if (rc == CSTG_OK) {
      CK(launch_traction_compact(m, d_nodes, d_fc, d_f, 1, ctx->stream));
      CK(cudaMemcpyAsync(fc.data(), d_fc, sizeof(double) * 2 * (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      for (int i = 0; i < m; ++i) {
        f[2 * (size_t)nodes[i]] = fc[2 * (size_t)i];
        f[2 * (size_t)nodes[i] + 1] = fc[2 * (size_t)i + 1];
      }
      return CSTG_OK;
    }
    if (rc != CSTG_ERR_MESH || !ctx->host_mesh) return rc;
    ctx->err.clear();
  }
  if (!ctx->host_mesh)
    return fail(ctx, CSTG_ERR_STATE, "add_traction: needs the host mesh of cstg_set_mesh");
  const int N = ctx->n_nodes, E = ctx->n_tri;
  if (ctx->h_xy.size() != 2 * (size_t)N || ctx->h_tri.size() != 3 * (size_t)E) {
    BEGIN(ctx);
    ctx->h_xy.resize(2 * (size_t)N);
    ctx->h_tri.resize(3 * (size_t)E);
    if (N)
      CK(cudaMemcpyAsync(ctx->h_xy.data(), ctx->xy.p, sizeof(double) * 2 * (size_t)N, cudaMemcpyDeviceToHost,
                         ctx->stream));
    if (E)
      CK(cudaMemcpyAsync(ctx->h_tri.data(), ctx->tri.p, sizeof(int32_t) * 3 * (size_t)E, cudaMemcpyDeviceToHost,
                         ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  const int32_t* tri = ctx->h_tri.data();
  const double* xy = ctx->h_xy.data();
  if (ctx->h_ne_ptr.empty()) {  // host node -> triangle incidence, built once per mesh
    ctx->h_ne_ptr.assign((size_t)N + 1, 0);
    for (long i = 0; i < 3L * E; ++i) {
      if (tri[i] < 0 || tri[i] >= N) {
        ctx->h_ne_ptr.clear();
        return fail(ctx, CSTG_ERR_MESH, "add_traction: triangle %ld has a node out of range", i / 3);
      }
      ctx->h_ne_ptr[tri[i] + 1]++;
    }
    for (int v = 0; v < N; ++v) ctx->h_ne_ptr[v + 1] += ctx->h_ne_ptr[v];
    ctx->h_ne.assign((size_t)3 * E, 0);
    std::vector<int> cur(ctx->h_ne_ptr.begin(), ctx->h_ne_ptr.end() - 1);
    for (int e = 0; e < E; ++e)
      for (int c = 0; c < 3; ++c) ctx->h_ne[cur[tri[3 * e + c]]++] = e;
  }
  const double g = 1.0 / std::sqrt(3.0);
  const double xi[2] = {-g, g};
  // every edge is checked before any load is added: on an error f is left as it was
  std::vector<int> opp((size_t)n_edges);
  for (int q = 0; q < n_edges; ++q) {
    const int a = edges[2 * q], b = edges[2 * q + 1];
    if (a < 0 || a >= N || b < 0 || b >= N)
      return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: edge %d has a node out of range", q);
    // triangles holding edge {a, b} as one of their three edges (bc.cpp:198-210)
    int count = 0, c = -1;
    for (int k = ctx->h_ne_ptr[a]; k < ctx->h_ne_ptr[a + 1]; ++k) {
      const int e = ctx->h_ne[k];
      const int32_t* t = tri + 3 * (size_t)e;
      for (int s = 0; s < 3; ++s) {
        const int u = t[s], v = t[(s + 1) % 3];
        if ((u == a && v == b) || (u == b && v == a)) {
          ++count;
          c = t[(s + 2) % 3];
        }
      }
    }
    if (count != 1)
      return fail(ctx, CSTG_ERR_MESH, "traction edge (%d, %d) is adjacent to %d triangles (expected 1)",
                  a, b, count);
    opp[(size_t)q] = c;
  }
  for (int q = 0; q < n_edges; ++q) {
    const int a = edges[2 * q], b = edges[2 * q + 1], c = opp[(size_t)q];
    const double xa = xy[2 * a], ya = xy[2 * a + 1];
    const double xb = xy[2 * b], yb = xy[2 * b + 1];
    const double len = std::hypot(xb - xa, yb - ya);
    double nx = (yb - ya) / len, ny = -(xb - xa) / len;
    if (nx * (xy[2 * c] - xa) + ny * (xy[2 * c + 1] - ya) > 0.0) {
      nx = -nx;
      ny = -ny;
    }
    (void)nx;
    (void)ny;
    for (double s : xi) {
      const double Na = 0.5 * (1.0 - s), Nb = 0.5 * (1.0 + s);
      const double w = thickness * 0.5 * len;
      f[2 * a] += w * Na * tx;
      f[2 * a + 1] += w * Na * ty;
      f[2 * b] += w * Nb * tx;
      f[2 * b + 1] += w * Nb * ty;
    }
  }
  return CSTG_OK;
}

int cstg_add_traction_device(cstg_ctx* ctx, int n_edges, const int32_t* d_edges, double thickness, int kind,
                             double p0, double p1, double* d_f) {
  BEGIN(ctx);
  if (ctx->kind != 1)
    return fail(ctx, CSTG_ERR_STATE, "add_traction: needs the node incidence of cstg_build_pattern");
  if (n_edges < 0 || (n_edges > 0 && (!d_edges || !d_f)))
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: bad arguments");
  if (kind != CSTG_TRACTION_CONSTANT && kind != CSTG_TRACTION_KIRSCH && kind != CSTG_TRACTION_STRESS)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: unknown traction kind %d", kind);
  if (n_edges == 0) return CSTG_OK;
  const int N = ctx->n_nodes;
  ENSURE(ctx->tr_con, sizeof(double) * 8 * (size_t)n_edges);
  ENSURE(ctx->tr_cnt, sizeof(int) * (size_t)N);
  ENSURE(ctx->tr_cur, sizeof(int) * (size_t)N);
  ENSURE(ctx->tr_ptr, sizeof(int) * ((size_t)N + 1));
  ENSURE(ctx->tr_rec, sizeof(int) * 2 * (size_t)n_edges);
  ENSURE(ctx->scan_tmp, sizeof(int) * (size_t)scan_tmp_ints(std::max(N, 1)));
  MeshDev m;
  m.n_nodes = N;
  m.n_tri = ctx->n_tri;
  m.xy = buf_ptr<double>(ctx->xy);
  m.tri = buf_ptr<int>(ctx->tri);
  int* err = buf_ptr<int>(ctx->err_word);
  RESET_ERR();
  CK(launch_traction_edges(n_edges, d_edges, m, buf_ptr<int>(ctx->ne_ptr), buf_ptr<int>(ctx->ne), thickness, kind, p0,
                           p1, buf_ptr<double>(ctx->tr_con), buf_ptr<int>(ctx->tr_cnt), err, ctx->stream));
  READ_ERR();
  if (ctx->h_err[kErrRange] != kErrNone)
    return fail(ctx, CSTG_ERR_INVALID_ARGUMENT, "add_traction: edge %d has a node out of range",
                ctx->h_err[kErrRange]);
  if (ctx->h_err[kErrEdge] != kErrNone) {
    int e2[2] = {0, 0};
    CK(cudaMemcpy(e2, d_edges + 2 * (size_t)ctx->h_err[kErrEdge], sizeof e2, cudaMemcpyDeviceToHost));
    return fail(ctx, CSTG_ERR_MESH, "traction edge (%d, %d) is not adjacent to exactly one triangle", e2[0], e2[1]);
  }
  CK(launch_traction_apply(n_edges, d_edges, N, buf_ptr<double>(ctx->tr_con), buf_ptr<int>(ctx->tr_cnt),
                           buf_ptr<int>(ctx->tr_ptr), buf_ptr<int>(ctx->tr_cur), buf_ptr<int>(ctx->tr_rec),
                           buf_ptr<int>(ctx->scan_tmp), d_f, ctx->stream));
  return CSTG_OK;  // asynchronous on the context's stream
}

}  // extern "C"
