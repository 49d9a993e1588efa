// Internal launcher declarations shared by the C-ABI layer and the kernel files.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cstg {

// Slots of the device error word (each holds the smallest offending index, INT_MAX if none).
enum ErrSlot {
  kErrMesh = 0,        // triangle with a node index out of range
  kErrNeighbours = 1,  // node whose neighbourhood exceeds kMaxNeighbours
  kErrRange = 2,       // Dirichlet entry with a DOF out of range
  kErrConflict = 3,    // Dirichlet DOF given two different values
  kErrDiag = 4,        // non-positive diagonal (Dirichlet row or Jacobi setup)
  kErrTimeout = 5,     // bounded device wait gave up
  kErrBatch = 6,       // batched solve: a node coupled to a node of another plate
  kErrEdge = 7,        // traction edge not adjacent to exactly one triangle
  kErrAmg = 8,         // multigrid setup: a row or an aggregate exceeded its bound
  kErrSlots = 12
};

struct Mat3 {  // 3x3 row-major constitutive matrix, passed by value to kernels
  double v[9];
};

struct MeshDev {
  int n_nodes = 0, n_tri = 0;
  const double* xy = nullptr;
  const int* tri = nullptr;
};

// Matrix views for the SpMV paths.
struct BlockMatrix {  // 2x2 node-block CSR (mesh pattern)
  int n_nodes = 0;
  const int* node_ptr = nullptr;
  const int* bnbr = nullptr;
  const double* vals = nullptr;  // reference CSR order (node n's 2 rows contiguous)
  const float* vals32 = nullptr; // same layout, FP32 (mixed precision)
};

struct CsrMatrixDev {  // generic scalar CSR (caller-supplied matrix)
  int n_rows = 0;
  const int* row_ptr = nullptr;
  const int* cols = nullptr;
  const double* vals = nullptr;
  const float* vals32 = nullptr;
  int sub = 8;  // lanes per row
};

// Solver state in device memory (scalars of the CG recurrence). 128-byte aligned.
// Mixed precision: forced replacements count towards the FP32 accuracy floor only once the true
// residual has fallen below this fraction of ||b|| (before that the CG residual may still rise).
constexpr double kStallGate = 1e-2;
// ... and a forced replacement whose true residual exceeds this multiple of the recursive one it
// replaces shows the FP32 recursion moving on without the true residual.
constexpr double kGapRatio = 1.5;

struct alignas(128) PcgState {
  double rz;       // r'z of the current iterate
  double alpha, beta;
  double bnorm;    // ||b||
  double rel;      // recursive ||r|| / ||b||
  double pAp;
  double true_rel; // ||b - A x|| / ||b||
  double rtol;
  double rr;       // r'r of the current iterate
  double rmax;     // largest recursive residual norm since the last reliable update (mixed)
  double rz_prev;  // r'z before the last update (mixed: beta after a reliable update)
  double delta;    // reliable-update threshold (mixed)
  int iter;        // completed CG iterations
  int done;        // 0 running, else CSTG_SOLVE_* + 1
  int max_iter;
  int hist_on;
  int restart_pending;  // mixed: 1 reliable update due, 2 confirm convergence in FP64
  int replace_count;    // residual replacements performed
  int final_checks;     // mixed: FP64 confirmations that failed
  int last_replace;     // mixed: iteration of the last reliable update
  int cycle_limit;      // mixed: force a reliable update after this many iterations
  int fp64_mode;        // mixed: the FP32 operator reached its accuracy floor; SpMV in FP64
  int fp64_switch_iter; // mixed: iteration of that switch (0: none)
  int stall_cycles;     // mixed: forced replacements in a row that found no progress of the true residual
  double best_true;     // mixed: smallest FP64 true residual seen at a reliable update
  double fb_rr0;        // learned (flexible CG): r'r at the start of the stagnation window
  int fallback;         // learned: the network is off, Jacobi-PCG from here on
  int use_jacobi;       // learned: this iteration's z is D^-1 r (fallback or a non-descent z)
  int mp_skip;          // learned: the network kernels skip (done or fallback)
  int fb_it0;           // learned: iteration at the start of the stagnation window
  unsigned int bar_count;  // persistent kernel: blocks arrived at the current grid barrier
  unsigned int bar_gen;    // persistent kernel: barrier generation (bumped on release)
  int bar_err;             // persistent kernel: a barrier wait ran out (the solve is abandoned)
  unsigned int ticket[8];  // last-block tickets, one per kernel kind
  int reliable_due;        // flexible CG, mixed: the recursive residual fell by the reliable-update factor
};
static_assert(sizeof(PcgState) <= 256, "PcgState must fit its 256-byte slot");

// Mixed-precision operator: FP32 off-diagonal 2x2 blocks + FP32 row-block sums (difference
// form, see mixed_kernels.cu). Node n's off-diagonal blocks start at node_ptr[n] - n.
struct MixedMatrix {
  int n_nodes = 0;
  const int* node_ptr = nullptr;
  const int* nbr32 = nullptr;
  const float4* val32 = nullptr;
  const double2* S64 = nullptr;  // row-block sums in FP64: [2n] = (s00, s01), [2n+1] = (s10, s11)
};

struct MixedBuffers {
  int n_nodes = 0;
  double* x = nullptr;            // FP64 vectors (see mixed_kernels.cu for why)
  const double* b = nullptr;
  const double* inv_diag = nullptr;
  double* r = nullptr;
  double* p = nullptr;
  double* Ap = nullptr;
  double* partials = nullptr;
  double* history = nullptr;
  PcgState* st = nullptr;
};

// mixed_kernels.cu
cudaError_t launch_make_mixed(int N, const int* node_ptr, const int* bnbr, const double* vals,
                              float4* val32, int* nbr32, double2* S64, cudaStream_t s);
cudaError_t launch_mixed_init(const MixedBuffers& w, double rtol, int max_iter, bool hist, double delta,
                              cudaStream_t s);
// One iteration: FP32 SpMV + p'Ap, update + reliable-update decision, the (usually idle)
// FP64 replacement, p update.
cudaError_t launch_mixed_iteration(const MixedBuffers& w, const MixedMatrix& A32, const BlockMatrix& A64,
                                   int max_final_checks, cudaStream_t s);
cudaError_t launch_spmv_mixed(const MixedMatrix& A32, const double* x, double* y, cudaStream_t s);

// batch.cu: one result per (plate, load case); the layout of cstg_batch_result.
struct BatchResultDev {
  int iterations, status, refinements, fp64;
  double rel, true_rel;
};

struct BatchArgs {
  int n_sys = 0;
  const int* sys_node = nullptr;  // [n_sys + 1] first node of each plate
  const int* order = nullptr;     // [n_sys] plates, largest first (the work queue's order)
  int* queue = nullptr;           // work counter, zero at launch
  MixedMatrix A32;                // FP32 difference-form operator (unused when start_fp64)
  BlockMatrix A64;                // FP64 operator (true residuals, FP64 mode)
  int start_fp64 = 0;
  const double* inv_diag = nullptr;
  const double* b = nullptr;      // [N][R][2]
  double *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
  double rtol = 1e-10;
  int max_iter = 0, max_refine = 0;
  BatchResultDev* res = nullptr;
  int res_stride = 0, res_offset = 0;  // result index = plate * res_stride + res_offset + q
};
cudaError_t batch_max_clusters(int R, int cluster, int threads, int* n);
cudaError_t launch_batch_pcg(const BatchArgs& a, int R, int cluster, int threads, int n_clusters,
                             cudaStream_t s);
cudaError_t launch_batch_pack(int N, int R, int q0, long long ld, const double* src, double* dst,
                              cudaStream_t s);
cudaError_t launch_batch_unpack(int N, int R, int q0, long long ld, const double* src, double* dst,
                                cudaStream_t s);
cudaError_t launch_batch_check(int N, int n_sys, const int* sys_node, const int* node_ptr, const int* bnbr,
                               int* err, cudaStream_t s);

// mpnn.cu: the learned preconditioner's network (F = 64 features, 3 message-passing layers).
// Packed parameter vector: W_in[64][8], b_in[64], (W_l[64][128], b_l[64]) x 3, W_out[2][64], b_out[2].
constexpr int kMpF = 64, kMpIn = 8, kMpL = 3, kMpTile = 128;  // features, inputs, layers, nodes per tile
constexpr int kMpOffWin = 0, kMpOffBin = kMpF * kMpIn, kMpOffL0 = kMpOffBin + kMpF;
constexpr int kMpLStride = kMpF * 2 * kMpF + kMpF;
constexpr int kMpOffWout = kMpOffL0 + kMpL * kMpLStride, kMpOffBout = kMpOffWout + 2 * kMpF;
constexpr int kMpParams = kMpOffBout + 2;
constexpr int kMpPartBlocks = 148;  // blocks of the weight-gradient kernels (partials, fixed order)
constexpr int kMpPartStride = kMpF * 2 * kMpF + kMpF;

struct MpnnParams {  // device copies of the packed parameters
  const __nv_bfloat16* pb = nullptr;  // BF16 (weights are read from here)
  const float* pf = nullptr;          // FP32 (biases are read from here)
};

// Per-tile gather plan of the message-passing layers (built on the GPU from the pattern, once
// per matrix): for each tile of 128 consecutive nodes, the rows its nodes read (their own and
// their neighbours') as at most kPlanMaxRuns runs of consecutive nodes holding at most
// kPlanMaxUnion rows, and per node its degree (neighbours without itself) and the positions of
// its neighbours' rows (ascending pattern order) in that union; an unused position holds
// kPlanNone, the row after the union (which the layers keep at -0.0, so a padded sum needs no
// branch). A tile that does not fit is marked and its neighbours are gathered from global memory
// instead.
constexpr int kPlanMaxRuns = 8, kPlanMaxUnion = 400, kPlanMaxLocal = 7, kPlanSpan = 4096;
constexpr int kPlanNone = kPlanMaxUnion;
struct MpTilePlan {
  const int4* hdr = nullptr;    // [tiles]: (runs, union rows, fallback, 0)
  const int2* runs = nullptr;   // [tiles][kPlanMaxRuns]: (first node, rows)
  const uint4* local = nullptr; // [nodes]: 8 uint16: [0] degree, [1..deg] neighbours, kPlanNone unused
};
struct MpnnGraph {  // the node-block pattern (self included; the network skips self)
  int n_nodes = 0;
  const int* node_ptr = nullptr;
  const int* nbr = nullptr;
  MpTilePlan plan;  // optional (hdr null: every tile gathers row by row)
};
cudaError_t launch_mp_tile_plan(int N, const int* node_ptr, const int* nbr, int4* hdr, int2* runs, uint4* local,
                                cudaStream_t s);

struct MpnnWork {  // activations (training keeps every layer; inference ping-pongs H[0]/H[1])
  __nv_bfloat16* H[kMpL + 1] = {};
  __nv_bfloat16* G[kMpL] = {};
  __nv_bfloat16* A[kMpL] = {};
  __nv_bfloat16* X = nullptr;  // [N][8]
  float* Y = nullptr;          // [N][2]
  float* dY = nullptr;         // [2N]
  float *dH = nullptr, *dH2 = nullptr, *dU = nullptr, *dAs = nullptr;  // [N][64]
  float* part = nullptr;       // [kMpPartBlocks][kMpPartStride]
};

struct MpScratch {  // small device scalars of the network's reductions
  double dsum;      // sum of the matrix diagonal (the static inputs' scale)
  double rr;        // r'r
  double dots[3];   // z'r, z'Az, e'r
  double loss;
  unsigned int ticket[4];
  double partials[3 * 296];
};

constexpr long long kMpMbarSpinDefault = 1LL << 22;  // polls of the tensor-core wait before it gives up
cudaError_t mpnn_prepare_device();
cudaError_t launch_mp_params(const float* p32, __nv_bfloat16* pb, float* pf, cudaStream_t s);
cudaError_t launch_mp_rr(int n, const double* r, MpScratch* sc, cudaStream_t s, const int* skip = nullptr);
// The network's static inputs per node (6 floats): diagonal / its mean (2), xy / coord_scale (2),
// the caller's two material values (mat, 2 floats per node, device).
cudaError_t launch_mp_static(int N, const double* invd, const double* xy, const float* mat, double coord_scale,
                             MpScratch* sc, float* sf, cudaStream_t s);
// out = factor / lambda (lambda: one device double) * invd
cudaError_t launch_mp_smoother_weights(int n, const double* invd, const double* lam, double factor, double* out,
                                       cudaStream_t s);
// z = zbase + M(r): encoder, three tensor-core layers (the last with the decoder). `rr` points at
// r'r (device), `skip` (device int, may be null) turns the network off (z = zbase + D^-1 r),
// zbase may be null (z = M(r)) or z itself. spin_limit: polls of the tensor-core wait before it
// reports a timeout (kMpMbarSpinDefault normally).
cudaError_t launch_mp_forward(const MpnnGraph& g, const MpnnParams& P, const double* r, const double* invd,
                              const double* rr, const float* sf, const int* skip, MpnnWork& w, bool train,
                              const double* zbase, double* z, long long spin_limit, int* err, cudaStream_t s);
// One stage of the inference forward pass alone (timing): 0 the encoder, 1..kMpL the layers (the
// last with the decoder), on the inference ping-pong buffers of w.
cudaError_t launch_mp_stage(const MpnnGraph& g, const MpnnParams& P, int stage, const double* r, const double* invd,
                            const double* rr, const float* sf, MpnnWork& w, double* z, long long spin_limit, int* err,
                            cudaStream_t s);
cudaError_t launch_mp_loss(int N, const double* z, const double* az, const double* r, const double* e,
                           const double* invd, MpScratch* sc, MpnnWork& w, cudaStream_t s);
// The backward pass; the layers' weight gradients run on the tensor cores (spin_limit / err: the
// bounded wait of their matrix multiplies, as in launch_mp_forward).
cudaError_t launch_mp_backward(const MpnnGraph& g, const MpnnParams& P, MpnnWork& w, float* grad, long long spin_limit,
                               int* err, cudaStream_t s);
cudaError_t launch_mp_adam(float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
                           int step, float scale, __nv_bfloat16* pb, float* pf, cudaStream_t s);

// fcg.cu: flexible CG with the learned preconditioner (Polak-Ribiere beta), Jacobi fallback.
// Truncated flexible CG: besides the current direction p (and q = A p), up to kFcgMaxHist earlier
// directions and their products sit in a ring, and each new direction is A-orthogonalised
// against all of them (depth = ring size + 1; depth 1 is the one-term flexible CG).
constexpr int kFcgMaxHist = 4;
struct FcgRing {
  double pq[kFcgMaxHist];         // p_j'q_j of the ring's directions
  double beta[kFcgMaxHist + 1];   // this step's coefficients: [0] current p, [1 + j] ring slot j
  int count;                      // directions in the ring
  int head;                       // slot the current p is pushed into (the oldest when full)
  int push;                       // 1: this step pushes the current p / q into slot `head` (before it moves)
  int push_slot;
};
struct FcgBuffers {
  int n = 0;  // rows (2 x nodes)
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr;
  const double* b = nullptr;
  const double* inv_diag = nullptr;
  double* partials = nullptr;
  PcgState* st = nullptr;
  int hist = 0;                   // ring size (0: one-term flexible CG)
  double* ph[kFcgMaxHist] = {};   // ring of earlier directions
  double* qh[kFcgMaxHist] = {};   // and of their A-products
  FcgRing* ring = nullptr;
};
cudaError_t launch_fcg_init(const FcgBuffers& w, double rtol, int max_iter, int window, cudaStream_t s);
cudaError_t launch_fcg_dots(const FcgBuffers& w, cudaStream_t s);  // beta, r'z; then p = z + beta p
cudaError_t launch_fcg_update(const FcgBuffers& w, int window, double ratio2, cudaStream_t s,
                              double reliable_delta = 0.0);
// Reliable update of the flexible CG (mixed precision): when k_fcg_update found the recursive
// residual below reliable_delta times its largest value since the last update, r = b - A x with
// the FP64 matrix (p, z and the ring are kept: no restart); a no-op otherwise.
cudaError_t launch_fcg_reliable(const FcgBuffers& w, const BlockMatrix& A, cudaStream_t s);
cudaError_t launch_fcg_pupdate(const FcgBuffers& w, cudaStream_t s);  // p = z + beta p alone
// the truncated variant (w.hist ring directions; 0 falls back to launch_fcg_dots): the betas against
// the current and the stored directions, then the new p (the ring state must start cleared)
cudaError_t launch_fcg_dots_ring(const FcgBuffers& w, cudaStream_t s);
// q = A p with p'Ap and alpha = r'z / p'Ap (the PCG variants of the SpMVs)
cudaError_t launch_spmv_pcg(const BlockMatrix& A, const double* p, double* q, double* partials, PcgState* st,
                            cudaStream_t s);
cudaError_t launch_spmv_mixed_pcg(const MixedMatrix& A32, const BlockMatrix& A64, const double* p, double* q,
                                  double* partials, PcgState* st, cudaStream_t s);

// traction.cu: add_traction on the GPU (con: 8 doubles per edge; cnt/cur: n_nodes ints;
// ptr: n_nodes + 1 ints; rec: 2 n_edges ints)
cudaError_t launch_traction_edges(int n_edges, const int* edges, const MeshDev& m, const int* ne_ptr, const int* ne,
                                  double thickness, int kind, double p0, double p1, double* con, int* cnt, int* err,
                                  cudaStream_t s);
cudaError_t launch_traction_compact(int m, const int* nodes, double* fc, double* f, int dir, cudaStream_t s);
cudaError_t launch_traction_apply(int n_edges, const int* edges, int n_nodes, const double* con, const int* cnt,
                                  int* ptr, int* cur, int* rec, int* scan_tmp, double* f, cudaStream_t s);

// amg.cu: smoothed-aggregation multigrid (block-sparse rows; B = 2 on the finest level, 3 below)
constexpr int kAmgMaxRow = 64;  // distinct block columns of a P, AP or coarse row
constexpr int kAmgMaxAgg = 64;  // nodes of an aggregate
struct AmgBsr {  // n block rows, ptr[n + 1], col[ptr[n]], val: B x B (or B x 3 for P) row-major blocks
  int n = 0;
  const int* ptr = nullptr;
  const int* col = nullptr;
  const double* val = nullptr;
};
struct AmgBsr32 {  // a coarse operator's FP32 copy (3 x 3 blocks), same pattern, entry-major values
  int n = 0;
  int nnzb = 0;  // blocks: entry e of block k at val[e * nnzb + k]
  const int* ptr = nullptr;
  const int* col = nullptr;
  const float* val = nullptr;
};
cudaError_t amg_fine_bsr(int N, const int* node_ptr, const double* vals, double* out, cudaStream_t s);
cudaError_t amg_dinv(int B, const AmgBsr& A, double* dinv, int* err, cudaStream_t s);
// strong[k] = block k of A is a strong connection (aggregation graph); dn: scratch of A.n doubles
cudaError_t amg_strength(int B, const AmgBsr& A, double theta, double* dn, unsigned char* strong, cudaStream_t s);
// strong == nullptr: every block of the pattern is a connection
cudaError_t amg_mis_round(const AmgBsr& A, const unsigned char* strong, int* state, unsigned long long* m1,
                          int* newroot, int* near, int* undecided, cudaStream_t s);
cudaError_t amg_flag_eq(int n, const int* a, int v, int* f, cudaStream_t s);
cudaError_t amg_aggregate(int B, const AmgBsr& A, const unsigned char* strong, const int* state, const int* root_id,
                          int* agg1, int* agg2, cudaStream_t s);
cudaError_t amg_flag_negative(int n, const int* a, int* f, cudaStream_t s);
cudaError_t amg_phase3(int n, int n_agg, const int* left_id, int* agg, cudaStream_t s);
cudaError_t amg_group(int n, const int* key, int m, int* ptr, int* cnt, int* cur, int* out, int* scan_tmp,
                      cudaStream_t s);
cudaError_t amg_tentative(int B, int n_agg, const int* agg_ptr, const int* members, const double* Bf, double* P0,
                          double* Bc, int* err, cudaStream_t s);
// lambda_max(D^-1 A) by `iters` power-iteration steps on the cycle's FP32 operators: the finest
// level's difference form (fine) or a coarse level's entry-major copy (coarse); exactly one of
// the two is given
cudaError_t amg_lambda_f32(const MixedMatrix* fine, const AmgBsr32* coarse, const double* dinv, double* x, double* y,
                           double* part, double* lam, int iters, cudaStream_t s);
size_t amg_lambda_scratch();  // bytes of `part` that amg_lambda needs
cudaError_t amg_p_count(int B, const AmgBsr& A, const int* agg, int* cnt, int* err, cudaStream_t s);
cudaError_t amg_p_fill(int B, const AmgBsr& A, const int* agg, const double* P0, const double* dinv, const double* lam,
                       const AmgBsr& P, cudaStream_t s);
cudaError_t amg_ap_count(int B, const AmgBsr& A, const AmgBsr& P, int* cnt, int* err, cudaStream_t s);
cudaError_t amg_ap_fill(int B, const AmgBsr& A, const AmgBsr& P, const AmgBsr& AP, cudaStream_t s);
cudaError_t amg_pt(int n, int nc, const AmgBsr& P, int* p_row, int* pt_ptr, int* cnt, int* cur, int* pt_tmp,
                   int* pt_idx, int* scan_tmp, cudaStream_t s);
cudaError_t amg_ac_count(int B, int nc, const int* pt_ptr, const int* pt_idx, const int* p_row, const AmgBsr& AP,
                         int* cnt, int* err, cudaStream_t s);
cudaError_t amg_ac_fill(int B, int nc, const int* pt_ptr, const int* pt_idx, const int* p_row, const AmgBsr& P,
                        const AmgBsr& AP, const AmgBsr& Ac, cudaStream_t s);
cudaError_t amg_coarsest(int B, const AmgBsr& A, double* M, double* piv, cudaStream_t s);
// smoother steps (amg.cu): x + gamma D^-1 (b - A x); b - A x; the two steps from x = 0 in one
// launch (x not read); the second Chebyshev step (reads the previous iterate xp). cheb: Chebyshev
// coefficients (else damped Jacobi), computed in the kernel from lambda_max.
constexpr int kSweepSmooth = 0, kSweepResidual = 1, kSweepFirst = 2, kSweepSecond = 3;
void amg_prepare_launch_shapes();  // occupancy queries of the one-wave launches (call outside a capture)
// skip (all cycle launchers): a device flag; non-zero makes the launch return at once (may be null)
// dots (may be null): the flexible-CG scalars taken in this sweep (its output is z, its b is r):
// z'r and z'q reduced into partials (2 x grid doubles) with st->ticket[6], then beta and r'z in st
struct FcgDotSink {
  const double* q = nullptr;
  double* partials = nullptr;
  PcgState* st = nullptr;
};
cudaError_t amg_sweep_f32(const int* skip, int mode, int cheb, const MixedMatrix& M, const double* dinv,
                          const double* lam, const double* b, const double* x, const double* xp, double* xo,
                          cudaStream_t s, const FcgDotSink* dots = nullptr);
// cycle operators in FP32 (values only; vectors and accumulation stay FP64)
cudaError_t amg_coarse_f32(const AmgBsr& A, float* val32, cudaStream_t s);
cudaError_t amg_transfer_f32(int B, const AmgBsr& P, int nnz_p, const int* pt_idx, const int* p_row, float* p32,
                             int* pt_row, float* pt32, cudaStream_t s);
cudaError_t amg_sweep3_f32(const int* skip, int mode, int cheb, const AmgBsr32& A, const double* dinv,
                           const double* lam, const double* b, const double* x, const double* xp, double* xo,
                           cudaStream_t s);
cudaError_t amg_restrict_f32(const int* skip, int B, int nc, const int* pt_ptr, const int* pt_row, const float* pt32,
                             const double* r, double* bc, cudaStream_t s);
cudaError_t amg_prolong_f32(const int* skip, int B, int n, const int* p_ptr, const int* p_col, const float* p32,
                            const double* xc, double* x, cudaStream_t s);
cudaError_t amg_gemv(const int* skip, int n, const double* M, const double* b, double* x, cudaStream_t s);

// The bottom of the V-cycle in one thread-block cluster (levels >= 1 with 3 x 3 blocks, then the
// dense coarsest solve): level 0 of the tail takes b and writes x like the per-level path.
constexpr int kAmgTailMax = 8;         // levels in a tail, the coarsest included
constexpr int kAmgTailThreads = 512;   // threads per CTA of the tail cluster
struct AmgTailLevel {
  AmgBsr32 A;
  const double* dinv = nullptr;
  const double* lam = nullptr;
  double* b = nullptr;   // right-hand side (level 0: the caller's; below: the restriction)
  double* x = nullptr;   // the level's result
  double* xa = nullptr;  // sweep scratch
  double* r = nullptr;   // residual
  int nc = 0;            // transfer to the next level
  const int* pt_ptr = nullptr;
  const int* pt_row = nullptr;
  const float* pt32 = nullptr;
  const int* p_ptr = nullptr;
  const int* p_col = nullptr;
  const float* p32 = nullptr;
};
struct AmgTail {
  int nl = 0;  // levels, the last one the dense coarsest (only its b and x are used)
  int cheb = 1;  // Chebyshev smoothing (else damped Jacobi)
  int n_coarse = 0;
  const double* Minv = nullptr;
  AmgTailLevel L[kAmgTailMax];
};
// cluster: CTAs in the one cluster (1..16); max_clusters != nullptr: only query how many such
// clusters fit at once (0 = the shape cannot launch), nothing is launched
cudaError_t amg_tail(const int* skip, const AmgTail& t, int cluster, int* max_clusters, cudaStream_t s);
cudaError_t amg_rigid_modes(int N, const double* xy, double* Bf, cudaStream_t s);

// Process-wide count of kernel launches issued by this library (graph launches count every
// kernel node they run).
void count_launches(long long k);
long long launches_total();

// mesh_kernels.cu
cudaError_t scan_exclusive(const int* in, int n, int* out, int* tmp, cudaStream_t s);
int scan_tmp_ints(int n);
cudaError_t launch_incidence(const MeshDev& m, int* cnt, int* cursor, int* ne_ptr, int* ne,
                             int* scan_tmp, int* err, cudaStream_t s);
cudaError_t launch_pattern_count(const MeshDev& m, const int* ne_ptr, const int* ne, int* deg,
                                 int* node_ptr, int* scan_tmp, int* err, cudaStream_t s);
cudaError_t launch_pattern_fill(const MeshDev& m, const int* ne_ptr, const int* ne,
                                const int* node_ptr, int* bnbr, int* slot, int* row_ptr,
                                int* cols, cudaStream_t s);
cudaError_t launch_assemble(const MeshDev& m, const int* ne_ptr, const int* ne, const int* slot,
                            const int* node_ptr, const Mat3& D, double t, const int* mat,
                            const double* Dtab, const double* ttab, double* vals, cudaStream_t s);
cudaError_t launch_dirichlet(int n_rows, const int* row_ptr, const int* cols, double* vals,
                             int n_fixed, const int* dofs, const double* values,
                             unsigned char* fixed, double* ubar, double* b, int n_rhs,
                             int* err, cudaStream_t s, bool apply);
cudaError_t launch_inv_diag(int n_rows, const int* row_ptr, const int* cols, const double* vals,
                            double* inv_diag, int* err, cudaStream_t s);
cudaError_t launch_element_stresses(const MeshDev& m, const double* u, const Mat3& D, double nu,
                                    int plane_strain, double* out, cudaStream_t s);

// pcg_kernels.cu
struct PcgBuffers {
  int n = 0;  // rows
  double* x = nullptr;
  double* r = nullptr;
  double* p = nullptr;
  double* Ap = nullptr;
  const double* inv_diag = nullptr;
  const double* b = nullptr;
  double* partials = nullptr;  // 4 * kMaxGrid doubles
  double* history = nullptr;   // max_iter + 1 or null
  PcgState* st = nullptr;
  int* err = nullptr;
  // mixed precision work vectors
  float* p32 = nullptr;
  float* Ap32 = nullptr;
  float* inv_diag32 = nullptr;
};

cudaError_t launch_pcg_init(const PcgBuffers& w, double rtol, int max_iter, bool hist,
                            cudaStream_t s);
// One CG iteration: SpMV + p'Ap, x/r update + norms, p update.
// The two phases of launch_pcg_iteration, launched separately (the instrumented solve times
// each): q = A p with p'Ap, then x / r / p updates with their dots.
// The architecture the library's kernels were compiled for, as the runtime reports it (100: sm_100a).
cudaError_t kernel_binary_version(int* version);
cudaError_t launch_spmv_phase(const PcgBuffers& w, const BlockMatrix* bm, const CsrMatrixDev* cm, cudaStream_t s);
cudaError_t launch_vector_phase(const PcgBuffers& w, cudaStream_t s);
cudaError_t launch_pcg_iteration(const PcgBuffers& w, const BlockMatrix* bm,
                                 const CsrMatrixDev* cm, cudaStream_t s);
// y = A x (plain SpMV).
cudaError_t launch_spmv(const BlockMatrix* bm, const CsrMatrixDev* cm, const double* x, double* y,
                        cudaStream_t s);
// True residual: r_true = b - A x into w.Ap (A x must already be in w.Ap), ||.|| -> st->true_rel.
// With `restart`, also r = r_true, p = D^-1 r, rz, and done = 0 when the iteration may go on.
cudaError_t launch_true_residual(const PcgBuffers& w, bool restart, int max_replacements,
                                 cudaStream_t s);

// persistent.cu: every iteration of a mesh-pattern solve in one cooperative kernel (FP64, or
// mixed when A32 is given); the state must be initialised (launch_pcg_init / launch_mixed_init).
// spin_limit: polls of a grid-barrier wait before the solve gives up (kBarrierSpinDefault).
constexpr long long kBarrierSpinDefault = 50000000LL;  // polls of ~40 ns: ~2 s
cudaError_t launch_pcg_persistent(const PcgBuffers& w, const BlockMatrix& A64, const MixedMatrix* A32,
                                  int max_final_checks, long long spin_limit, cudaStream_t s);

}  // namespace cstg
