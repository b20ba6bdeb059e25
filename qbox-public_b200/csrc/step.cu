// The electronic step on one GPU: ChargeDensity::update_density,
// EnergyFunctional::update_vhxc / energy, the PSDA stepper and
// SlaterDet::gram / ortho_align, orchestrated from the host over the
// kernels of fft.cu and kernels.cu and the dense linear algebra of cuBLAS and
// cuSOLVER (FP64).
//
// Matrices follow the reference's "DoubleMatrix proxy" view of a Gamma-point
// SlaterDet: C (ngw complex rows x nst columns, column-major) is read as a
// real 2*ngw x nst matrix, so C^T C counts +G and -G once each except the
// G=0 row, which the rank-1 corrections below remove
// (src/SlaterDet.cpp:480-534,768-876).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>

#include "qbx_internal.h"

namespace qbx {

static bool mixed(const Context& ctx) { return ctx.precision == MIXED; }

// S = 2 C^T C - c0 c0^T, lower triangle, then S = L L^T in place.  In the
// mixed path the product uses the BF16 split of c in slot `split` and the
// diagonal is recomputed exactly in FP64.  The factorisation's info code
// goes to the status word `status` (checked when the step's scalars are
// read back: a matrix that is not positive definite is an error there).
static void overlap_cholesky(Context& ctx, const double* c, double* S, int status, int split,
                             bool diag_from_split = false) {
  ProfScope ps(ctx, "overlap_cholesky");
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  const double two = 2.0, zero = 0.0;
  if (split >= 0) {
    // lower triangle only, as the FP64 path's syrk: potrf reads nothing else
    split_gemm(ctx, true, false, n, n, K, 2.0, ctx.cs_hi[split], ctx.cs_lo[split], ctx.ldp,
               ctx.cs_hi[split], ctx.cs_lo[split], ctx.ldp, 0.0, S, true);
    launch_rank1_fix(ctx, S, n, c, K, c, K, n, n, -1.0, true);
    if (diag_from_split) overlap_diag_from_split(ctx, c, K, n, ctx.ldp, S);
    else overlap_diag_f64(ctx, c, K, n, S);
  } else {
    QBX_BLAS(cublasDsyrk(ctx.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, n, K, &two, c, K, &zero,
                         S, n));
    launch_rank1_fix(ctx, S, n, c, K, c, K, n, n, -1.0, true);
  }
  QBX_SOLVER(cusolverDnDpotrf(ctx.solver, CUBLAS_FILL_MODE_LOWER, n, S, n, ctx.d_solver_work,
                              ctx.solver_lwork, ctx.d_status + status));
}

static void rotate(Context& ctx, double* x, const double* M);

// SlaterDet::gram (src/SlaterDet.cpp:480-534): C <- C L^-T.  With
// split_overlap in the mixed path (the MD extrapolation), the overlap is the
// split BF16 product with its FP64 diagonal and C L^-T the split TF32
// rotation C - C (I - L^-T), as in ortho_align; otherwise FP64 throughout.
void gram(Context& ctx, bool split_overlap) {
  launch_cleanup(ctx, ctx.d_c);
  if (split_overlap && mixed(ctx)) {
    const int n = ctx.nst, K = 2 * ctx.wb.ng;
    const double one = 1.0;
    split_bf16_2d(ctx, ctx.d_c, K, n, K, ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp);
    overlap_cholesky(ctx, ctx.d_c, ctx.d_nn, ST_INFO_GRAM, 1);
    double* X = ctx.d_nn2;
    launch_identity_axpy(ctx, X, X, n, 0.0);
    QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                         CUBLAS_DIAG_NON_UNIT, n, n, &one, ctx.d_nn, n, X, n));   // L^-T
    rotate(ctx, ctx.d_c, X);
    return;
  }
  overlap_cholesky(ctx, ctx.d_c, ctx.d_nn, ST_INFO_GRAM, -1);
  const double one = 1.0;
  QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                       CUBLAS_DIAG_NON_UNIT, 2 * ctx.wb.ng, ctx.nst, &one, ctx.d_nn, ctx.nst,
                       ctx.d_c, 2 * ctx.wb.ng));
}

// DoubleMatrix::polar (src/Matrix.cpp:2446-2540) on x (n x n, in place):
// Bjorck-Bowie steps x <- x (I + q/2 (I + 3q/4)), q = I - x^T x, while
// ||q||_F < 1, Higham steps x <- (x + x^-T)/2 otherwise; stops after the
// step in which ||q||_F <= tol.

// q = I - x^T x (full matrix) and SLOT_FROB = ||q||_F^2
static void polar_q(Context& ctx, const double* x, double* q) {
  const int n = ctx.nst;
  const double one = 1.0, mone = -1.0;
  launch_identity_axpy(ctx, q, q, n, 0.0);   // q = I
  QBX_BLAS(cublasDsyrk(ctx.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, n, n, &mone, x, n, &one, q, n));
  launch_symmetrize_lower(ctx, q, n);
  launch_frob2(ctx, q, n);
}

// x <- x (I + q/2 (I + 3q/4))
static void polar_bjorck(Context& ctx, double* x, const double* q, double* t, double* qt,
                         double* xp) {
  const int n = ctx.nst;
  const double one = 1.0, zero = 0.0;
  launch_identity_axpy(ctx, t, q, n, 0.75);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, q, n, t, n, &zero, qt, n));
  launch_identity_axpy(ctx, t, qt, n, 0.5);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, x, n, t, n, &zero, xp, n));
  QBX_CUDA(cudaMemcpyAsync(x, xp, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, ctx.stream));
}

// t = P I for the row interchanges of an LU factorisation (ipiv 1-based,
// applied in order), one thread per column
__global__ void k_pivoted_identity(double* __restrict__ t, const int* __restrict__ ipiv, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double* col = t + (size_t)j * n;
  for (int i = 0; i < n; i++) col[i] = i == j ? 1.0 : 0.0;
  for (int i = 0; i < n; i++) {
    const int p = ipiv[i] - 1;
    if (p != i && p >= 0 && p < n) {
      const double a = col[i];
      col[i] = col[p];
      col[p] = a;
    }
  }
}

// x <- (x + x^-T)/2, x^-T by an LU factorisation of x^T (P x^T = L U) and
// the two triangular solves of U^-1 L^-1 P.  (cuSOLVER's getrs would do the
// same; at some sizes it allocates stream-ordered memory, which a
// conditional graph body cannot hold.)
static void polar_higham(Context& ctx, double* x, double* t, double* qt) {
  const int n = ctx.nst;
  const double one = 1.0, zero = 0.0;
  QBX_BLAS(cublasDgeam(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, &one, x, n, &zero, x, n, qt, n));
  QBX_SOLVER(cusolverDnDgetrf(ctx.solver, n, n, qt, n, ctx.d_solver_work, ctx.d_ipiv,
                              ctx.d_status + ST_INFO_POLAR));
  k_pivoted_identity<<<(n + 127) / 128, 128, 0, ctx.stream>>>(t, ctx.d_ipiv, n);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                       CUBLAS_DIAG_UNIT, n, n, &one, qt, n, t, n));
  QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                       CUBLAS_DIAG_NON_UNIT, n, n, &one, qt, n, t, n));
  launch_avg_transpose(ctx, x, t, n);
}

// ------------------------------------------------ inverse of a lower triangle
// The inverses of the diagonal 32 x 32 blocks of a lower-triangular L (ld n)
// into the same blocks of Li: one warp per block, thread j forms column j by
// forward substitution, x_i = (delta_ij - sum_{k<i} L_ik x_k) / L_ii with
// x_k = 0 above the diagonal, in FP64.  Only the lower triangle of L is read.
__global__ void __launch_bounds__(32) k_tri_inv_diag32(const double* __restrict__ L, int n,
                                                       double* __restrict__ Li) {
  __shared__ double sl[32][33];
  const int k0 = 32 * blockIdx.x, j = threadIdx.x;
  for (int c = 0; c < 32; c++) sl[j][c] = L[(size_t)(k0 + c) * n + k0 + j];
  __syncwarp();
  double x[32];
#pragma unroll
  for (int i = 0; i < 32; i++) {
    double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < i; k++) s -= sl[i][k] * x[k];
    x[i] = (i < j) ? 0.0 : s / sl[i][i];
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; i++) sl[i][j] = x[i];
  __syncwarp();
  for (int c = 0; c < 32; c++) Li[(size_t)(k0 + c) * n + k0 + j] = sl[j][c];
}

// Li = L^-1 for a lower-triangular n x n L (column-major, ld n; its upper
// triangle is not read), for n = 32 x a power of two: the diagonal 32 x 32
// blocks inverted directly, then, doubling the block size b, each pair of
// neighbouring inverted blocks A^-1 (upper left) and C^-1 (lower right) with
// the block B of L below A gets the off-diagonal block -C^-1 B A^-1 of the
// inverse: two strided-batched FP64 GEMMs per level, all pairs of a level in
// one call.  work holds n * n / 4 doubles.  Other n (or none of the blocked
// form): one triangular solve of I, as cuBLAS's trsm.
bool lower_inverse_blocked(int n) { return n >= 32 && n % 32 == 0 && ((n / 32) & (n / 32 - 1)) == 0; }

void lower_inverse(Context& ctx, const double* L, int n, double* Li, double* work) {
  const double one = 1.0, zero = 0.0, mone = -1.0;
  if (!lower_inverse_blocked(n)) {
    launch_identity_axpy(ctx, Li, Li, n, 0.0);
    QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                         CUBLAS_DIAG_NON_UNIT, n, n, &one, L, n, Li, n));
    return;
  }
  QBX_CUDA(cudaMemsetAsync(Li, 0, sizeof(double) * n * n, ctx.stream));
  k_tri_inv_diag32<<<n / 32, 32, 0, ctx.stream>>>(L, n, Li);
  QBX_LAUNCHED(ctx);
  for (int b = 32; b < n; b *= 2) {
    const int pairs = n / (2 * b);
    const long long st = 2LL * b * (n + 1);   // one pair's diagonal block to the next
    // work_p = B_p A_p^-1
    QBX_BLAS(cublasDgemmStridedBatched(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, b, b, b, &one, L + b,
                                       n, st, Li, n, st, &zero, work, b, (long long)b * b, pairs));
    // the block of Li below A_p^-1: -C_p^-1 work_p
    QBX_BLAS(cublasDgemmStridedBatched(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, b, b, b, &mone,
                                       Li + b + (size_t)b * n, n, st, work, b, (long long)b * b,
                                       &zero, Li + b, n, st, pairs));
  }
}

// The same Higham step for the mixed path, with x^-T = x (x^T x)^-1 formed
// from the Cholesky factor of x^T x = I - q (q of this iteration, full):
// S = L L^T, W = L^-1, S^-1 = W^T W, x <- x (I + S^-1) / 2.  One Cholesky
// factor and one triangular inverse instead of a pivoted LU and two solves
// (cuSOLVER's pivoted getrf took 2.1 ms at n = 1 024, the whole step 0.8 ms).
// x^T x squares x's condition number; the Bjorck-Bowie steps that follow
// converge to the same polar factor in FP64.
static void polar_higham_chol(Context& ctx, double* x, const double* q, double* t, double* qt,
                              double* xp) {
  const int n = ctx.nst;
  const double one = 1.0, zero = 0.0, half = 0.5;
  launch_identity_axpy(ctx, qt, q, n, -1.0);    // S = I - q = x^T x
  QBX_SOLVER(cusolverDnDpotrf(ctx.solver, CUBLAS_FILL_MODE_LOWER, n, qt, n, ctx.d_solver_work,
                              ctx.solver_lwork, ctx.d_status + ST_INFO_POLAR));
  lower_inverse(ctx, qt, n, t, xp);              // t = L^-1 (xp is free until the syrk)
  QBX_BLAS(cublasDsyrk(ctx.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, n, n, &one, t, n, &zero,
                       xp, n));                  // S^-1 = W^T W (lower)
  launch_symmetrize_lower(ctx, xp, n);
  launch_identity_axpy(ctx, qt, xp, n, 1.0);    // I + S^-1
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &half, x, n, qt, n, &zero, xp,
                       n));
  QBX_CUDA(cudaMemcpyAsync(x, xp, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, ctx.stream));
}

// After q of an iteration: choose the branch (1: Bjorck-Bowie, 0: Higham)
// and whether another iteration follows, as the host loop below does.
__global__ void k_polar_decide_gamma(const double* __restrict__ frob2, double tol, int maxiter,
                               int* __restrict__ iters, cudaGraphConditionalHandle loop,
                               cudaGraphConditionalHandle branch) {
  const double qn = sqrt(*frob2);
  const int it = *iters + 1;
  *iters = it;
  cudaGraphSetConditional(branch, qn < 1.0 ? 1u : 0u);
  cudaGraphSetConditional(loop, (qn > tol && it < maxiter) ? 1u : 0u);
}

// ------------------------------------------------ conditional graph nodes
// The graph being captured on stream s.
cudaGraph_t capture_graph(cudaStream_t s) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  QBX_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr));
  QBX_REQUIRE(st == cudaStreamCaptureStatusActive && g, 56, "stream is not capturing");
  return g;
}

// Appends a conditional node of the given type after the current capture
// dependencies of s, makes it the only dependency, and returns its bodies.
cudaGraph_t* add_conditional(cudaStream_t s, cudaGraphConditionalHandle h,
                             cudaGraphConditionalNodeType type, unsigned size) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  QBX_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  QBX_REQUIRE(st == cudaStreamCaptureStatusActive, 56, "stream is not capturing");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = size;
  cudaGraphNode_t node;
  QBX_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  QBX_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return p.conditional.phGraph_out;
}

// Runs f with ctx.stream (and cuBLAS/cuSOLVER) on s, capturing into body.
void capture_body(Context& ctx, cudaGraph_t body, cudaStream_t s, const std::function<void()>& f) {
  cudaStream_t saved = ctx.stream;
  QBX_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed));
  ctx.stream = s;
  bind_stream(ctx, s);
  try {
    f();
  } catch (...) {
    cudaGraph_t g;
    cudaStreamEndCapture(s, &g);
    ctx.stream = saved;
    bind_stream(ctx, saved);
    throw;
  }
  ctx.stream = saved;
  bind_stream(ctx, saved);
  cudaGraph_t g;
  QBX_CUDA(cudaStreamEndCapture(s, &g));
}

static void polar(Context& ctx, double* x, double tol, int maxiter) {
  ProfScope ps(ctx, "polar");
  const int n = ctx.nst;
  double* q = ctx.d_nn3;
  double* t = ctx.d_nn4;
  double* qt = ctx.d_nn4 + (size_t)n * n;
  double* xp = ctx.d_nn4 + 2 * (size_t)n * n;
  if (!ctx.capturing) {
    ctx.polar_iters = 0;
    for (int iter = 0; iter < maxiter; iter++) {
      polar_q(ctx, x, q);
      const double qn = std::sqrt(read_slot(ctx, SLOT_FROB));
      if (qn < 1.0) polar_bjorck(ctx, x, q, t, qt, xp);
      else if (mixed(ctx)) polar_higham_chol(ctx, x, q, t, qt, xp);
      else polar_higham(ctx, x, t, qt);
      ctx.polar_iters = iter + 1;
      if (qn <= tol) break;
    }
    return;
  }
  // Captured: a WHILE node whose body forms q, decides on the device, and
  // runs the chosen step in an IF/ELSE node.  The loop handle is reset to 1
  // at every launch of the graph, so the body runs at least once.
  int* iters = ctx.d_status + ST_POLAR_ITERS;
  QBX_CUDA(cudaMemsetAsync(iters, 0, sizeof(int), ctx.stream));
  cudaGraphConditionalHandle loop;
  QBX_CUDA(cudaGraphConditionalHandleCreate(&loop, capture_graph(ctx.stream), 1,
                                            cudaGraphCondAssignDefault));
  cudaGraph_t body = add_conditional(ctx.stream, loop, cudaGraphCondTypeWhile, 1)[0];
  capture_body(ctx, body, ctx.side[0], [&]() {
    polar_q(ctx, x, q);
    cudaGraphConditionalHandle branch;
    QBX_CUDA(cudaGraphConditionalHandleCreate(&branch, capture_graph(ctx.stream), 0, 0));
    k_polar_decide_gamma<<<1, 1, 0, ctx.stream>>>(ctx.d_scalars + SLOT_FROB, tol, maxiter, iters,
                                                  loop, branch);
    QBX_LAUNCHED(ctx);
    cudaGraph_t* arms = add_conditional(ctx.stream, branch, cudaGraphCondTypeIf, 2);
    cudaGraph_t bjorck = arms[0], higham = arms[1];
    capture_body(ctx, bjorck, ctx.side[1], [&]() { polar_bjorck(ctx, x, q, t, qt, xp); });
    capture_body(ctx, higham, ctx.side[1], [&]() {
      if (mixed(ctx)) polar_higham_chol(ctx, x, q, t, qt, xp);
      else polar_higham(ctx, x, t, qt);
    });
  });
}

void launch_polar_decide(Context& ctx, double tol, int maxiter, int* iters,
                         cudaGraphConditionalHandle loop, cudaGraphConditionalHandle branch) {
  k_polar_decide_gamma<<<1, 1, 0, ctx.stream>>>(ctx.d_scalars + SLOT_FROB, tol, maxiter, iters,
                                                loop, branch);
  QBX_LAUNCHED(ctx);
}

// The orthogonal polar factor of x (nst x nst, device) in place, eagerly or
// inside a capture (the form ortho_align uses).
void polar_factor(Context& ctx, double* x, double tol, int maxiter) { polar(ctx, x, tol, maxiter); }

// DoubleMatrix::polar as an operation of its own: x (nst x nst, device) in
// place, eagerly or captured into a graph (the form the captured step uses)
// and launched once.  Returns the iterations run.
int polar_entry(Context& ctx, double* x, double tol, int maxiter, bool graph) {
  if (!graph) {
    polar(ctx, x, tol, maxiter);
    return ctx.polar_iters;
  }
  const bool prof = ctx.prof.on;
  ctx.prof.on = false;
  cudaGraph_t g = nullptr;
  QBX_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeRelaxed));
  ctx.capturing = true;
  try {
    polar(ctx, x, tol, maxiter);
  } catch (...) {
    cudaStreamEndCapture(ctx.stream, &g);
    if (g) cudaGraphDestroy(g);
    ctx.capturing = false;
    ctx.prof.on = prof;
    throw;
  }
  ctx.capturing = false;
  ctx.prof.on = prof;
  QBX_CUDA(cudaStreamEndCapture(ctx.stream, &g));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  QBX_CUDA(e);
  const cudaError_t l = cudaGraphLaunch(ex, ctx.stream);
  const cudaError_t w = cudaStreamSynchronize(ctx.stream);
  cudaGraphExecDestroy(ex);
  QBX_CUDA(l);
  QBX_CUDA(w);
  int iters = 0;
  QBX_CUDA(cudaMemcpy(&iters, ctx.d_status + ST_POLAR_ITERS, sizeof(int), cudaMemcpyDeviceToHost));
  return iters;
}

// out += alpha * c * M for the FP64 wavefunction block c (K x n) and an n x n
// matrix M: the tcgen05 kernel on the split of c (BF16 or TF32 hi/lo of the
// given kind: its plain split, read MN-major, with the 256 x 256 CTA pairs;
// else its transposed split), or three cuBLAS TF32 products on its plain
// split.  out may be c itself: both read the split copy of c.
static void tall_update(Context& ctx, int kind, const double* c, const double* M, double alpha,
                        double* out, const void* c_hi = nullptr, const void* c_lo = nullptr) {
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  if (ctx.gemm_backend == 1) {
    const int ld = Context::tall_ld_of(kind, n);
    split_plain(ctx, kind, M, n, n, n, ctx.tm_hi, ctx.tm_lo, ld);   // M is K-major as stored
    if (ctx.tc_pair == 2 && (kind == TALL_BF16 || ctx.tc_tf32_mn)) {
      // the CTA-pair kernel reads c's plain split as an MN-major operand:
      // the caller's (c_hi, c_lo: this kind, ld ldp) or one made here
      if (!c_hi) {
        split_plain(ctx, kind, c, K, n, K, ctx.ct_hi, ctx.ct_lo, ctx.ldp);
        c_hi = ctx.ct_hi;
        c_lo = ctx.ct_lo;
      }
      tc_gemm_kind_nn_mn(ctx, kind, K, n, n, alpha, c_hi, c_lo, ctx.ldp, ctx.tm_hi, ctx.tm_lo, ld,
                         1.0, out, K);
      return;
    }
    split_t(ctx, kind, c, K, n, K, ctx.ct_hi, ctx.ct_lo, ld);
    tc_gemm_kind_tn(ctx, kind, K, n, n, alpha, ctx.ct_hi, ctx.ct_lo, ld, ctx.tm_hi, ctx.tm_lo, ld,
                    1.0, out, K);
  } else {
    split_tf32(ctx, M, n, n, n, ctx.s32, ctx.s32lo, pad4(n));
    split_tf32(ctx, c, K, n, K, ctx.c32, ctx.c32lo, ctx.ldp);
    tf32x3_gemm_nn(ctx, K, n, n, alpha, ctx.c32, ctx.c32lo, ctx.ldp, ctx.s32, ctx.s32lo, pad4(n),
                   1.0, out, K);
  }
}

// SlaterDet::ortho_align (src/SlaterDet.cpp:768-876)
bool ortho_splits_both(const Context& ctx) {
  return mixed(ctx) && ctx.gemm_backend == 1 && ctx.tc_pair == 2 && ctx.tc_tf32_mn &&
         ctx.tall_kind == TALL_TF32 && ctx.d_colred;
}

void ortho_align(Context& ctx, bool c_split_done) {
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  const double one = 1.0, two = 2.0, zero = 0.0;
  const bool mx = mixed(ctx);
  // in the mixed path slot 0 holds the split of C_last (made in energy());
  // where the rotation reads C's plain TF32 split, both splits of C are made
  // in one pass (or by the PSDA step that formed C)
  const bool both = ortho_splits_both(ctx);
  QBX_REQUIRE(!c_split_done || both, 50, "ortho_align: C's splits were made for another path");
  if (!c_split_done) launch_cleanup(ctx, ctx.d_c);
  double* L = ctx.d_nn;
  double* X = ctx.d_nn2;
  if (!mx)
    QBX_CUDA(cudaMemcpyAsync(ctx.d_ctmp, ctx.d_c, sizeof(double) * (size_t)K * n,
                             cudaMemcpyDeviceToDevice, ctx.stream));
  if (both && !c_split_done)
    split_bf16_tf32(ctx, ctx.d_c, K, n, K, ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp, (float*)ctx.ct_hi,
                    (float*)ctx.ct_lo, ctx.ldp);
  else if (mx && !both)
    split_bf16_2d(ctx, ctx.d_c, K, n, K, ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp);
  overlap_cholesky(ctx, ctx.d_c, L, ST_INFO_ORTHO, mx ? 1 : -1, both);
  // B = 2 C^T C_last - c0 c_last0^T
  {
    ProfScope ps(ctx, "gemm_overlap_last");
    if (mx)
      split_gemm(ctx, true, false, n, n, K, 2.0, ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp,
                 ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp, 0.0, X);
    else
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, ctx.d_c, K,
                           ctx.d_c_last, K, &zero, X, n));
  }
  launch_rank1_fix(ctx, X, n, ctx.d_c, K, ctx.d_c_last, K, n, n, -1.0, false);
  if (mx) {
    // L^-1 once (one triangular solve of I), then two products in place of
    // the two solves with L and L^T (each solve as slow as the inverse)
    double* Li = ctx.d_nn5;
    double* T = L;   // L is not read after L^-1 is formed
    lower_inverse(ctx, L, n, Li, ctx.d_nn3);   // d_nn3 is free until the rotation
    QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, Li, n, X, n, &zero, T,
                         n));
    polar(ctx, T, 1.e-6, 20);
    QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, Li, n, T, n, &zero, X,
                         n));
  } else {
    QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                         CUBLAS_DIAG_NON_UNIT, n, n, &one, L, n, X, n));
    polar(ctx, X, 1.e-6, 20);
    QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                         CUBLAS_DIAG_NON_UNIT, n, n, &one, L, n, X, n));
  }
  ProfScope ps(ctx, "gemm_rotate");
  if (mx) {
    // C <- C - C (I - X): the split-precision error only touches the
    // correction, so C stays orthonormal to the accuracy of the overlap.
    double* T = ctx.d_nn3;
    launch_identity_axpy(ctx, T, X, n, -1.0);
    // rotation: TF32 splits, so that C stays orthonormal to ~1e-7
    tall_update(ctx, ctx.tall_kind, ctx.d_c, T, -1.0, ctx.d_c, both ? ctx.ct_hi : nullptr,
                both ? ctx.ct_lo : nullptr);
  } else {
    QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &one, ctx.d_ctmp, K, X, n,
                         &zero, ctx.d_c, K));
  }
}

// zero the strictly upper triangle of an n x n column-major matrix
__global__ void k_lower_only(double* __restrict__ a, int n) {
  const size_t nn = (size_t)n * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nn;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    if (i < j) a[t] = 0.0;
  }
}

// x <- x M for a K x n wavefunction block x and an n x n matrix M: in the
// mixed path x - x (I - M) through the TF32 tall update (M close to the
// identity, so the split error only touches the correction), else one FP64
// GEMM from a copy of x
static void rotate(Context& ctx, double* x, const double* M) {
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  if (mixed(ctx)) {
    double* T = ctx.d_nn3;
    launch_identity_axpy(ctx, T, M, n, -1.0);
    tall_update(ctx, ctx.tall_kind, x, T, -1.0, x);
    return;
  }
  const double one = 1.0, zero = 0.0;
  QBX_CUDA(cudaMemcpyAsync(ctx.d_ctmp, x, sizeof(double) * (size_t)K * n,
                           cudaMemcpyDeviceToDevice, ctx.stream));
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &one, ctx.d_ctmp, K, M, n,
                       &zero, x, K));
}

// SlaterDet::align (src/SlaterDet.cpp:979-1044) of the block cv to C:
// cv <- cv X, X the orthogonal polar factor of B = 2 cv^T C - cv0 c0^T
// (BF16 split product in the mixed path)
void align_to_c(Context& ctx, double* cv) {
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  double* X = ctx.d_nn2;
  if (mixed(ctx)) {
    split_bf16_2d(ctx, cv, K, n, K, ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp);
    split_bf16_2d(ctx, ctx.d_c, K, n, K, ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp);
    split_gemm(ctx, true, false, n, n, K, 2.0, ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp,
               ctx.cs_hi[1], ctx.cs_lo[1], ctx.ldp, 0.0, X);
  } else {
    const double two = 2.0, zero = 0.0;
    QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, cv, K, ctx.d_c, K,
                         &zero, X, n));
  }
  launch_rank1_fix(ctx, X, n, cv, K, ctx.d_c, K, n, n, -1.0, false);
  polar(ctx, X, 1.e-6, 20);
  rotate(ctx, cv, X);
}

// SlaterDet::lowdin (src/SlaterDet.cpp:674-721): S = 2 C^T C - c0 c0^T =
// L L^T, U the orthogonal polar factor of L^T, C <- C L^-T U
void lowdin(Context& ctx) {
  const int n = ctx.nst;
  const double one = 1.0, zero = 0.0;
  const bool mx = mixed(ctx);
  launch_cleanup(ctx, ctx.d_c);
  double* L = ctx.d_nn;
  double* X = ctx.d_nn2;
  if (mx) split_bf16_2d(ctx, ctx.d_c, 2 * ctx.wb.ng, n, 2 * ctx.wb.ng, ctx.cs_hi[1], ctx.cs_lo[1],
                        ctx.ldp);
  overlap_cholesky(ctx, ctx.d_c, L, ST_INFO_GRAM, mx ? 1 : -1);
  k_lower_only<<<(int)std::min<size_t>(((size_t)n * n + 255) / 256, 148 * 16), 256, 0,
                 ctx.stream>>>(L, n);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasDgeam(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, &one, L, n, &zero, L, n, X, n));
  polar(ctx, X, 1.e-6, 20);
  // X <- L^-T U
  QBX_BLAS(cublasDtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                       CUBLAS_DIAG_NON_UNIT, n, n, &one, L, n, X, n));
  rotate(ctx, ctx.d_c, X);
}

// ChargeDensity::update_density (src/ChargeDensity.cpp:136-198)
void update_density(Context& ctx) {
  ProfScope ps(ctx, "update_density");
  launch_density(ctx, ctx.d_c, ctx.d_rhor);
  launch_sum(ctx, ctx.d_rhor, ctx.N(), SLOT_CHARGE);   // total charge
  vb_forward_real(ctx, ctx.d_rhor, ctx.vb.omega, ctx.d_rhog);
}

// EnergyFunctional::update_vhxc (src/EnergyFunctional.cpp:231-394)
void update_vhxc(Context& ctx) {
  ProfScope ps(ctx, "update_vhxc");
  launch_xc(ctx);
  launch_vhxc_gspace(ctx);
}

// NonLocalPotential::energy (src/NonLocalPotential.cpp:1258-1640):
// F = 2 A^T C - a0 c0^T, E_nl, and H C += A (D F / Omega)
static void nonlocal(Context& ctx, bool hpsi) {
  if (ctx.nproj == 0) return;
  const int n = ctx.nst, K = 2 * ctx.wb.ng, np = ctx.nproj;
  const double one = 1.0, two = 2.0, zero = 0.0;
  const bool mx = mixed(ctx);
  {
    ProfScope ps(ctx, "gemm_nl_project");
    if (mx)
      split_gemm(ctx, true, false, np, n, K, 2.0, ctx.as_hi, ctx.as_lo, ctx.ldp, ctx.cs_hi[0],
                 ctx.cs_lo[0], ctx.ldp, 0.0, ctx.d_fnl);
    else
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, np, n, K, &two, ctx.d_anl, K,
                           ctx.d_c, K, &zero, ctx.d_fnl, np));
  }
  launch_rank1_fix(ctx, ctx.d_fnl, np, ctx.d_anl, K, ctx.d_c, K, np, n, -1.0, false);
  launch_enl(ctx);
  if (hpsi) {
    ProfScope ps(ctx, "gemm_nl_apply");
    if (mx) {
      if (ctx.gemm_backend == 1) {
        // F (np x n) is already K-major for this product: a plain split
        const int kind = ctx.tall_kind_hc, ld = Context::tall_ld_of(kind, np);
        split_plain(ctx, kind, ctx.d_fnl, np, n, np, ctx.tm_hi, ctx.tm_lo, ld);
        tc_gemm_kind_tn(ctx, kind, K, n, np, 1.0, ctx.at_hi, ctx.at_lo, ld, ctx.tm_hi, ctx.tm_lo,
                        ld, 1.0, ctx.d_hc, K);
      } else {
        split_tf32(ctx, ctx.d_fnl, np, n, np, ctx.s32, ctx.s32lo, pad4(np));
        tf32x3_gemm_nn(ctx, K, n, np, 1.0, ctx.a32, ctx.a32lo, ctx.ldp, ctx.s32, ctx.s32lo,
                       pad4(np), 1.0, ctx.d_hc, K);
      }
    } else {
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, np, &one, ctx.d_anl, K,
                           ctx.d_fnl, np, &one, ctx.d_hc, K));
    }
  }
}

void nonlocal_only(Context& ctx, bool hpsi, double* out) {
  const int K = 2 * ctx.wb.ng;
  if (mixed(ctx))
    split_bf16_2d(ctx, ctx.d_c, K, ctx.nst, K, ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp);
  if (hpsi)
    QBX_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)K * ctx.nst, ctx.stream));
  double* saved = ctx.d_hc;
  ctx.d_hc = out;
  try {
    nonlocal(ctx, hpsi);
  } catch (...) {
    ctx.d_hc = saved;
    throw;
  }
  ctx.d_hc = saved;
}

bool energy_forms_prec(const Context& ctx) { return mixed(ctx) && ctx.d_colred && ctx.step_fuse; }

// EnergyFunctional::energy (src/EnergyFunctional.cpp:397-1044)
void energy(Context& ctx, bool hpsi, bool forces) {
  ProfScope ps(ctx, "energy");
  if (energy_forms_prec(ctx)) {
    // the split for the inner products, the kinetic sum and the
    // preconditioner's band energies in one pass over C
    split_bf16_ekin(ctx, ctx.d_c, 2 * ctx.wb.ng, ctx.nst, 2 * ctx.wb.ng, ctx.cs_hi[0],
                    ctx.cs_lo[0], ctx.ldp, ctx.d_g2_w, ctx.d_occ, ctx.d_scalars + SLOT_EKIN,
                    ctx.d_prec);
  } else {
    if (mixed(ctx))
      split_bf16_2d(ctx, ctx.d_c, 2 * ctx.wb.ng, ctx.nst, 2 * ctx.wb.ng, ctx.cs_hi[0],
                    ctx.cs_lo[0], ctx.ldp);
    launch_ekin(ctx);
  }
  if (hpsi) {
    ProfScope pv(ctx, "vpsi");
    launch_vpsi(ctx, ctx.d_c, ctx.d_vr, ctx.d_hc);   // hc = 1/2 G^2 c + V psi
  }
  nonlocal(ctx, hpsi);
  // the energies are formed on the host from the slots (finish_energy)
  if (forces) {
    int natoms = 0;
    for (auto& t : ctx.tau) natoms += (int)t.size() / 3;
    QBX_CUDA(cudaMemsetAsync(ctx.d_fion, 0, sizeof(double) * 3 * natoms, ctx.stream));
    launch_local_forces(ctx, ctx.d_fion);
    if (ctx.nproj) launch_nl_forces(ctx, ctx.d_fion);
  }
}

// PSDAWavefunctionStepper::update (src/PSDAWavefunctionStepper.cpp:46-249)
void psda_update(Context& ctx, unsigned fuse) {
  ProfScope ps(ctx, "psda_update");
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  const double one = 1.0, two = 2.0, zero = 0.0, mone = -1.0;
  double* A = ctx.d_nn;
  const bool eig_in_split = (fuse & PSDA_EIGSUM) && mixed(ctx) && ctx.d_colred && ctx.step_fuse;
  if ((fuse & PSDA_EIGSUM) && !eig_in_split) launch_eigsum(ctx);
  {
    ProfScope pg(ctx, "gemm_residual");
    if (mixed(ctx)) {
      if (eig_in_split)
        split_bf16_dot(ctx, ctx.d_hc, ctx.d_c, K, n, K, ctx.hs_hi, ctx.hs_lo, ctx.ldp,
                       ctx.d_scalars + SLOT_EIG);
      else
        split_bf16_2d(ctx, ctx.d_hc, K, n, K, ctx.hs_hi, ctx.hs_lo, ctx.ldp);
      split_gemm(ctx, true, false, n, n, K, 2.0, ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp, ctx.hs_hi,
                 ctx.hs_lo, ctx.ldp, 0.0, A);
      launch_rank1_fix(ctx, A, n, ctx.d_c, K, ctx.d_hc, K, n, n, -1.0, false);
      // C's BF16 split from energy() is the MN-major operand when the kinds agree
      const bool bf = ctx.tall_kind_hc == TALL_BF16;
      tall_update(ctx, ctx.tall_kind_hc, ctx.d_c, A, -1.0, ctx.d_hc, bf ? ctx.cs_hi[0] : nullptr,
                  bf ? ctx.cs_lo[0] : nullptr);
    } else {
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, ctx.d_c, K, ctx.d_hc,
                           K, &zero, A, n));
      launch_rank1_fix(ctx, A, n, ctx.d_c, K, ctx.d_hc, K, n, n, -1.0, false);
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &mone, ctx.d_c, K, A, n,
                           &one, ctx.d_hc, K));
    }
  }
  if (!((fuse & PSDA_PREC_FROM_ENERGY) && energy_forms_prec(ctx))) launch_precond_update(ctx);
  // the step writes the new C's splits for ortho_align in the same pass
  const bool split_c = ortho_splits_both(ctx) && ctx.step_fuse;
  launch_psda_elementwise(ctx, split_c);
  ortho_align(ctx, split_c);
  ctx.extrapolate = true;
}

// Wavefunction::diag(dwf, eigvec) (src/Wavefunction.cpp:834-917), real
// basis: h = 2 C^T (H C) - c0 hc0^T (the H C of the last energy()), its
// eigenvalues by syevd into w (device, nst); with eigvec the eigenvectors Z
// rotate C <- C Z and H*C takes the previous C, as the reference overwrites
// dwf with it.  The products are FP64 in both precisions.
void diag(Context& ctx, bool eigvec, double* w) {
  ProfScope ps(ctx, "diag");
  const int n = ctx.nst, K = 2 * ctx.wb.ng;
  const double one = 1.0, two = 2.0, zero = 0.0;
  double* h = ctx.d_nn;
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, ctx.d_c, K, ctx.d_hc, K,
                       &zero, h, n));
  launch_rank1_fix(ctx, h, n, ctx.d_c, K, ctx.d_hc, K, n, n, -1.0, false);
  int lwork = 0;
  const cusolverEigMode_t mode = eigvec ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
  QBX_SOLVER(cusolverDnDsyevd_bufferSize(ctx.solver, mode, CUBLAS_FILL_MODE_LOWER, n, h, n, w,
                                         &lwork));
  double* work = dalloc<double>(std::max(1, lwork));
  try {
    QBX_SOLVER(cusolverDnDsyevd(ctx.solver, mode, CUBLAS_FILL_MODE_LOWER, n, h, n, w, work, lwork,
                                ctx.d_info));
    int info = 0;
    QBX_CUDA(cudaMemcpyAsync(&info, ctx.d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    QBX_CUDA(cudaStreamSynchronize(ctx.stream));
    QBX_REQUIRE(info == 0, 41, "syevd of the subspace Hamiltonian failed (info=" +
                                   std::to_string(info) + ")");
    if (eigvec) {
      QBX_CUDA(cudaMemcpyAsync(ctx.d_hc, ctx.d_c, sizeof(double) * (size_t)K * n,
                               cudaMemcpyDeviceToDevice, ctx.stream));
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &one, ctx.d_hc, K, h, n,
                           &zero, ctx.d_c, K));
      ctx.extrapolate = false;
    }
    QBX_CUDA(cudaStreamSynchronize(ctx.stream));
  } catch (...) {
    dfree(work);
    throw;
  }
  dfree(work);
}

// JDWavefunctionStepper::update (src/JDWavefunctionStepper.cpp:47-376),
// real basis: Y = C, HY = H C; residual R = HY - Y (Y^T HY); Z = -K R made
// orthogonal to Y and orthonormal (gram); H Z by a second energy(); the
// 2n x 2n matrix of H on span(Y, Z) (lower blocks Y^T HY, Z^T HY, Z^T HZ)
// diagonalised by syevd; C <- Y q_Y + Z q_Z for the lowest n eigenvectors.
// The products are FP64 in both precisions.
void jd_update(Context& ctx) {
  ProfScope ps(ctx, "jd_update");
  const int n = ctx.nst, K = 2 * ctx.wb.ng, n2 = 2 * n;
  const double one = 1.0, two = 2.0, zero = 0.0, mone = -1.0;
  double* Y = ctx.d_c_last;
  double* HY = ctx.d_dc_last;
  double* A = ctx.d_nn;
  const size_t wf = (size_t)K * n;
  if (!ctx.d_jd_h) {
    ctx.d_jd_h = dalloc<double>((size_t)n2 * n2);
    ctx.d_jd_w = dalloc<double>(n2);
    QBX_SOLVER(cusolverDnDsyevd_bufferSize(ctx.solver, CUSOLVER_EIG_MODE_VECTOR,
                                           CUBLAS_FILL_MODE_LOWER, n2, ctx.d_jd_h, n2,
                                           ctx.d_jd_w, &ctx.jd_lwork));
    ctx.d_jd_work = dalloc<double>(std::max(1, ctx.jd_lwork));
  }
  QBX_CUDA(cudaMemcpyAsync(Y, ctx.d_c, wf * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
  QBX_CUDA(cudaMemcpyAsync(HY, ctx.d_hc, wf * sizeof(double), cudaMemcpyDeviceToDevice,
                           ctx.stream));
  // residual in HC
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, Y, K, HY, K, &zero, A, n));
  launch_rank1_fix(ctx, A, n, Y, K, HY, K, n, n, -1.0, false);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &mone, Y, K, A, n, &one,
                       ctx.d_hc, K));
  launch_precond_update(ctx);                       // kinetic energies of Y
  launch_precondition_into(ctx, ctx.d_hc, ctx.d_c); // Z = -K R
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, Y, K, ctx.d_c, K, &zero,
                       A, n));
  launch_rank1_fix(ctx, A, n, Y, K, ctx.d_c, K, n, n, -1.0, false);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &mone, Y, K, A, n, &one,
                       ctx.d_c, K));
  gram(ctx);
  energy(ctx, true, false);                         // H Z into HC
  double* H = ctx.d_jd_h;
  QBX_CUDA(cudaMemsetAsync(H, 0, sizeof(double) * (size_t)n2 * n2, ctx.stream));
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, Y, K, HY, K, &zero, H,
                       n2));
  launch_rank1_fix(ctx, H, n2, Y, K, HY, K, n, n, -1.0, false);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, ctx.d_c, K, HY, K, &zero,
                       H + n, n2));
  launch_rank1_fix(ctx, H + n, n2, ctx.d_c, K, HY, K, n, n, -1.0, false);
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, K, &two, ctx.d_c, K, ctx.d_hc, K,
                       &zero, H + n + (size_t)n * n2, n2));
  launch_rank1_fix(ctx, H + n + (size_t)n * n2, n2, ctx.d_c, K, ctx.d_hc, K, n, n, -1.0, false);
  QBX_SOLVER(cusolverDnDsyevd(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n2, H,
                              n2, ctx.d_jd_w, ctx.d_jd_work, ctx.jd_lwork, ctx.d_info));
  // C = Y q[0:n, 0:n] + Z q[n:2n, 0:n]
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &one, ctx.d_c, K, H + n, n2,
                       &zero, ctx.d_hc, K));
  QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &one, Y, K, H, n2, &one,
                       ctx.d_hc, K));
  QBX_CUDA(cudaMemcpyAsync(ctx.d_c, ctx.d_hc, wf * sizeof(double), cudaMemcpyDeviceToDevice,
                           ctx.stream));
  int info = 0;
  QBX_CUDA(cudaMemcpyAsync(&info, ctx.d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  QBX_CUDA(cudaStreamSynchronize(ctx.stream));
  QBX_REQUIRE(info == 0, 41, "syevd of the JD projected Hamiltonian failed (info=" +
                                 std::to_string(info) + ")");
  ctx.extrapolate = false;
}

void free_mixed(Context& ctx) {
  void** bufs[] = {&ctx.d_acc32, &ctx.cs_hi[0], &ctx.cs_lo[0], &ctx.cs_hi[1], &ctx.cs_lo[1],
                   &ctx.hs_hi, &ctx.hs_lo, &ctx.as_hi, &ctx.as_lo, &ctx.ss_hi, &ctx.ss_lo,
                   &ctx.d_tc_ws};
  for (void** b : bufs)
    if (*b) { cudaFree(*b); *b = nullptr; }
  dfree(ctx.d_colred);
  ctx.colred_elems = 0;
  dfree(ctx.c32);
  dfree(ctx.c32lo);
  dfree(ctx.a32);
  dfree(ctx.a32lo);
  dfree(ctx.s32);
  dfree(ctx.s32lo);
  void** tall[] = {&ctx.at_hi, &ctx.at_lo, &ctx.ct_hi, &ctx.ct_lo, &ctx.tm_hi, &ctx.tm_lo};
  for (void** b : tall)
    if (*b) { cudaFree(*b); *b = nullptr; }
  ctx.acc32_elems = 0;
  ctx.tc_ws_elems = 0;
}

// Buffers of the split-precision products; the projector split is rebuilt
// whenever the projectors change.
void alloc_mixed(Context& ctx) {
  free_mixed(ctx);
  if (ctx.precision != MIXED || !ctx.have_cell) return;
  const size_t K = 2 * (size_t)ctx.wb.ng, n = ctx.nst, np = ctx.nproj;
  ctx.ldp = (int)((K + 63) / 64 * 64);
  const size_t wf = (size_t)ctx.ldp * n;
  const size_t small = std::max(np * n, n * n);
  ctx.acc32_elems = std::max(wf, std::max(np * n, std::max(K * np, n * n)));
  QBX_CUDA(cudaMalloc(&ctx.d_acc32, ctx.acc32_elems * sizeof(float)));
  ctx.colred_elems = 129 * n;   // up to two partial arrays of 64 per column, then one total
  ctx.d_colred = dalloc<double>(ctx.colred_elems);
  for (int s = 0; s < 2; s++) {
    QBX_CUDA(cudaMalloc(&ctx.cs_hi[s], wf * 2));
    QBX_CUDA(cudaMalloc(&ctx.cs_lo[s], wf * 2));
  }
  QBX_CUDA(cudaMalloc(&ctx.hs_hi, wf * 2));
  QBX_CUDA(cudaMalloc(&ctx.hs_lo, wf * 2));
  QBX_CUDA(cudaMalloc(&ctx.ss_hi, std::max<size_t>(small, 1) * 2));
  QBX_CUDA(cudaMalloc(&ctx.ss_lo, std::max<size_t>(small, 1) * 2));
  // TF32 splits for the cuBLAS products: only with that backend
  const bool cublas_tf32 = ctx.gemm_backend == 0;
  if (cublas_tf32) {
    ctx.c32 = dalloc<float>((size_t)ctx.ldp * n);
    ctx.c32lo = dalloc<float>((size_t)ctx.ldp * n);
    const size_t small4 = std::max<size_t>((size_t)pad4((int)std::max(np, n)) * n, 1);
    ctx.s32 = dalloc<float>(small4);
    ctx.s32lo = dalloc<float>(small4);
  }
  // tall-update splits: room for either kind (TF32 4 bytes at ld pad4,
  // BF16 2 bytes at ld pad8)
  auto tall_bytes = [](size_t rows, size_t cols) { return (size_t)pad8((int)rows) * cols * 4; };
  // ct holds the transposed split of a wavefunction block, or its plain
  // split (ld ldp) for the MN-major tall updates
  const size_t ct_bytes = std::max(tall_bytes(n, K), (size_t)ctx.ldp * n * 4);
  QBX_CUDA(cudaMalloc(&ctx.ct_hi, ct_bytes));
  QBX_CUDA(cudaMalloc(&ctx.ct_lo, ct_bytes));
  QBX_CUDA(cudaMalloc(&ctx.tm_hi, tall_bytes(std::max(np, n), n)));
  QBX_CUDA(cudaMalloc(&ctx.tm_lo, tall_bytes(std::max(np, n), n)));
  if (np) {
    QBX_CUDA(cudaMalloc(&ctx.as_hi, (size_t)ctx.ldp * np * 2));
    QBX_CUDA(cudaMalloc(&ctx.as_lo, (size_t)ctx.ldp * np * 2));
    if (cublas_tf32) {
      ctx.a32 = dalloc<float>((size_t)ctx.ldp * np);
      ctx.a32lo = dalloc<float>((size_t)ctx.ldp * np);
    }
    QBX_CUDA(cudaMalloc(&ctx.at_hi, tall_bytes(np, K)));
    QBX_CUDA(cudaMalloc(&ctx.at_lo, tall_bytes(np, K)));
    split_projectors(ctx);
  }
  QBX_CUDA(cudaStreamSynchronize(ctx.stream));
}

// The split copies of the projectors A_nl (BF16 hi/lo for F = 2 A^T C,
// TF32 hi/lo for the cuBLAS fallback, the transposed split of the H*C
// update), rebuilt in place whenever the projectors change.
void split_projectors(Context& ctx) {
  if (ctx.precision != MIXED || !ctx.d_anl || !ctx.nproj) return;
  const int K = 2 * ctx.wb.ng, np = ctx.nproj;
  split_bf16_2d(ctx, ctx.d_anl, K, np, K, ctx.as_hi, ctx.as_lo, ctx.ldp);
  if (ctx.a32) split_tf32(ctx, ctx.d_anl, K, np, K, ctx.a32, ctx.a32lo, ctx.ldp);
  split_t(ctx, ctx.tall_kind_hc, ctx.d_anl, K, np, K, ctx.at_hi, ctx.at_lo,
          Context::tall_ld_of(ctx.tall_kind_hc, np));
}

}  // namespace qbx
