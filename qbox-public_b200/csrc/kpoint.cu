// The electronic step on k points off Gamma.  Each k point is a complex
// SlaterDet (src/SlaterDet.cpp, the !basis_->real() branches): one band per
// FFT through the stick kernels of fft.cu, inner products C^H C as ZGEMM /
// ZHERK, and the k-weighted sums of ChargeDensity::update_density
// (src/ChargeDensity.cpp:136-198), EnergyFunctional::energy
// (src/EnergyFunctional.cpp:440-560, 700-716) and Wavefunction::dot
// (src/Wavefunction.cpp:814-830).  The density, the potentials and the
// Coulomb and XC energies are the Gamma machinery: the density grid and its
// basis do not depend on k.
//
// Arithmetic is FP64 throughout (cuBLAS Z routines, cuSOLVER zpotrf/zgetrf,
// the FP64 stick and plane FFT kernels), whatever the context's precision.
// Coefficients are ngw x nst complex, column-major, in the sorted Miller
// order of the k point's basis (build_kbasis).
#include <cmath>
#include <vector>

#include "qbx.h"
#include "qbx_internal.h"
#include "reduce.cuh"

namespace qbx {

using namespace red;

namespace {

int nblk(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

const cuDoubleComplex kOne = {1.0, 0.0}, kZero = {0.0, 0.0}, kMone = {-1.0, 0.0};

cuDoubleComplex* zc(double* p) { return reinterpret_cast<cuDoubleComplex*>(p); }
const cuDoubleComplex* zc(const double* p) { return reinterpret_cast<const cuDoubleComplex*>(p); }

void free_kp(KPointSet& kp) {
  free_sticks(kp.dks);
  double** bufs[] = {&kp.d_c, &kp.d_hc, &kp.d_c_last, &kp.d_dc_last, &kp.d_ctmp, &kp.d_g2,
                     &kp.d_q, &kp.d_twnl, &kp.d_anl, &kp.d_w2, &kp.d_prec};
  for (double** b : bufs) dfree(*b);
  kp.anl_ready = false;
}

double* znn(Context& ctx, int i) { return ctx.d_znn + 2 * (size_t)i * ctx.nst * ctx.nst; }

// ---------------------------------------------------------------- sums
// E_kin of one k point: sum_n occ_n sum_G 1/2 |k+G|^2 |c|^2
// (src/EnergyFunctional.cpp:455-492, fac = 0.5 on a complex basis)
struct EkinKF {
  const double2* c; const double* g2; const double* occ; int ngw;
  __device__ void operator()(size_t i, double* a) const {
    const int n = (int)(i / ngw), ig = (int)(i - (size_t)n * ngw);
    const double2 v = c[i];
    a[0] += 0.5 * occ[n] * (v.x * v.x + v.y * v.y) * g2[ig];
  }
};

// E_nl of one k point: sum occ_n D_p |F_pn|^2 / Omega
// (src/NonLocalPotential.cpp:1574-1597, complex branch)
struct EnlKF {
  const double2* f; const double* dfac; const double* occ; int np; double om_inv;
  __device__ void operator()(size_t i, double* a) const {
    const int p = (int)(i % np), n = (int)(i / np);
    const double2 v = f[i];
    a[0] += occ[n] * dfac[p] * (v.x * v.x + v.y * v.y) * om_inv;
  }
};

// Re tr(C^H HC) (SlaterDet::dot, complex branch, src/SlaterDet.cpp:1149-1152)
struct EigKF {
  const double2* c; const double2* hc;
  __device__ void operator()(size_t i, double* a) const {
    const double2 x = c[i], y = hc[i];
    a[0] += x.x * y.x + x.y * y.y;
  }
};

// the Anderson sums a = F.(F - F_last), b = |F - F_last|^2 over every real
// component (src/PSDAWavefunctionStepper.cpp:122-135, complex branch)
struct AndersonKF {
  const double* f; const double* flast;
  __device__ void operator()(size_t i, double* a) const {
    const double v = f[i], d = v - flast[i];
    a[0] += v * d;
    a[1] += d * d;
  }
};

__global__ void k_fnl_scale_c(double2* f, const double* dfac, int np, size_t n, double om_inv) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double s = dfac[i % np] * om_inv;
    f[i].x *= s;
    f[i].y *= s;
  }
}

// Preconditioner::update on a complex basis (src/Preconditioner.cpp:88-143):
// ekin_n = (sum |c|^2 |k+G|^2) / (2 (sum |c|^2 - |c_first|^2 / 2)); the
// reference removes half of the first local coefficient from the norm on
// every basis (its G = 0 correction), here rod (0,0)'s first.  One CTA per band.
__global__ void k_prec_k(const double2* __restrict__ c, const double* __restrict__ g2, int ngw,
                         int first, double* __restrict__ ekin) {
  __shared__ double sh[32];
  const int n = blockIdx.x;
  const double2* cn = c + (size_t)n * ngw;
  double sn = 0.0, se = 0.0;
  for (int i = threadIdx.x; i < ngw; i += blockDim.x) {
    const double p = cn[i].x * cn[i].x + cn[i].y * cn[i].y;
    sn += p;
    se += p * g2[i];
  }
  const double tn = block_sum(sn, sh);
  __syncthreads();
  const double te = block_sum(se, sh);
  if (threadIdx.x == 0) {
    const double p0 = cn[first].x * cn[first].x + cn[first].y * cn[first].y;
    const double bn = tn - 0.5 * p0;
    ekin[n] = (0.5 * bn > 0.0) ? 0.5 * te / bn : 0.0;
  }
}

// dc = -K (HC - C A) in place (src/PSDAWavefunctionStepper.cpp:90-110 with
// Preconditioner::diag, src/Preconditioner.cpp:49-85, ecutprec = 0)
__global__ void k_precondition_k(double2* __restrict__ hc, const double* __restrict__ g2,
                                 const double* __restrict__ ekin, int ngw, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / ngw), ig = (int)(i - (size_t)b * ngw);
    double en = ekin[b];
    if (en == 0.0) en = 1.0;
    const double e = 0.5 * g2[ig];
    const double f = (e < en) ? 0.5 / en : 0.5 / e;
    hc[i].x *= -f;
    hc[i].y *= -f;
  }
}

// x <- x + theta (x - x_last) + f + theta (f - f_last); x_last <- x;
// f_last <- f, with theta from the sums in ab (or 0 without extrapolation)
// (src/PSDAWavefunctionStepper.cpp:112-190)
__global__ void k_psda_apply_k(double* __restrict__ x, double* __restrict__ xlast,
                               const double* __restrict__ f, double* __restrict__ flast, size_t n,
                               const double* __restrict__ ab, int extrapolate,
                               double* __restrict__ theta_out) {
  double theta = 0.0;
  if (extrapolate) {
    const double a = ab[0], b = ab[1];
    if (b != 0.0) theta = -a / b;
    if (theta < -1.0) theta = 0.0;
    theta = fmin(2.0, theta);
  }
  if (theta_out && blockIdx.x == 0 && threadIdx.x == 0) *theta_out = theta;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double xv = x[i], fv = f[i];
    if (extrapolate) {
      x[i] = xv + theta * (xv - xlast[i]) + fv + theta * (fv - flast[i]);
    } else {
      x[i] = xv + fv;
    }
    xlast[i] = xv;
    flast[i] = fv;
  }
}

// m <- alpha I + beta m (n x n complex)
__global__ void k_zaxpy_identity(double2* m, int n, double alpha, double beta) {
  const size_t nn = (size_t)n * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % n), col = (int)(i / n);
    double2 v = m[i];
    v.x *= beta;
    v.y *= beta;
    if (r == col) v.x += alpha;
    m[i] = v;
  }
}

// x <- (x + t) / 2
__global__ void k_zaverage(double2* x, const double2* t, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = make_double2(0.5 * (x[i].x + t[i].x), 0.5 * (x[i].y + t[i].y));
}

void ensure_zwork(Context& ctx) {
  if (ctx.d_zwork) return;
  const int n = ctx.nst;
  int l1 = 0, l2 = 0;
  QBX_SOLVER(cusolverDnZpotrf_bufferSize(ctx.solver, CUBLAS_FILL_MODE_LOWER, n, zc(znn(ctx, 0)), n,
                                         &l1));
  QBX_SOLVER(cusolverDnZgetrf_bufferSize(ctx.solver, n, n, zc(znn(ctx, 0)), n, &l2));
  ctx.zwork_len = std::max(1, std::max(l1, l2));
  ctx.d_zwork = dalloc<double>(2 * (size_t)ctx.zwork_len);
  QBX_CUDA(cudaMalloc(&ctx.d_zipiv, sizeof(int) * (n + 1)));
}

// S = C^H C = L L^H into znn(0) (lower triangle), Cholesky on the device; its
// info code goes to the status word `status`, checked when the step's
// scalars are read back (no host read inside a step)
void overlap_cholesky_k(Context& ctx, const double* c, int ngw, int status) {
  const int n = ctx.nst;
  const double one = 1.0, zero = 0.0;
  double* L = znn(ctx, 0);
  QBX_BLAS(cublasZherk(ctx.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, n, ngw, &one, zc(c), ngw,
                       &zero, zc(L), n));
  QBX_SOLVER(cusolverDnZpotrf(ctx.solver, CUBLAS_FILL_MODE_LOWER, n, zc(L), n, zc(ctx.d_zwork),
                              ctx.zwork_len, ctx.d_status + status));
}

// t = P I for the row interchanges of an LU factorisation (ipiv 1-based,
// applied in order), one thread per column, complex
__global__ void k_zpivoted_identity(double2* __restrict__ t, const int* __restrict__ ipiv, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double2* col = t + (size_t)j * n;
  for (int i = 0; i < n; i++) col[i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  for (int i = 0; i < n; i++) {
    const int p = ipiv[i] - 1;
    if (p != i && p >= 0 && p < n) {
      const double2 a = col[i];
      col[i] = col[p];
      col[p] = a;
    }
  }
}

// ComplexMatrix::polar (src/Matrix.cpp:2524-2595): Bjorck-Bowie steps while
// ||I - X^H X||_F < 1, else the Higham step X <- (X + X^-H) / 2 (X^-H with
// the conjugated diagonal, as the ScaLAPACK build's pztranc gives it).
// q = I - X^H X and SLOT_FROB = ||q||_F^2
static void polar_q_k(Context& ctx, const double* x, double* q) {
  const int n = ctx.nst;
  const size_t nn = (size_t)n * n;
  QBX_CUDA(cudaMemsetAsync(q, 0, 2 * nn * sizeof(double), ctx.stream));
  k_zaxpy_identity<<<nblk(nn), 256, 0, ctx.stream>>>((double2*)q, n, 1.0, 0.0);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_C, CUBLAS_OP_N, n, n, n, &kMone, zc(x), n, zc(x), n,
                       &kOne, zc(q), n));
  launch_sumsq(ctx, q, 2 * nn, SLOT_FROB);
}

// x <- x (I + q/2 (I + 3q/4))
static void polar_bjorck_k(Context& ctx, double* x, const double* q, double* t, double* qt,
                           double* xp) {
  const int n = ctx.nst;
  const size_t nn = (size_t)n * n;
  QBX_CUDA(cudaMemcpyAsync(t, q, 2 * nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
  k_zaxpy_identity<<<nblk(nn), 256, 0, ctx.stream>>>((double2*)t, n, 1.0, 0.75);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &kOne, zc(q), n, zc(t), n,
                       &kZero, zc(qt), n));
  k_zaxpy_identity<<<nblk(nn), 256, 0, ctx.stream>>>((double2*)qt, n, 1.0, 0.5);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &kOne, zc(x), n, zc(qt), n,
                       &kZero, zc(xp), n));
  QBX_CUDA(cudaMemcpyAsync(x, xp, 2 * nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
}

// x <- (x + x^-H)/2: x^-H by an LU factorisation of x^H (P x^H = L U) and the
// two triangular solves of U^-1 L^-1 P (getrs would allocate stream-ordered
// memory at some sizes, which a conditional graph body cannot hold)
static void polar_higham_k(Context& ctx, double* x, double* t, double* qt) {
  const int n = ctx.nst;
  const size_t nn = (size_t)n * n;
  QBX_BLAS(cublasZgeam(ctx.blas, CUBLAS_OP_C, CUBLAS_OP_N, n, n, &kOne, zc(x), n, &kZero, zc(x), n,
                       zc(t), n));
  QBX_SOLVER(cusolverDnZgetrf(ctx.solver, n, n, zc(t), n, zc(ctx.d_zwork), ctx.d_zipiv,
                              ctx.d_status + ST_INFO_POLAR));
  k_zpivoted_identity<<<(n + 127) / 128, 128, 0, ctx.stream>>>((double2*)qt, ctx.d_zipiv, n);
  QBX_LAUNCHED(ctx);
  QBX_BLAS(cublasZtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                       CUBLAS_DIAG_UNIT, n, n, &kOne, zc(t), n, zc(qt), n));
  QBX_BLAS(cublasZtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                       CUBLAS_DIAG_NON_UNIT, n, n, &kOne, zc(t), n, zc(qt), n));
  k_zaverage<<<nblk(nn), 256, 0, ctx.stream>>>((double2*)x, (const double2*)qt, nn);
  QBX_LAUNCHED(ctx);
}

// Eagerly the norm is read back after each q; inside a captured step the
// loop is a WHILE conditional node whose body decides on the device and runs
// the chosen step in an IF/ELSE node, as the Gamma polar does.
void polar_k(Context& ctx, double* x, double tol, int maxiter) {
  double* q = znn(ctx, 2);
  double* t = znn(ctx, 3);
  double* qt = znn(ctx, 4);
  double* xp = znn(ctx, 5);
  if (!ctx.capturing) {
    for (int iter = 0; iter < maxiter; iter++) {
      polar_q_k(ctx, x, q);
      const double qn = std::sqrt(read_slot(ctx, SLOT_FROB));
      if (qn < 1.0) polar_bjorck_k(ctx, x, q, t, qt, xp);
      else polar_higham_k(ctx, x, t, qt);
      if (qn <= tol) break;
    }
    return;
  }
  int* iters = ctx.d_status + ST_POLAR_ITERS;
  QBX_CUDA(cudaMemsetAsync(iters, 0, sizeof(int), ctx.stream));
  cudaGraphConditionalHandle loop;
  QBX_CUDA(cudaGraphConditionalHandleCreate(&loop, capture_graph(ctx.stream), 1,
                                            cudaGraphCondAssignDefault));
  cudaGraph_t body = add_conditional(ctx.stream, loop, cudaGraphCondTypeWhile, 1)[0];
  capture_body(ctx, body, ctx.side[0], [&]() {
    polar_q_k(ctx, x, q);
    cudaGraphConditionalHandle branch;
    QBX_CUDA(cudaGraphConditionalHandleCreate(&branch, capture_graph(ctx.stream), 0, 0));
    launch_polar_decide(ctx, tol, maxiter, iters, loop, branch);
    cudaGraph_t* arms = add_conditional(ctx.stream, branch, cudaGraphCondTypeIf, 2);
    cudaGraph_t bjorck = arms[0], higham = arms[1];
    capture_body(ctx, bjorck, ctx.side[1], [&]() { polar_bjorck_k(ctx, x, q, t, qt, xp); });
    capture_body(ctx, higham, ctx.side[1], [&]() { polar_higham_k(ctx, x, t, qt); });
  });
}

// SlaterDet::ortho_align, complex branch (src/SlaterDet.cpp:877-975)
void ortho_align_k(Context& ctx, KPointSet& kp) {
  ProfScope ps(ctx, "ortho_align_k");
  const int n = ctx.nst, K = kp.kb.ng;
  double* L = znn(ctx, 0);
  double* X = znn(ctx, 1);
  overlap_cholesky_k(ctx, kp.d_c, K, ST_INFO_ORTHO);
  QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_C, CUBLAS_OP_N, n, n, K, &kOne, zc(kp.d_c), K,
                       zc(kp.d_c_last), K, &kZero, zc(X), n));
  QBX_BLAS(cublasZtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                       CUBLAS_DIAG_NON_UNIT, n, n, &kOne, zc(L), n, zc(X), n));
  polar_k(ctx, X, 1.e-6, 20);
  QBX_BLAS(cublasZtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C,
                       CUBLAS_DIAG_NON_UNIT, n, n, &kOne, zc(L), n, zc(X), n));
  const size_t sz = 2 * (size_t)K * n * sizeof(double);
  QBX_CUDA(cudaMemcpyAsync(kp.d_ctmp, kp.d_c, sz, cudaMemcpyDeviceToDevice, ctx.stream));
  QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &kOne, zc(kp.d_ctmp), K,
                       zc(X), n, &kZero, zc(kp.d_c), K));
}

void ensure_anl(Context& ctx, KPointSet& kp) {
  if (kp.anl_ready || ctx.nproj == 0) return;
  const int ngw = kp.kb.ng;
  if (!kp.d_twnl) {
    const std::vector<double> tw = twnl_rows(ctx, kp.kb);
    kp.d_twnl = dupload(tw);
  }
  if (!kp.d_anl) kp.d_anl = dalloc<double>(2 * (size_t)ngw * ctx.nproj);
  build_anl(ctx, kp.d_q, ngw, kp.d_twnl, kp.d_anl);
  if (!ctx.d_fnlk) ctx.d_fnlk = dalloc<double>(2 * (size_t)ctx.nproj * ctx.nst);
  kp.anl_ready = true;
}

}  // namespace

void free_kpoints(Context& ctx) {
  for (KPointSet& kp : ctx.kpts) free_kp(kp);
  ctx.kpts.clear();
  dfree(ctx.d_fnlk);
  dfree(ctx.d_znn);
  dfree(ctx.d_zwork);
  if (ctx.d_zipiv) { cudaFree(ctx.d_zipiv); ctx.d_zipiv = nullptr; }
  ctx.zwork_len = 0;
  ctx.kpts_extrapolate = false;
}

void kpoints_atoms_changed(Context& ctx) {
  for (KPointSet& kp : ctx.kpts) {
    kp.anl_ready = false;
    dfree(kp.d_anl);
    dfree(kp.d_twnl);
  }
  dfree(ctx.d_fnlk);
}

// Wavefunction::add_kpoint for each k point, the Gamma point removed
// (src/Wavefunction.cpp:400-485): a complex basis per k point on the
// wavefunction grid, its coefficients zero until set.
void set_kpoints(Context& ctx, int nk, const double* k, const double* w) {
  // arguments first, so that a refused set leaves the context as it was
  for (int i = 0; i < nk; i++) {
    const double* ki = k + 3 * i;
    QBX_REQUIRE(std::fabs(ki[0]) + std::fabs(ki[1]) + std::fabs(ki[2]) > 0.0, 1,
                "the Gamma point is the real basis: give only k points off Gamma");
    QBX_REQUIRE(w[i] >= 0.0, 1, "negative k point weight");
    for (int j = 0; j < i; j++) {
      const double* kj = k + 3 * j;
      const double d = std::fabs(kj[0] - ki[0]) + std::fabs(kj[1] - ki[1]) + std::fabs(kj[2] - ki[2]);
      QBX_REQUIRE(d > 1e-6, 1, "k point already defined");
    }
  }
  free_kpoints(ctx);
  if (nk == 0) return;
  const int n = ctx.nst;
  ctx.kpts.resize(nk);
  for (int i = 0; i < nk; i++) {
    KPointSet& kp = ctx.kpts[i];
    for (int a = 0; a < 3; a++) kp.k[a] = k[3 * i + a];
    kp.weight = w[i];
    build_kbasis(kp.kb, ctx.wb.cell, ctx.wb.ecut, kp.k);
    set_grid_complex(kp.kb, ctx.wb.n0, ctx.wb.n1, ctx.wb.n2);
    upload_sticks(kp.dks, kp.kb);
    const size_t sz = 2 * (size_t)kp.kb.ng * n;
    kp.d_c = dalloc<double>(sz);
    kp.d_hc = dalloc<double>(sz);
    kp.d_c_last = dalloc<double>(sz);
    kp.d_dc_last = dalloc<double>(sz);
    kp.d_ctmp = dalloc<double>(sz);
    QBX_CUDA(cudaMemset(kp.d_c, 0, sz * sizeof(double)));
    QBX_CUDA(cudaMemset(kp.d_hc, 0, sz * sizeof(double)));
    kp.d_g2 = dupload(kp.kb.g2);
    kp.d_q = dupload(kp.kb.gx);
    std::vector<double> w2(2 * n);
    for (int b = 0; b < n; b++) w2[2 * b] = w2[2 * b + 1] = kp.weight * ctx.occ[b] / ctx.wb.omega;
    kp.d_w2 = dupload(w2);
    kp.d_prec = dalloc<double>(n);
  }
  ctx.d_znn = dalloc<double>(6 * 2 * (size_t)n * n);
  ensure_zwork(ctx);
}

// SlaterDet::gram, complex branch (src/SlaterDet.cpp:524-533): C <- C L^-H
void gram_k(Context& ctx) {
  const int n = ctx.nst;
  for (KPointSet& kp : ctx.kpts) {
    const int K = kp.kb.ng;
    overlap_cholesky_k(ctx, kp.d_c, K, ST_INFO_GRAM);
    QBX_BLAS(cublasZtrsm(ctx.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C,
                         CUBLAS_DIAG_NON_UNIT, K, n, &kOne, zc(znn(ctx, 0)), n, zc(kp.d_c), K));
  }
}

// ChargeDensity::update_density over the k points (weights wk occ / Omega)
void update_density_k(Context& ctx) {
  ProfScope ps(ctx, "update_density");
  QBX_CUDA(cudaMemsetAsync(ctx.d_rhor, 0, ctx.N() * sizeof(double), ctx.stream));
  for (KPointSet& kp : ctx.kpts) launch_density_k(ctx, kp, ctx.d_rhor);
  launch_sum(ctx, ctx.d_rhor, ctx.N(), SLOT_CHARGE);
  vb_forward_real(ctx, ctx.d_rhor, ctx.vb.omega, ctx.d_rhog);
}

// EnergyFunctional::energy over the k points: E_kin and E_nl weighted by
// wk into their slots; with hpsi, HC = 1/2 |k+G|^2 C + V psi + A D F / Omega
// per k point (NonLocalPotential::energy, src/NonLocalPotential.cpp:1420-1640,
// complex branch: F = A^H C by ZGEMM, HC += A F by ZGEMM)
void energy_k(Context& ctx, bool hpsi) {
  ProfScope ps(ctx, "energy");
  const int n = ctx.nst, np = ctx.nproj;
  QBX_CUDA(cudaMemsetAsync(ctx.d_scalars + SLOT_EKIN, 0, sizeof(double), ctx.stream));
  QBX_CUDA(cudaMemsetAsync(ctx.d_scalars + SLOT_ENL, 0, sizeof(double), ctx.stream));
  for (KPointSet& kp : ctx.kpts) {
    const int K = kp.kb.ng;
    reduce_acc<1>(ctx, EkinKF{(const double2*)kp.d_c, kp.d_g2, ctx.d_occ, K}, (size_t)K * n,
                  SLOT_EKIN, kp.weight);
    if (hpsi) launch_vpsi_k(ctx, kp, ctx.d_vr);
    if (np == 0) continue;
    ensure_anl(ctx, kp);
    ProfScope pn(ctx, "nonlocal_k");
    QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_C, CUBLAS_OP_N, np, n, K, &kOne, zc(kp.d_anl), K,
                         zc(kp.d_c), K, &kZero, zc(ctx.d_fnlk), np));
    const double om_inv = 1.0 / ctx.wb.omega;
    reduce_acc<1>(ctx, EnlKF{(const double2*)ctx.d_fnlk, ctx.d_pdfac, ctx.d_occ, np, om_inv},
                  (size_t)np * n, SLOT_ENL, kp.weight);
    if (hpsi) {
      k_fnl_scale_c<<<nblk((size_t)np * n), 256, 0, ctx.stream>>>((double2*)ctx.d_fnlk,
                                                                   ctx.d_pdfac, np,
                                                                   (size_t)np * n, om_inv);
      QBX_LAUNCHED(ctx);
      QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, np, &kOne, zc(kp.d_anl), K,
                           zc(ctx.d_fnlk), np, &kOne, zc(kp.d_hc), K));
    }
  }
}

// Wavefunction::dot(dwf): sum_k wk Re tr(C^H HC)
void eigsum_k(Context& ctx) {
  QBX_CUDA(cudaMemsetAsync(ctx.d_scalars + SLOT_EIG, 0, sizeof(double), ctx.stream));
  for (KPointSet& kp : ctx.kpts)
    reduce_acc<1>(ctx, EigKF{(const double2*)kp.d_c, (const double2*)kp.d_hc},
                  (size_t)kp.kb.ng * ctx.nst, SLOT_EIG, kp.weight);
}

// PSDAWavefunctionStepper::update, complex branch, per k point
// (src/PSDAWavefunctionStepper.cpp:46-249): A = C^H HC, HC <- HC - C A,
// preconditioning, Anderson extrapolation with the k point's own theta,
// ortho_align.  The first k point's theta goes to the theta slot.
void psda_update_k(Context& ctx) {
  ProfScope ps(ctx, "psda_update");
  const int n = ctx.nst;
  for (size_t ik = 0; ik < ctx.kpts.size(); ik++) {
    KPointSet& kp = ctx.kpts[ik];
    const int K = kp.kb.ng;
    const size_t len = 2 * (size_t)K * n;
    double* A = znn(ctx, 1);
    QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_C, CUBLAS_OP_N, n, n, K, &kOne, zc(kp.d_c), K,
                         zc(kp.d_hc), K, &kZero, zc(A), n));
    QBX_BLAS(cublasZgemm(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, K, n, n, &kMone, zc(kp.d_c), K, zc(A),
                         n, &kOne, zc(kp.d_hc), K));
    k_prec_k<<<n, 256, 0, ctx.stream>>>((const double2*)kp.d_c, kp.d_g2, K, kp.kb.first,
                                        kp.d_prec);
    QBX_LAUNCHED(ctx);
    k_precondition_k<<<nblk(len / 2), 256, 0, ctx.stream>>>((double2*)kp.d_hc, kp.d_g2,
                                                            kp.d_prec, K, len / 2);
    QBX_LAUNCHED(ctx);
    if (ctx.kpts_extrapolate)
      reduce<2>(ctx, AndersonKF{kp.d_hc, kp.d_dc_last}, len, SLOT_SCRATCH);
    k_psda_apply_k<<<nblk(len), 256, 0, ctx.stream>>>(
        kp.d_c, kp.d_c_last, kp.d_hc, kp.d_dc_last, len, ctx.d_scalars + SLOT_SCRATCH,
        ctx.kpts_extrapolate ? 1 : 0, ik == 0 ? ctx.d_scalars + SLOT_THETA : nullptr);
    QBX_LAUNCHED(ctx);
    ortho_align_k(ctx, kp);
  }
  ctx.kpts_extrapolate = true;
}

}  // namespace qbx
