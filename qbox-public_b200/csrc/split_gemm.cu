// Split-precision GEMMs of the mixed path.
//
// An FP64 operand x is written as x = hi + lo with hi = bf16(x) and
// lo = bf16(x - hi) (about 16 significant bits together).  A product is then
// formed from three BF16 tensor-core products accumulated in FP32,
//     A B  ~  A_hi B_hi + A_hi B_lo + A_lo B_hi,
// whose relative error is ~2^-16 per term and random in sign, so inner
// products over the 145 838 plane-wave rows keep ~1e-8 absolute accuracy off
// the diagonal.  On the diagonal of C^T C the dropped A_lo B_lo term has a
// fixed sign; the overlap matrix therefore gets its diagonal from an FP64
// reduction (|c_n|^2 summed exactly) before the FP64 Cholesky.
//
// The products themselves run through GemmBackend: cuBLAS BF16 GEMMs with
// FP32 output here, or the library's own tcgen05 kernel (tc_gemm.cu).
#include <algorithm>

#include "qbx_internal.h"
#include "reduce.cuh"
#include "split.cuh"

namespace qbx {

__global__ void k_split_bf16(const double* __restrict__ x, size_t n, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[i] = h;
    lo[i] = __double2bfloat16(v - (double)__bfloat162float(h));
  }
}

// out = alpha * acc + beta * out  (column-major, both ld = m)
__global__ void k_acc_to_f64(const float* __restrict__ acc, size_t n, double alpha, double beta,
                             double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = alpha * (double)acc[i] + (beta != 0.0 ? beta * out[i] : 0.0);
}

// diag(S)_n = 2 sum_G |c_n(G)|^2 - c_n(0)^2 in FP64 (one CTA per band)
__global__ void k_diag_overlap(const double* __restrict__ c, int K, int n, double* __restrict__ S) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  const double* p = c + (size_t)b * K;
  double s = 0.0;
  for (int i = threadIdx.x; i < K; i += blockDim.x) s += p[i] * p[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    S[b + (size_t)b * n] = 2.0 * t - p[0] * p[0];
  }
}

static int nblocks(size_t n) {
  return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 32));
}

// column-major rows x cols (ld ldx) -> hi/lo with leading dimension ldp >=
// rows; the padding rows are zero
__global__ void k_split_bf16_2d(const double* __restrict__ x, int rows, int cols, int ldx,
                                __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                int ldp) {
  const size_t n = (size_t)ldp * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / ldp), r = (int)(t - (size_t)c * ldp);
    double v = 0.0;
    if (r < rows) v = x[(size_t)c * ldx + r];
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[t] = h;
    lo[t] = __double2bfloat16(v - (double)__bfloat162float(h));
  }
}


void split_bf16(Context& ctx, const double* x, size_t n, void* hi, void* lo) {
  k_split_bf16<<<nblocks(n), 256, 0, ctx.stream>>>(x, n, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo);
  QBX_LAUNCHED(ctx);
}

void overlap_diag_f64(Context& ctx, const double* c, int K, int n, double* S) {
  k_diag_overlap<<<n, 256, 0, ctx.stream>>>(c, K, n, S);
  QBX_LAUNCHED(ctx);
}

// D (m x n, FP32, ld m) = sum of the three split products of op(A) op(B),
// A and B given as hi/lo BF16 pairs.  ta/tb: true = transpose (the operand
// is stored K-major, i.e. column-major with ld = k).
static void cublas_split(Context& ctx, bool ta, bool tb, int m, int n, int k, const void* ahi,
                         const void* alo, int lda, const void* bhi, const void* blo, int ldb,
                         float* D) {
  const float one = 1.0f, zero = 0.0f;
  const cublasOperation_t oa = ta ? CUBLAS_OP_T : CUBLAS_OP_N;
  const cublasOperation_t ob = tb ? CUBLAS_OP_T : CUBLAS_OP_N;
  const void* as[3] = {ahi, ahi, alo};
  const void* bs[3] = {bhi, blo, bhi};
  for (int t = 0; t < 3; t++)
    QBX_BLAS(cublasGemmEx(ctx.blas, oa, ob, m, n, k, &one, as[t], CUDA_R_16BF, lda, bs[t],
                          CUDA_R_16BF, ldb, t == 0 ? &zero : &one, D, CUDA_R_32F, m,
                          CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
}

void split_gemm(Context& ctx, bool ta, bool tb, int m, int n, int k, double alpha,
                const void* ahi, const void* alo, int lda, const void* bhi, const void* blo,
                int ldb, double beta, double* C, bool lower) {
  if (ctx.gemm_backend == 1 && tc_gemm_supported(ctx, ta, tb, m, n, k)) {
    tc_split_gemm(ctx, ta, tb, m, n, k, alpha, ahi, alo, lda, bhi, blo, ldb, beta, C, lower);
    return;
  }
  float* D = (float*)ctx.d_acc32;
  QBX_REQUIRE((size_t)m * n <= ctx.acc32_elems, 50, "split GEMM accumulator too small");
  cublas_split(ctx, ta, tb, m, n, k, ahi, alo, lda, bhi, blo, ldb, D);
  const size_t nn = (size_t)m * n;
  k_acc_to_f64<<<nblocks(nn), 256, 0, ctx.stream>>>(D, nn, alpha, beta, C);
  QBX_LAUNCHED(ctx);
}

// ---- FP32-accurate products for the tall updates (C A, A_nl F, C (I-X)).
// An FP64 operand is split into two TF32 values, x ~ hi + lo with
// hi = tf32(x) and lo = tf32(x - hi) (about 22 significant bits together),
// and the product is formed from three TF32 tensor-core products
// accumulated in FP32, A_lo B_hi + A_hi B_lo + A_hi B_hi (the small terms
// first), then added into the FP64 output: relative error ~3e-7 per element,
// that of an FP32 product, against ~1e-5 for three BF16 products.

// The splits of a column-major FP64 block, four consecutive rows a thread
// (two 16-byte loads, 8- or 16-byte stores), one column per grid row, so no
// index division: BF16 hi/lo (ld ldb, the padding rows up to ldb zero) and/or
// TF32 hi/lo (ld ldt, rows < rows only).  Needs x 16-byte aligned, ldx even
// and ldb, ldt multiples of 4.
// RED also sums, per column, the squares of its FP64 values (1), the
// squares weighted by g2[row / 2] (2, the kinetic sum of a band over its
// complex coefficients), both of these (3: the weighted sum first, the plain
// one in a second partial array cols x gridDim.x further on), or the
// products with the same column of a second block y of x's layout (4) into
// part[column * gridDim.x + blockIdx.x]: fixed partials that the finishing
// kernels add in order.
template <bool BF, bool TF, int RED = 0>
__global__ void k_split2d_v4(const double* __restrict__ x, int rows, int ldx,
                             __nv_bfloat16* __restrict__ bhi, __nv_bfloat16* __restrict__ blo,
                             int ldb, float* __restrict__ thi, float* __restrict__ tlo, int ldt,
                             int span, const double* __restrict__ g2 = nullptr,
                             double* __restrict__ part = nullptr,
                             const double* __restrict__ y = nullptr) {
  const int c = blockIdx.y;
  const double* xc = x + (size_t)c * ldx;
  double acc = 0.0, acc2 = 0.0;
  for (int r = 4 * (blockIdx.x * blockDim.x + threadIdx.x); r < span;
       r += 4 * gridDim.x * blockDim.x) {
    double v[4];
    if (r + 3 < rows) {
      const double2 a = *reinterpret_cast<const double2*>(xc + r);
      const double2 b = *reinterpret_cast<const double2*>(xc + r + 2);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = r + q < rows ? xc[r + q] : 0.0;
    }
    if constexpr (RED == 1) {
      acc += v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
    } else if constexpr (RED == 2 || RED == 3) {
      // rows r .. r + 3 are the real and imaginary parts of coefficients
      // r / 2 and r / 2 + 1 (r even); rows past `rows` are zero
      if (r < rows) {
        const double w0 = g2[r >> 1], w1 = r + 2 < rows ? g2[(r >> 1) + 1] : 0.0;
        const double s0 = v[0] * v[0] + v[1] * v[1], s1 = v[2] * v[2] + v[3] * v[3];
        acc += s0 * w0 + s1 * w1;
        if constexpr (RED == 3) acc2 += s0 + s1;
      }
    } else if constexpr (RED == 4) {
      const double* yc = y + (size_t)c * ldx;
      if (r + 3 < rows) {
        const double2 a = *reinterpret_cast<const double2*>(yc + r);
        const double2 b = *reinterpret_cast<const double2*>(yc + r + 2);
        acc += v[0] * a.x + v[1] * a.y + v[2] * b.x + v[3] * b.y;
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (r + q < rows) acc += v[q] * yc[r + q];
      }
    }
    store_splits4<BF, TF>(v, r, rows, c, bhi, blo, ldb, thi, tlo, ldt);
  }
  if constexpr (RED != 0) {
    __shared__ double sh[32];
    const double t = red::block_sum(acc, sh);
    if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = t;
    if constexpr (RED == 3) {
      const double t2 = red::block_sum(acc2, sh);
      if (threadIdx.x == 0) part[((size_t)gridDim.y + c) * gridDim.x + blockIdx.x] = t2;
    }
  }
}

static bool v4_ok(const double* x, int ldx, int ld_out) {
  return ((uintptr_t)x % 16) == 0 && ldx % 2 == 0 && ld_out % 4 == 0;
}

int split_blocks_per_column(int span) {
  const int per = (span + 1023) / 1024;   // 256 threads x 4 rows
  return std::max(1, std::min(per, 64));
}

// grid of the v4 kernel: columns in y, rows / 4 threads in x (capped)
static dim3 v4_grid(int span, int cols) {
  return dim3((unsigned)split_blocks_per_column(span), (unsigned)cols);
}

void split_bf16_2d(Context& ctx, const double* x, int rows, int cols, int ldx, void* hi, void* lo,
                   int ldp) {
  if (v4_ok(x, ldx, ldp) && ((uintptr_t)hi | (uintptr_t)lo) % 8 == 0 && cols <= 65535) {
    k_split2d_v4<true, false><<<v4_grid(ldp, cols), 256, 0, ctx.stream>>>(
        x, rows, ldx, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ldp, nullptr, nullptr, 4, ldp);
  } else {
    const size_t n = (size_t)ldp * cols;
    k_split_bf16_2d<<<nblocks(n), 256, 0, ctx.stream>>>(x, rows, cols, ldx, (__nv_bfloat16*)hi,
                                                        (__nv_bfloat16*)lo, ldp);
  }
  QBX_LAUNCHED(ctx);
}

__global__ void k_split_tf32(const double* __restrict__ x, int rows, int cols, int ldx,
                             float* __restrict__ hi, float* __restrict__ lo, int ldy) {
  const size_t n = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / rows), r = (int)(t - (size_t)c * rows);
    const double v = x[(size_t)c * ldx + r];
    const float h = tf32_round((float)v);
    hi[(size_t)c * ldy + r] = h;
    lo[(size_t)c * ldy + r] = tf32_round((float)(v - (double)h));
  }
}

void split_tf32(Context& ctx, const double* x, int rows, int cols, int ldx, float* hi, float* lo,
                int ldy) {
  if (v4_ok(x, ldx, ldy) && ((uintptr_t)hi | (uintptr_t)lo) % 16 == 0 && cols <= 65535) {
    k_split2d_v4<false, true><<<v4_grid(rows, cols), 256, 0, ctx.stream>>>(
        x, rows, ldx, nullptr, nullptr, 4, hi, lo, ldy, rows);
  } else {
    const size_t n = (size_t)rows * cols;
    k_split_tf32<<<nblocks(n), 256, 0, ctx.stream>>>(x, rows, cols, ldx, hi, lo, ldy);
  }
  QBX_LAUNCHED(ctx);
}

// diag(S)_c = 2 sum of the squares of column c - x(0, c)^2, from the
// partials of k_split2d_v4<..., 1> (one thread per column, partials in order)
__global__ void k_diag_from_partials(const double* __restrict__ part, int nb,
                                     const double* __restrict__ x, int ldx, int cols,
                                     double* __restrict__ S, int lds) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double t = 0.0;
  for (int b = 0; b < nb; b++) t += part[(size_t)c * nb + b];
  const double x0 = x[(size_t)c * ldx];
  S[(size_t)c * lds + c] = 2.0 * t - x0 * x0;
}

// sum over columns of w[c] times the column's partials, into out[0]
__global__ void k_weighted_from_partials(const double* __restrict__ part, int nb,
                                         const double* __restrict__ w, int cols,
                                         double* __restrict__ out) {
  __shared__ double sh[32];
  double a = 0.0;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) {
    double t = 0.0;
    for (int b = 0; b < nb; b++) t += part[(size_t)c * nb + b];
    a += w[c] * t;
  }
  const double s = red::block_sum(a, sh);
  if (threadIdx.x == 0) out[0] = s;
}

// Per column c of the partials of k_split2d_v4<..., 3> of a wavefunction
// block x: w[c] times its kinetic sum into wt[c] (added over the columns by
// k_reduce_final) and the band's kinetic energy for the preconditioner,
// prec_c = sum |c|^2 G^2 / (2 sum |c|^2 - |c_0|^2) on the half sphere, 1 where
// that is not positive (Preconditioner::update, src/Preconditioner.cpp:88-143;
// the formula of the one-band-per-CTA kernel of the FP64 path).  One thread
// per column.
__global__ void k_ekin_prec_columns(const double* __restrict__ part, int nb,
                                    const double* __restrict__ w, int cols,
                                    const double* __restrict__ x, int ldx,
                                    double* __restrict__ wt, double* __restrict__ prec) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const double* part2 = part + (size_t)cols * nb;
  double te = 0.0, tn = 0.0;
  for (int b = 0; b < nb; b++) {
    te += part[(size_t)c * nb + b];
    tn += part2[(size_t)c * nb + b];
  }
  wt[c] = w[c] * te;
  const double re = x[(size_t)c * ldx], im = x[(size_t)c * ldx + 1];
  const double bn = 2.0 * (tn - 0.5 * (re * re + im * im)), be = 2.0 * te;
  double e = (0.5 * bn > 0.0) ? 0.5 * be / bn : 0.0;
  if (e == 0.0) e = 1.0;
  prec[c] = e;
}

// Per column c of the partials of k_split2d_v4<..., 4>: 2 (column's sum) -
// x(0, c) y(0, c) into wt[c], i.e. 2 Re <x_c, y_c> on the half sphere with
// G = 0 counted once.  One thread per column.
__global__ void k_dot_columns(const double* __restrict__ part, int nb, int cols,
                              const double* __restrict__ x, const double* __restrict__ y, int ldx,
                              double* __restrict__ wt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double t = 0.0;
  for (int b = 0; b < nb; b++) t += part[(size_t)c * nb + b];
  wt[c] = 2.0 * t - x[(size_t)c * ldx] * y[(size_t)c * ldx];
}

void split_bf16_ekin(Context& ctx, const double* x, int rows, int cols, int ldx, void* hi,
                     void* lo, int ldp, const double* g2, const double* occ, double* out,
                     double* prec) {
  QBX_REQUIRE(v4_ok(x, ldx, ldp) && ((uintptr_t)hi | (uintptr_t)lo) % 8 == 0 && cols <= 65535 &&
                  rows % 2 == 0 && (size_t)cols * (prec ? 129 : 64) <= ctx.colred_elems,
              50, "split with the kinetic sums: unaligned operands or no room for the partials");
  const dim3 g = v4_grid(ldp, cols);
  if (prec) {
    k_split2d_v4<true, false, 3><<<g, 256, 0, ctx.stream>>>(
        x, rows, ldx, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ldp, nullptr, nullptr, 4, ldp, g2,
        ctx.d_colred);
    QBX_LAUNCHED(ctx);
    double* wt = ctx.d_colred + (size_t)2 * cols * g.x;   // after the two partial arrays
    k_ekin_prec_columns<<<(cols + 127) / 128, 128, 0, ctx.stream>>>(ctx.d_colred, (int)g.x, occ,
                                                                    cols, x, ldx, wt, prec);
    QBX_LAUNCHED(ctx);
    red::k_reduce_final<1><<<1, 256, 0, ctx.stream>>>(wt, cols, out);
  } else {
    k_split2d_v4<true, false, 2><<<g, 256, 0, ctx.stream>>>(
        x, rows, ldx, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ldp, nullptr, nullptr, 4, ldp, g2,
        ctx.d_colred);
    QBX_LAUNCHED(ctx);
    k_weighted_from_partials<<<1, 256, 0, ctx.stream>>>(ctx.d_colred, (int)g.x, occ, cols, out);
  }
  QBX_LAUNCHED(ctx);
}

void split_bf16_dot(Context& ctx, const double* x, const double* y, int rows, int cols, int ldx,
                    void* hi, void* lo, int ldp, double* out) {
  QBX_REQUIRE(v4_ok(x, ldx, ldp) && ((uintptr_t)y % 16) == 0 &&
                  ((uintptr_t)hi | (uintptr_t)lo) % 8 == 0 && cols <= 65535 &&
                  (size_t)cols * 65 <= ctx.colred_elems,
              50, "split with the column products: unaligned operands or no room for the partials");
  const dim3 g = v4_grid(ldp, cols);
  k_split2d_v4<true, false, 4><<<g, 256, 0, ctx.stream>>>(
      x, rows, ldx, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ldp, nullptr, nullptr, 4, ldp, nullptr,
      ctx.d_colred, y);
  QBX_LAUNCHED(ctx);
  double* wt = ctx.d_colred + (size_t)cols * g.x;   // after the partials
  k_dot_columns<<<(cols + 127) / 128, 128, 0, ctx.stream>>>(ctx.d_colred, (int)g.x, cols, x, y,
                                                            ldx, wt);
  QBX_LAUNCHED(ctx);
  red::k_reduce_final<1><<<1, 256, 0, ctx.stream>>>(wt, cols, out);
  QBX_LAUNCHED(ctx);
}

void split_bf16_tf32(Context& ctx, const double* x, int rows, int cols, int ldx, void* bhi,
                     void* blo, int ldb, float* thi, float* tlo, int ldt) {
  QBX_REQUIRE(v4_ok(x, ldx, ldb) && ldt % 4 == 0 && ldb >= rows && ldt >= rows && cols <= 65535 &&
                  ((uintptr_t)bhi | (uintptr_t)blo) % 8 == 0 &&
                  ((uintptr_t)thi | (uintptr_t)tlo) % 16 == 0,
              50, "split of a block into BF16 and TF32: unaligned operands");
  QBX_REQUIRE((size_t)cols * 64 <= ctx.colred_elems, 50, "no room for the column partials");
  k_split2d_v4<true, true, 1><<<v4_grid(ldb, cols), 256, 0, ctx.stream>>>(
      x, rows, ldx, (__nv_bfloat16*)bhi, (__nv_bfloat16*)blo, ldb, thi, tlo, ldt, ldb, nullptr,
      ctx.d_colred);
  QBX_LAUNCHED(ctx);
}

void overlap_diag_from_split(Context& ctx, const double* c, int K, int n, int ldp, double* S) {
  const int nb = (int)v4_grid(ldp, n).x;
  k_diag_from_partials<<<(n + 127) / 128, 128, 0, ctx.stream>>>(ctx.d_colred, nb, c, K, n, S, n);
  QBX_LAUNCHED(ctx);
}

// Transposed split: x (rows x cols, column-major, ld ldx) -> y = x^T (cols x
// rows, ld ldy) as hi/lo pairs of TF32 (stored as FP32) or BF16, through
// 32 x 32 tiles in shared memory so that both the FP64 reads and the split
// writes are coalesced.
template <typename OUT>
__device__ __forceinline__ void split_pair(double v, OUT& h, OUT& l);
template <>
__device__ __forceinline__ void split_pair<float>(double v, float& h, float& l) {
  h = tf32_round((float)v);
  l = tf32_round((float)(v - (double)h));
}
template <>
__device__ __forceinline__ void split_pair<__nv_bfloat16>(double v, __nv_bfloat16& h,
                                                          __nv_bfloat16& l) {
  h = __double2bfloat16(v);
  l = __double2bfloat16(v - (double)__bfloat162float(h));
}

template <typename OUT>
__global__ void k_split_t(const double* __restrict__ x, int rows, int cols, int ldx,
                          OUT* __restrict__ hi, OUT* __restrict__ lo, int ldy) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
  for (int j = ty; j < 32; j += 8) {
    const int r = r0 + tx, c = c0 + j;
    t[j][tx] = (r < rows && c < cols) ? x[(size_t)c * ldx + r] : 0.0;
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int c = c0 + tx, r = r0 + j;      // y(c, r) at r * ldy + c
    if (c < cols && r < rows) {
      OUT h, l;
      split_pair<OUT>(t[tx][j], h, l);
      hi[(size_t)r * ldy + c] = h;
      lo[(size_t)r * ldy + c] = l;
    }
  }
}

void split_plain(Context& ctx, int kind, const double* x, int rows, int cols, int ldx, void* hi,
                 void* lo, int ldy) {
  if (kind == TALL_TF32)
    split_tf32(ctx, x, rows, cols, ldx, (float*)hi, (float*)lo, ldy);
  else
    split_bf16_2d(ctx, x, rows, cols, ldx, hi, lo, ldy);
}

void split_t(Context& ctx, int kind, const double* x, int rows, int cols, int ldx, void* hi,
             void* lo, int ldy) {
  dim3 grid((rows + 31) / 32, (cols + 31) / 32);
  QBX_REQUIRE(grid.y <= 65535, 50, "too many columns for the transposed split");
  if (kind == TALL_TF32)
    k_split_t<float><<<grid, 256, 0, ctx.stream>>>(x, rows, cols, ldx, (float*)hi, (float*)lo, ldy);
  else
    k_split_t<__nv_bfloat16><<<grid, 256, 0, ctx.stream>>>(
        x, rows, cols, ldx, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, ldy);
  QBX_LAUNCHED(ctx);
}

// out (rows x cols, ld ldo) = alpha * acc (ld lda) + beta * out
__global__ void k_acc2d_to_f64(const float* __restrict__ acc, int lda, int rows, int cols,
                               double alpha, double beta, double* __restrict__ out, int ldo) {
  const size_t n = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / rows), r = (int)(t - (size_t)c * rows);
    double* o = out + (size_t)c * ldo + r;
    *o = alpha * (double)acc[(size_t)c * lda + r] + (beta != 0.0 ? beta * *o : 0.0);
  }
}

// C (m x n, ld ldc) = alpha A B + beta C with A (m x k, ld lda) and B (k x n,
// ld ldb) given as TF32 hi/lo splits.  Leading dimensions of the FP32
// operands should be multiples of 4 (16-byte rows) for the fast TF32
// kernels; the FP32 product is kept with ld = m rounded up to 4.
void tf32x3_gemm_nn(Context& ctx, int m, int n, int k, double alpha, const float* Ahi,
                    const float* Alo, int lda, const float* Bhi, const float* Blo, int ldb,
                    double beta, double* C, int ldc) {
  float* D = (float*)ctx.d_acc32;
  const int ldd = (m + 3) / 4 * 4;
  QBX_REQUIRE((size_t)ldd * n <= ctx.acc32_elems, 50, "FP32 product accumulator too small");
  const float one = 1.0f, zero = 0.0f;
  const float* as[3] = {Alo, Ahi, Ahi};
  const float* bs[3] = {Bhi, Blo, Bhi};
  for (int t = 0; t < 3; t++)
    QBX_BLAS(cublasGemmEx(ctx.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &one, as[t], CUDA_R_32F,
                          lda, bs[t], CUDA_R_32F, ldb, t == 0 ? &zero : &one, D, CUDA_R_32F, ldd,
                          CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT));
  const size_t nn = (size_t)m * n;
  k_acc2d_to_f64<<<nblocks(nn), 256, 0, ctx.stream>>>(D, ldd, m, n, alpha, beta, C, ldc);
  QBX_LAUNCHED(ctx);
}

}  // namespace qbx
