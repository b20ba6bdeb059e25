// Register-resident 1-D FFTs split over a small group of lanes, for the FP32
// plane pass (fft_fast.cuh).
//
// A line of N = T * M points is held by T consecutive lanes (T = 2 or 4),
// M values per lane.  With the input index x = t + T k (lane t, register k)
// the transform is
//
//   X[k2 + M m] = sum_t W_N^{t k2} W_T^{t m} ( sum_k x[t + T k] W_M^{k k2} )
//
// i.e. an M-point DFT in each lane's registers, a twiddle by W_N^{t k2}, and
// T-point DFTs across the lanes of the group done with warp shuffles.  The
// cross-lane DFT leaves output m = bitrev(t) on lane t; the opposite
// direction starts from that distribution (decimation in time) and ends in
// the natural one, so a backward transform, a pointwise operation and a
// forward transform need no reordering.  No shared memory is used for the
// line itself and no warp synchronisation other than the shuffles.
//
// The M-point register DFT is a compile-time mixed-radix Cooley-Tukey
// recursion (radices 2, 3, 4, 5, 7, 11 of fft_reg.cuh); its twiddles are
// compile-time constants computed by a constexpr cosine/sine below.
#pragma once

#include <cuda_runtime.h>

#include "fft_reg.cuh"

namespace qbx {
namespace lane {

using reg::cadd;
using reg::cmk;
using reg::cmul;
using reg::cmulc;
using reg::csub;

// ------------------------------------------------------------ constexpr trig
// cos and sin of 2 pi p / q for integers 0 <= p < q, by Taylor series after
// reduction to |angle| <= pi/4 (the octant symmetries of the circle); the
// series is summed to double precision.
__host__ __device__ constexpr double cx_pi() { return 3.14159265358979323846264338327950288; }
__host__ __device__ constexpr double taylor_sin(double a) {
  double term = a, sum = a;
  for (int n = 1; n < 14; ++n) {
    term *= -a * a / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_cos(double a) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; ++n) {
    term *= -a * a / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}
// angle 2 pi p / q = (pi/4) * (8 p / q): octant o and remainder r in [0, 1)
__host__ __device__ constexpr void cx_cossin(long p, long q, double& c, double& s) {
  p %= q;
  if (p < 0) p += q;
  const long num = 8 * p;
  const long o = num / q;                         // octant 0..7
  const double r = (double)(num - o * q) / (double)q;   // fraction of the octant
  const double a = r * cx_pi() / 4.0;            // in [0, pi/4)
  const double b = (1.0 - r) * cx_pi() / 4.0;    // pi/4 - a
  double cc = 0, ss = 0;
  switch (o) {
    case 0: cc = taylor_cos(a); ss = taylor_sin(a); break;
    case 1: cc = taylor_sin(b); ss = taylor_cos(b); break;
    case 2: cc = -taylor_sin(a); ss = taylor_cos(a); break;
    case 3: cc = -taylor_cos(b); ss = taylor_sin(b); break;
    case 4: cc = -taylor_cos(a); ss = -taylor_sin(a); break;
    case 5: cc = -taylor_sin(b); ss = -taylor_cos(b); break;
    case 6: cc = taylor_sin(a); ss = -taylor_cos(a); break;
    default: cc = taylor_cos(b); ss = -taylor_sin(b); break;
  }
  c = cc;
  s = ss;
}
__host__ __device__ constexpr double cx_cos(long p, long q) {
  double c = 0, s = 0;
  cx_cossin(p, q, c, s);
  return c;
}
__host__ __device__ constexpr double cx_sin(long p, long q) {
  double c = 0, s = 0;
  cx_cossin(p, q, c, s);
  return s;
}

// ------------------------------------------------------------ register DFT
__host__ __device__ constexpr int first_radix(int m) {
  return m % 4 == 0 && m != 8 ? 4 : m % 2 == 0 ? 2 : m % 3 == 0 ? 3 : m % 5 == 0 ? 5
       : m % 7 == 0 ? 7 : m % 11 == 0 ? 11 : 0;
}
__host__ __device__ constexpr bool reg_ok(int m) {
  while (m > 1) {
    const int r = first_radix(m);
    if (r == 0) return false;
    m /= r;
  }
  return true;
}

// v[k] <- sum_j v[j] exp(DIR 2 pi i jk/M), all in registers (M <= ~36)
template <int M, int DIR, typename C>
__device__ __forceinline__ void dft_reg(C (&v)[M]) {
  if constexpr (M == 1) {
    return;
  } else if constexpr (M == 2 || M == 3 || M == 4 || M == 5 || M == 7 || M == 11) {
    reg::dft<M, DIR>(v);
  } else {
    // M = R Q: R interleaved sub-sequences of length Q, then R-point DFTs
    constexpr int R = first_radix(M);
    constexpr int Q = M / R;
    static_assert(R > 0, "register DFT length must factor into 2, 3, 5, 7, 11");
    using Real = decltype(v[0].x);
    C sub[R][Q];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int k = 0; k < Q; ++k) sub[r][k] = v[r + R * k];
#pragma unroll
    for (int r = 0; r < R; ++r) dft_reg<Q, DIR>(sub[r]);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      C w[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (r == 0 || q == 0) {
          w[r] = sub[r][q];
        } else {
          const Real c = (Real)cx_cos((long)r * q, M);
          const Real s = (Real)(DIR * cx_sin((long)r * q, M));
          const C x = sub[r][q];
          w[r] = cmk<C>(x.x * c - x.y * s, x.x * s + x.y * c);
        }
      }
      reg::dft<R, DIR>(w);
#pragma unroll
      for (int s2 = 0; s2 < R; ++s2) v[q + Q * s2] = w[s2];
    }
  }
}

// ------------------------------------------------------------ lane groups
template <typename C> __device__ __forceinline__ C shfl_xor(C v, int m) {
  C r;
  r.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  r.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  return r;
}

__host__ __device__ constexpr int bitrev(int t, int T) {
  int r = 0;
  for (int b = 1; b < T; b <<= 1) {
    r = (r << 1) | (t & 1);
    t >>= 1;
  }
  return r;
}

// One butterfly of a cross-lane stage: the lower lane of the pair keeps
// a + b, the upper one b - a, both as s*a + b with s = +-1 per lane (an
// exact fused multiply-add), so every lane runs the same two instructions
// instead of forming both results and selecting one.
template <typename C> __device__ __forceinline__ C lane_bfly(C a, C b, float s) {
  using Real = decltype(a.x);
  C r;
  r.x = (Real)s * a.x + b.x;
  r.y = (Real)s * a.y + b.y;
  return r;
}
// x or x * (DIR i), chosen per lane
template <int DIR, typename C> __device__ __forceinline__ C rot_if(C x, bool rot) {
  const C r = reg::cmuli<DIR>(x);
  C o;
  o.x = rot ? r.x : x.x;
  o.y = rot ? r.y : x.y;
  return o;
}

// T-point DFT across the lanes t = 0..T-1 of a group, one value per lane:
// natural input, output X[bitrev(t)] on lane t (decimation in frequency).
template <int T, int DIR, typename C>
__device__ __forceinline__ C group_dft_n2r(C a, int t) {
  static_assert(T == 1 || T == 2 || T == 4, "lane groups of 1, 2 or 4");
#pragma unroll
  for (int h = T / 2; h >= 1; h >>= 1) {
    const C b = shfl_xor(a, h);
    const int j = t & (2 * h - 1);
    a = lane_bfly(a, b, j < h ? 1.f : -1.f);
    // W_{2h}^{j-h} on the upper lanes: only W_4^1 = DIR i is not 1
    if (h == 2) a = rot_if<DIR>(a, j == 3);
  }
  return a;
}

// T-point DFT across the lanes of a group from the bit-reversed
// distribution (lane t holds input bitrev(t)) to natural output
// (decimation in time).
template <int T, int DIR, typename C>
__device__ __forceinline__ C group_dft_r2n(C a, int t) {
#pragma unroll
  for (int h = 1; h <= T / 2; h <<= 1) {
    const int j = t & (2 * h - 1);
    // the upper element of each butterfly is twiddled before the exchange
    if (h == 2) a = rot_if<DIR>(a, j == 3);
    const C b = shfl_xor(a, h);
    a = lane_bfly(a, b, j < h ? 1.f : -1.f);
  }
  return a;
}

// ------------------------------------------------------------ whole lines
// Line of N = T M points, lane t of the group holds v[k] = x[t + T k].
// Backward-style transform (direction DIR) leaving v[k2] = X[k2 + M bitrev(t)].
template <int T, int M, int DIR, typename C>
__device__ __forceinline__ void line_n2r(C (&v)[M], int t, const C* tw /* N entries */) {
  dft_reg<M, DIR>(v);
  if constexpr (T > 1) {
    // twiddle loads stay after the register DFT (hoisted above it they would
    // hold M more values in registers through it)
    asm volatile("" ::: "memory");
#pragma unroll
    for (int k2 = 1; k2 < M; ++k2) {
      const C w = tw[t * k2];
      v[k2] = DIR > 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2) v[k2] = group_dft_n2r<T, DIR>(v[k2], t);
  }
}

// The opposite: lane t holds v[k2] = x[k2 + M bitrev(t)]; afterwards
// v[k] = X[t + T k].
template <int T, int M, int DIR, typename C>
__device__ __forceinline__ void line_r2n(C (&v)[M], int t, const C* tw) {
  if constexpr (T > 1) {
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2) v[k2] = group_dft_r2n<T, DIR>(v[k2], t);
    asm volatile("" ::: "memory");
#pragma unroll
    for (int k2 = 1; k2 < M; ++k2) {
      const C w = tw[t * k2];
      v[k2] = DIR > 0 ? cmul(v[k2], w) : cmulc(v[k2], w);
    }
  }
  dft_reg<M, DIR>(v);
}

// Lanes per line for a length: 4 when N/4 has a register plan of at most 36
// points, else 2 (N/2 <= 36), else 0 (no register plan).
__host__ __device__ constexpr int lanes_for(int n) {
  return (n % 4 == 0 && n / 4 <= 36 && reg_ok(n / 4)) ? 4
       : (n % 2 == 0 && n / 2 <= 36 && reg_ok(n / 2)) ? 2 : 0;
}

}  // namespace lane
}  // namespace qbx
