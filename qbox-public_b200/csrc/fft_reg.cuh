// Warp-synchronous 1-D FFTs of compile-time length for the staged 3-D
// transforms (fft_fast.cuh).
//
// One warp transforms one line of N complex values held in shared memory.
// The length is factored into radix stages at compile time, odd radices
// first (11, 7, 5, 3), then a 2, then 4s, so that the last stages write
// stride-1 across the lanes.  Each stage is a self-sorting Stockham pass done
// in place: every lane first loads the inputs of its butterflies (N/R of
// them, spread over the 32 lanes) into registers, the warp synchronises, and
// the lanes then twiddle, transform and store.  Only __syncwarp separates the
// stages, so the warps of a CTA work on different lines independently.
//
// The first stage can read its inputs through a loader functor and the last
// stage can hand its outputs to a storer functor, which is how the kernels
// fuse the gather from the coefficient sphere or the plane tile, the
// multiplication by V(r) and the density accumulation into the transforms.
//
// Sign convention: DIR = +1 computes out[k] = sum_j in[j] exp(+2 pi i jk/N)
// (the reference's backward transform, unscaled), DIR = -1 the forward one.
// Twiddles exp(+2 pi i k/N) come from a length-N table in shared memory,
// conjugated for DIR = -1.  The small DFTs use the cosines and sines of
// 2 pi j/R as literal constants.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qbx {
namespace reg {

template <typename T> struct CT;
template <> struct CT<float> { using c = float2; };
template <> struct CT<double> { using c = double2; };

// ------------------------------------------------------------ plan
struct CPlan {
  int n = 0, ns = 0, rest = 1;
  int r[16] = {0};
};

__host__ __device__ constexpr CPlan cplan(int n) {
  CPlan p{};
  p.n = n;
  int m = n, twos = 0;
  while (m % 2 == 0) { m /= 2; ++twos; }
  const int odd[4] = {11, 7, 5, 3};
  for (int i = 0; i < 4; ++i)
    while (m % odd[i] == 0) { p.r[p.ns++] = odd[i]; m /= odd[i]; }
  if (twos % 2) p.r[p.ns++] = 2;
  for (int i = 0; i < twos / 2; ++i) p.r[p.ns++] = 4;
  p.rest = m;
  return p;
}
__host__ __device__ constexpr int stage_count(int n) { return cplan(n).ns; }
__host__ __device__ constexpr int stage_radix(int n, int s) { return cplan(n).r[s]; }
__host__ __device__ constexpr int stage_ns(int n, int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= cplan(n).r[i];
  return p;
}
__host__ __device__ constexpr bool plan_ok(int n) { return n > 1 && cplan(n).rest == 1; }

// cos(2 pi j/R), sin(2 pi j/R) for 1 <= j <= (R-1)/2
__host__ __device__ constexpr double rcos(int R, int j) {
  return R == 3 ? -0.5
       : R == 5 ? (j == 1 ? 0.30901699437494745 : -0.8090169943749475)
       : R == 7 ? (j == 1 ? 0.6234898018587335 : j == 2 ? -0.2225209339563144 : -0.9009688679024191)
       : (j == 1 ? 0.8412535328311812 : j == 2 ? 0.41541501300188644
          : j == 3 ? -0.14231483827328514 : j == 4 ? -0.6548607339452851 : -0.9594929736144974);
}
__host__ __device__ constexpr double rsin(int R, int j) {
  return R == 3 ? 0.8660254037844386
       : R == 5 ? (j == 1 ? 0.9510565162951535 : 0.5877852522924731)
       : R == 7 ? (j == 1 ? 0.7818314824680298 : j == 2 ? 0.9749279121818236 : 0.4338837391175581)
       : (j == 1 ? 0.5406408174555976 : j == 2 ? 0.9096319953545183
          : j == 3 ? 0.9898214418809327 : j == 4 ? 0.7557495743542583 : 0.28173255684142967);
}

// ------------------------------------------------------------ arithmetic
template <typename C> __device__ __forceinline__ C cmk(double x, double y) {
  C r; r.x = x; r.y = y; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  C r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  C r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
// DIR * i * a
template <int DIR, typename C> __device__ __forceinline__ C cmuli(C a) {
  C r;
  if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

// R-point DFT in registers: v[k] <- sum_q v[q] exp(DIR 2 pi i qk/R)
template <int R, int DIR, typename C>
__device__ __forceinline__ void dft(C (&v)[R]) {
  if constexpr (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const C c = cadd(v[1], v[3]), d = cmuli<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  } else {
    // odd prime R: pair q with R-q,
    //   out_k = v0 + sum_m (v_m + v_{R-m}) cos(2 pi mk/R)
    //              + DIR i sum_m (v_m - v_{R-m}) sin(2 pi mk/R)
    using Real = decltype(v[0].x);
    constexpr int H = (R - 1) / 2;
    C a[H + 1], b[H + 1];
    C s0 = v[0];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      a[m] = cadd(v[m], v[R - m]);
      b[m] = csub(v[m], v[R - m]);
      s0 = cadd(s0, a[m]);
    }
    C out[R];
    out[0] = s0;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      Real rx = v[0].x, ry = v[0].y, ix = 0, iy = 0;
#pragma unroll
      for (int m = 1; m <= H; ++m) {
        const int j = (m * k) % R;
        const Real cs = (Real)rcos(R, j <= H ? j : R - j);
        const Real sn = (Real)(j <= H ? rsin(R, j) : -rsin(R, R - j));
        rx += a[m].x * cs;
        ry += a[m].y * cs;
        ix += b[m].x * sn;
        iy += b[m].y * sn;
      }
      out[k] = cmk<C>(rx - DIR * iy, ry + DIR * ix);
      out[R - k] = cmk<C>(rx + DIR * iy, ry - DIR * ix);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
  }
}

// ------------------------------------------------------------ functors
template <typename C> struct BufLoad {
  const C* b;
  __device__ __forceinline__ C operator()(int i) const { return b[i]; }
};
template <typename C> struct BufStore {
  C* b;
  __device__ __forceinline__ void operator()(int i, C v) const { b[i] = v; }
};

// ------------------------------------------------------------ shared memory
// The working line and the twiddle table are addressed through 32-bit
// shared-window offsets that the optimiser cannot see through (see
// warp_fft), with explicit ld/st.shared.
__device__ __forceinline__ float2 lds(uint32_t a, float2*) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ double2 lds(uint32_t a, double2*) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts(uint32_t a, float2 v) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void sts(uint32_t a, double2 v) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void warp_sync_mem() {
  asm volatile("" ::: "memory");
  __syncwarp();
  asm volatile("" ::: "memory");
}

// ------------------------------------------------------------ stages
// First-stage geometry of a length-N line: lane + 32*rd is the butterfly,
// q its input; input index = butterfly + q * NB.
template <int N> struct FirstStage {
  static constexpr int R = stage_radix(N, 0);
  static constexpr int NB = N / R;
  static constexpr int RD = (NB + 31) / 32;
};

template <int N, int S, int DIR, typename C, typename LD, typename ST>
__device__ __forceinline__ void wstage(uint32_t sbuf, uint32_t stw, int lane, const LD& ld,
                                       const ST& st) {
  constexpr int R = stage_radix(N, S);
  constexpr int NS = stage_ns(N, S);
  constexpr int NB = N / R;
  constexpr int RD = (NB + 31) / 32;
  constexpr bool FIRST = (S == 0);
  constexpr bool LAST = (S == stage_count(N) - 1);
  constexpr uint32_t E = sizeof(C);
  C v[RD][R];
#pragma unroll
  for (int rd = 0; rd < RD; ++rd) {
    const int i = lane + 32 * rd;
    if (NB % 32 == 0 || i < NB) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if constexpr (FIRST) v[rd][q] = ld(rd, q, i + q * NB);
        else v[rd][q] = lds(sbuf + (uint32_t)(i + q * NB) * E, (C*)nullptr);
      }
    }
  }
  warp_sync_mem();
#pragma unroll
  for (int rd = 0; rd < RD; ++rd) {
    const int i = lane + 32 * rd;
    if (NB % 32 == 0 || i < NB) {
      const int j = i % NS;
      if constexpr (NS > 1) {
        constexpr int TS = N / (NS * R);
#pragma unroll
        for (int q = 1; q < R; ++q) {
          const C w = lds(stw + (uint32_t)(q * j * TS) * E, (C*)nullptr);
          v[rd][q] = DIR > 0 ? cmul(v[rd][q], w) : cmulc(v[rd][q], w);
        }
      }
      dft<R, DIR>(v[rd]);
      const int base = (i - j) * R + j;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        if constexpr (LAST) st(base + q * NS, v[rd][q]);
        else sts(sbuf + (uint32_t)(base + q * NS) * E, v[rd][q]);
      }
    }
  }
  warp_sync_mem();
}

template <int N, int S, int DIR, typename C, typename LD, typename ST>
__device__ __forceinline__ void wstages(uint32_t sbuf, uint32_t stw, int lane, const LD& ld,
                                        const ST& st) {
  wstage<N, S, DIR, C>(sbuf, stw, lane, ld, st);
  if constexpr (S + 1 < stage_count(N)) wstages<N, S + 1, DIR, C>(sbuf, stw, lane, ld, st);
}

// Adapts a loader of the form ld(i) to the first stage's ld(rd, q, i).
template <typename LD> struct IndexLoad {
  const LD& f;
  __device__ __forceinline__ auto operator()(int, int, int i) const { return f(i); }
};

// Transform one line with the warp.  buf (N values, shared memory) is the
// working line; ld(i) supplies input i to the first stage, st(k, value)
// takes output k from the last stage.
template <int N, int DIR, typename C, typename LD, typename ST>
__device__ __forceinline__ void warp_fft(C* buf, const C* tw, int lane, const LD& ld, const ST& st) {
  static_assert(plan_ok(N), "FFT length must factor into 2, 3, 5, 7, 11");
  uint32_t sbuf = (uint32_t)__cvta_generic_to_shared(buf);
  uint32_t stw = (uint32_t)__cvta_generic_to_shared(tw);
  // Hide the addresses and the lane from the optimiser: otherwise it keeps
  // every lane's twiddle and line offsets of every stage in registers across
  // the callers' loops, which costs more registers (and occupancy) than
  // recomputing them.
  asm volatile("" : "+r"(sbuf), "+r"(stw), "+r"(lane));
  wstages<N, 0, DIR, C>(sbuf, stw, lane, IndexLoad<LD>{ld}, st);
}

// As warp_fft, with a first-stage loader that also receives the butterfly
// round rd and input q (for values the caller prefetched into registers in
// FirstStage<N> order).
template <int N, int DIR, typename C, typename LD, typename ST>
__device__ __forceinline__ void warp_fft_rq(C* buf, const C* tw, int lane, const LD& ld,
                                            const ST& st) {
  static_assert(plan_ok(N), "FFT length must factor into 2, 3, 5, 7, 11");
  uint32_t sbuf = (uint32_t)__cvta_generic_to_shared(buf);
  uint32_t stw = (uint32_t)__cvta_generic_to_shared(tw);
  asm volatile("" : "+r"(sbuf), "+r"(stw), "+r"(lane));
  wstages<N, 0, DIR, C>(sbuf, stw, lane, ld, st);
}

}  // namespace reg
}  // namespace qbx
