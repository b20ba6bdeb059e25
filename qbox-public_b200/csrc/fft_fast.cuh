// Staged wavefunction FFT kernels specialised on the grid lengths.
//
// Same three-kernel structure as the generic path in fft.cu (z sticks ->
// plane tile -> z sticks, band pairs packed as psi_1 + i psi_2), with every
// 1-D transform a warp-synchronous register FFT of compile-time length
// (fft_reg.cuh) and the surrounding data movement fused into the first and
// last radix stages:
//
//   kz_bwd  : the first z stage reads the two bands' coefficients of the
//             stick's rod straight from HBM (+G: c1 + i c2, -G: conj(c1) +
//             i conj(c2)); the sticks of the CTA are then written
//             plane-major, coalesced across sticks.
//   kxy     : one CTA per (z plane, pair chunk).  The plane's sticks are
//             scattered into a compact tile P[column][y] (odd row pitch, so
//             strided lane accesses spread over the banks), y is transformed
//             column by column in place, then each warp takes whole x rows:
//             the first x stage reads the row straight out of P (zeros off
//             the occupied columns), and the last stage either accumulates
//             f1/Omega psi_1^2 + f2/Omega psi_2^2 (density) or multiplies by
//             V(r) into the warp's line, after which the forward x transform
//             writes only the occupied columns back into P; the forward y
//             pass and a coalesced gather return the sticks.
//   kz_fwd  : coalesced read of the sticks, forward z transform, unpack of
//             the two bands (src/BasisMapping.cpp:722-750), 1/N scale and
//             the kinetic term: hc = 1/2 |G|^2 c + result.
//
// Mixed precision accumulates the density of a CTA's pairs in an FP32 plane
// in shared memory and adds it to the FP64 grid once per CTA; FP64 adds each
// pair's contribution with FP64 atomics.
#pragma once

#include <algorithm>
#include <type_traits>

#include "fft_lane.cuh"
#include "fft_reg.cuh"
#include "qbx_internal.h"

namespace qbx {
namespace fast {

using reg::BufLoad;
using reg::BufStore;
using reg::cmk;

constexpr int kZThreads = 256;
// CTA shapes of the plane kernel (threads, CTAs per SM it is compiled for).
// FP64 lines need about twice the registers of FP32 lines; the FP32 density
// pass holds an FP32 plane in shared memory, so one CTA per SM; the FP32
// H*psi pass comes in two shapes, one 512-thread CTA or two 256-thread CTAs
// per SM, picked at run time.
template <typename T, int OP> struct XYDefault { static constexpr int shape = 3; };
template <> struct XYDefault<float, 0> { static constexpr int shape = 1; };
// Plane CTA shapes: 0 = 256 threads, two CTAs per SM; 1 = 512 threads, one
// per SM; 2 = 512 threads compiled for two per SM (64 registers per
// thread); 3 = 256 threads, one per SM (the FP64 kernels)
__host__ __device__ constexpr int xy_threads(int shape) {
  return (shape == 0 || shape == 3) ? 256 : 512;
}
__host__ __device__ constexpr int xy_minblocks(int shape) { return (shape == 0 || shape == 2) ? 2 : 1; }

template <typename C>
__device__ __forceinline__ void load_tw(C* dst, const double2* src, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = cmk<C>(src[k].x, src[k].y);
}

__host__ __device__ constexpr int pitch(int n) { return (n % 2 == 0) ? n + 1 : n; }

// cp.async: asynchronous copies from global into shared memory, completed by
// cp_async_wait_all (this thread's copies) and made visible to the CTA by a
// barrier after it
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ------------------------------------------------------------ z backward
template <typename T, int N2>
__global__ void __launch_bounds__(kZThreads)
kz_bwd(const double2* __restrict__ c, int ngw, int nst, int pair0, DeviceSticks g,
       const double2* __restrict__ twz, typename reg::CT<T>::c* __restrict__ zbuf,
       int rods_per_cta) {
  using C = typename reg::CT<T>::c;
  constexpr int LD = pitch(N2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* lines = tw + N2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const double2* c1 = c + (size_t)b1 * ngw;
  const double2* c2 = (b1 + 1 < nst) ? c + (size_t)(b1 + 1) * ngw : nullptr;
  load_tw(tw, twz, N2);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  constexpr int half = (N2 + 1) / 2;
  for (int line = warp; line < nl; line += nw) {
    const int s = s0 + line;
    const int r = (s + 1) >> 1;
    const int lmin = g.rod_lmin[r], size = g.rod_size[r], first = g.rod_first[r];
    const bool rod0 = (r == 0);
    const bool mstick = ((s & 1) == 0);   // the -G stick of a rod r > 0
    auto ld = [&](int z) -> C {
      const int lz = z < half ? z : z - N2;
      const bool minus = rod0 ? (lz <= 0) : mstick;
      const int l = minus ? -lz : lz;
      double vx = 0.0, vy = 0.0;
      if (l >= lmin && l < lmin + size) {
        const double2 p = c1[first + (l - lmin)];
        const double2 q = c2 ? c2[first + (l - lmin)] : make_double2(0.0, 0.0);
        if (!minus) { vx = p.x - q.y; vy = p.y + q.x; }
        else        { vx = p.x + q.y; vy = q.x - p.y; }
      }
      return cmk<C>(vx, vy);
    };
    C* buf = lines + line * LD;
    reg::warp_fft<N2, +1>(buf, tw, lane, ld, BufStore<C>{buf});
  }
  __syncthreads();
  C* out = zbuf + (size_t)pl * N2 * g.nvec;
  for (int t = threadIdx.x; t < nl * N2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    out[(size_t)z * g.nvec + s0 + line] = lines[line * LD + z];
  }
}

// ------------------------------------------------------------ z forward
template <typename T, int N2>
__global__ void __launch_bounds__(kZThreads)
kz_fwd(const typename reg::CT<T>::c* __restrict__ zbuf, int ngw, int nst, int pair0,
       DeviceSticks g, const double2* __restrict__ twz, double scale,
       const double2* __restrict__ c, const double* __restrict__ g2, double2* __restrict__ hc,
       int rods_per_cta) {
  using C = typename reg::CT<T>::c;
  constexpr int LD = pitch(N2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* lines = tw + N2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const bool two = (b1 + 1 < nst);
  load_tw(tw, twz, N2);
  const C* in = zbuf + (size_t)pl * N2 * g.nvec;
  for (int t = threadIdx.x; t < nl * N2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    lines[line * LD + z] = in[(size_t)z * g.nvec + s0 + line];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int line = warp; line < nl; line += nw) {
    C* buf = lines + line * LD;
    reg::warp_fft<N2, -1>(buf, tw, lane, BufLoad<C>{buf}, BufStore<C>{buf});
  }
  __syncthreads();
  // one warp per rod: unpack the pair and add the kinetic term
  for (int r = r0 + warp; r < r1; r += nw) {
    const int lmin = g.rod_lmin[r], size = g.rod_size[r], first = g.rod_first[r];
    const int sp = (r == 0) ? 0 : 2 * r - 1 - s0;
    const int sm = (r == 0) ? 0 : 2 * r - s0;
    for (int e = lane; e < size; e += 32) {
      const int l = lmin + e;
      const int zp = ((l % N2) + N2) % N2;
      const int zm = ((-l % N2) + N2) % N2;
      const C P = lines[sp * LD + zp];
      const C M = lines[sm * LD + zm];
      // c1 = (Z(G) + conj Z(-G))/2, c2 = -i (Z(G) - conj Z(-G))/2
      const double px = P.x, py = P.y, mx = M.x, my = M.y;
      const double c1x = 0.5 * (px + mx) * scale, c1y = 0.5 * (py - my) * scale;
      const double c2x = 0.5 * (py + my) * scale, c2y = 0.5 * (mx - px) * scale;
      const int ig = first + e;
      const double kin = 0.5 * g2[ig];
      const size_t i1 = (size_t)b1 * ngw + ig;
      const double2 a = c[i1];
      hc[i1] = make_double2(kin * a.x + c1x, kin * a.y + c1y);
      if (two) {
        const size_t i2 = i1 + ngw;
        const double2 b = c[i2];
        hc[i2] = make_double2(kin * b.x + c2x, kin * b.y + c2y);
      }
    }
  }
}

// ------------------------------------------------------------ z sticks,
// register lanes (FP32)
// The z transforms of kz_bwd / kz_fwd with each stick's line held in the
// registers of a group of lane::lanes_for(N2) lanes (fft_lane.cuh) instead
// of a warp working through shared-memory stages.  A CTA takes the sticks of
// rods_per_cta rods (2 rods_per_cta - 1 sticks, or 2 rods_per_cta) for one
// band pair, one lane group per stick.
//
// Backward: lane t of a group loads the stick's values at z = t + T k
// straight from the two bands' coefficients, transforms, and stores its
// outputs z = k2 + M bitrev(t) to the sticks: for each k2 a warp's 8 groups
// write T runs of 8 consecutive sticks.  No shared memory but the twiddles.
// Lane register k of a line held by T lanes (points t + T k, t < T) holds a
// point within prune_width(N) of 0 for some lane: the registers for which
// this is false carry only points outside the sphere, which the pruned
// kernels neither load nor store.
template <int N, int T> __host__ __device__ constexpr bool keep_reg(int k) {
  return T * k <= prune_width(N) || T * k + T - 1 >= N - prune_width(N);
}

template <int N2, int MINB, bool PRUNE = false>
__global__ void __launch_bounds__(256, MINB)
kz_bwd_lane(const double2* __restrict__ c, int ngw, int nst, int pair0, DeviceSticks g,
            const double2* __restrict__ twz, float2* __restrict__ zbuf, int rods_per_cta) {
  using C = float2;
  constexpr int T = lane::lanes_for(N2), M = N2 / T;
  static_assert(T > 0, "no register plan for this length");
  __shared__ C tw[N2];
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const double2* c1 = c + (size_t)b1 * ngw;
  const double2* c2 = (b1 + 1 < nst) ? c + (size_t)(b1 + 1) * ngw : nullptr;
  load_tw(tw, twz, N2);
  __syncthreads();
  const int t = threadIdx.x % T, mr = lane::bitrev(t, T);
  constexpr int half = (N2 + 1) / 2;
  C* out = zbuf + (size_t)pl * N2 * g.nvec;
  // rounds uniform across the CTA, so that every lane takes part in the shuffles
#pragma unroll 1
  for (int base = 0; base < nl; base += blockDim.x / T) {
    const int line = base + threadIdx.x / T;
    const bool ok = line < nl;
    const int s = s0 + (ok ? line : 0);
    const int r = (s + 1) >> 1;
    const int lmin = g.rod_lmin[r], size = g.rod_size[r], first = g.rod_first[r];
    const bool rod0 = (r == 0);
    const bool mstick = ((s & 1) == 0);   // the -G stick of a rod r > 0
    C v[M];
#pragma unroll
    for (int k = 0; k < M; ++k) {
      if (PRUNE && !keep_reg<N2, T>(k)) {
        v[k] = cmk<C>(0.0, 0.0);
        continue;
      }
      const int z = t + T * k;
      const int lz = z < half ? z : z - N2;
      const bool minus = rod0 ? (lz <= 0) : mstick;
      const int l = minus ? -lz : lz;
      double vx = 0.0, vy = 0.0;
      if (ok && l >= lmin && l < lmin + size) {
        const double2 p = c1[first + (l - lmin)];
        const double2 q = c2 ? c2[first + (l - lmin)] : make_double2(0.0, 0.0);
        if (!minus) { vx = p.x - q.y; vy = p.y + q.x; }
        else        { vx = p.x + q.y; vy = q.x - p.y; }
      }
      v[k] = cmk<C>(vx, vy);
    }
    lane::line_n2r<T, M, +1>(v, t, tw);
    if (ok) {
#pragma unroll
      for (int k2 = 0; k2 < M; ++k2) out[(size_t)(k2 + M * mr) * g.nvec + s] = v[k2];
    }
  }
}

// Forward: lane t loads z = k2 + M bitrev(t) of its stick (the distribution
// the backward kernel stored), transforms back to natural order, and puts the
// line into shared memory, from which one warp per rod unpacks the pair and
// adds the kinetic term exactly as kz_fwd does.
template <int N2, bool PRUNE = false>
__global__ void __launch_bounds__(256)
kz_fwd_lane(const float2* __restrict__ zbuf, int ngw, int nst, int pair0, DeviceSticks g,
            const double2* __restrict__ twz, double scale, const double2* __restrict__ c,
            const double* __restrict__ g2, double2* __restrict__ hc, int rods_per_cta) {
  using C = float2;
  constexpr int T = lane::lanes_for(N2), M = N2 / T;
  constexpr int LD = pitch(N2);
  static_assert(T > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* lines = tw + N2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const bool two = (b1 + 1 < nst);
  load_tw(tw, twz, N2);
  __syncthreads();
  const int t = threadIdx.x % T, mr = lane::bitrev(t, T);
  const C* in = zbuf + (size_t)pl * N2 * g.nvec;
#pragma unroll 1
  for (int base = 0; base < nl; base += blockDim.x / T) {
    const int line = base + threadIdx.x / T;
    const bool ok = line < nl;
    const int s = s0 + (ok ? line : 0);
    C v[M];
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2)
      v[k2] = ok ? in[(size_t)(k2 + M * mr) * g.nvec + s] : cmk<C>(0.0, 0.0);
    lane::line_r2n<T, M, -1>(v, t, tw);
    if (ok) {
      C* buf = lines + line * LD;
#pragma unroll
      for (int k = 0; k < M; ++k)
        if (!PRUNE || keep_reg<N2, T>(k)) buf[t + T * k] = v[k];
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = r0 + warp; r < r1; r += nw) {
    const int lmin = g.rod_lmin[r], size = g.rod_size[r], first = g.rod_first[r];
    const int sp = (r == 0) ? 0 : 2 * r - 1 - s0;
    const int sm = (r == 0) ? 0 : 2 * r - s0;
    for (int e = lane; e < size; e += 32) {
      const int l = lmin + e;
      const int zp = ((l % N2) + N2) % N2;
      const int zm = ((-l % N2) + N2) % N2;
      const C P = lines[sp * LD + zp];
      const C Mv = lines[sm * LD + zm];
      // c1 = (Z(G) + conj Z(-G))/2, c2 = -i (Z(G) - conj Z(-G))/2
      const double px = P.x, py = P.y, mx = Mv.x, my = Mv.y;
      const double c1x = 0.5 * (px + mx) * scale, c1y = 0.5 * (py - my) * scale;
      const double c2x = 0.5 * (py + my) * scale, c2y = 0.5 * (mx - px) * scale;
      const int ig = first + e;
      const double kin = 0.5 * g2[ig];
      const size_t i1 = (size_t)b1 * ngw + ig;
      const double2 a = c[i1];
      hc[i1] = make_double2(kin * a.x + c1x, kin * a.y + c1y);
      if (two) {
        const size_t i2 = i1 + ngw;
        const double2 b = c[i2];
        hc[i2] = make_double2(kin * b.x + c2x, kin * b.y + c2y);
      }
    }
  }
}

// ------------------------------------------------------------ xy plane
enum { XY_DENSITY = 0, XY_VPSI = 1 };

// density accumulator in shared memory: FP32 plane for the mixed path
template <typename T> struct UseSmemAcc { static constexpr bool v = false; };
template <> struct UseSmemAcc<float> { static constexpr bool v = true; };

template <typename T, int N0, int N1, int OP>
__host__ size_t xy_smem_bytes(int ncol, int nwarps) {
  using C = typename reg::CT<T>::c;
  size_t b = sizeof(C) * ((size_t)N0 + N1 + (size_t)ncol * pitch(N1) + (size_t)nwarps * N0);
  if (OP == XY_DENSITY && UseSmemAcc<T>::v) b += sizeof(float) * (size_t)N0 * N1;
  b += sizeof(int) * N0;
  return b;
}

// shared memory: [twx N0][twy N1][P ncol x pitch(N1)][one line of N0 per
// warp][FP32 density plane N1 x N0, mixed density only][xmap N0 ints]
template <typename T, int N0, int N1, int OP, int SHAPE>
__global__ void __launch_bounds__(xy_threads(SHAPE), xy_minblocks(SHAPE))
kxy(typename reg::CT<T>::c* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
    const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
    const T* __restrict__ v, double* __restrict__ rho, const double* __restrict__ w, int pair0,
    int nst) {
  using C = typename reg::CT<T>::c;
  constexpr int LD = pitch(N1);
  constexpr bool SACC = (OP == XY_DENSITY) && UseSmemAcc<T>::v;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  C* lines = P + (size_t)ncol * LD;
  float* acc = reinterpret_cast<float*>(lines + (size_t)nw * N0);
  int* xmap = reinterpret_cast<int*>(acc + (SACC ? (size_t)N0 * N1 : 0));
  C* line = lines + (size_t)warp * N0;
  const int z = blockIdx.x;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  if constexpr (SACC)
    for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
  #pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
    // tile: zero, then scatter the plane's sticks
    for (int t = threadIdx.x; t < ncol * LD; t += blockDim.x) P[t] = cmk<C>(0.0, 0.0);
    __syncthreads();
    for (int s = threadIdx.x; s < nvec; s += blockDim.x)
      P[g.stick_col[s] * LD + g.stick_y[s]] = zp[s];
    __syncthreads();
    // backward y, in place, one warp per occupied column
    #pragma unroll 1
    for (int cidx = warp; cidx < ncol; cidx += nw) {
      C* col = P + cidx * LD;
      reg::warp_fft<N1, +1>(col, twy, lane, BufLoad<C>{col}, BufStore<C>{col});
    }
    __syncthreads();
    double w1 = 0.0, w2 = 0.0;
    if (OP == XY_DENSITY) {
      const int b1 = 2 * (pair0 + pl);
      w1 = w[b1];
      w2 = (b1 + 1 < nst) ? w[b1 + 1] : 0.0;
    }
    // x rows, one warp per row; the first stage reads the row out of P
    #pragma unroll 1
    for (int y = warp; y < N1; y += nw) {
      auto ldP = [&](int x) -> C {
        const int cidx = xmap[x];
        return cidx >= 0 ? P[cidx * LD + y] : cmk<C>(0.0, 0.0);
      };
      const size_t rowbase = ((size_t)z * N1 + y) * N0;
      if constexpr (OP == XY_DENSITY) {
        if constexpr (SACC) {
          const float f1 = (float)w1, f2 = (float)w2;
          float* arow = acc + y * N0;
          auto st = [&](int x, C val) {
            arow[x] += f1 * (float)val.x * (float)val.x + f2 * (float)val.y * (float)val.y;
          };
          reg::warp_fft<N0, +1>(line, twx, lane, ldP, st);
        } else {
          auto st = [&](int x, C val) {
            atomicAdd(&rho[rowbase + x], w1 * (double)val.x * (double)val.x +
                                             w2 * (double)val.y * (double)val.y);
          };
          reg::warp_fft<N0, +1>(line, twx, lane, ldP, st);
        }
      } else {
        // V(r) of this row, prefetched in the order the forward transform's
        // first stage reads the row, multiplied in as it loads
        using FS = reg::FirstStage<N0>;
        const T* vrow = v + rowbase;
        T vpre[FS::RD][FS::R];
#pragma unroll
        for (int rd = 0; rd < FS::RD; ++rd)
#pragma unroll
          for (int q = 0; q < FS::R; ++q) {
            const int i = lane + 32 * rd;
            vpre[rd][q] = (FS::NB % 32 == 0 || i < FS::NB) ? vrow[i + q * FS::NB] : T(0);
          }
        reg::warp_fft<N0, +1>(line, twx, lane, ldP, BufStore<C>{line});
        auto ldv = [&](int rd, int q, int i) -> C {
          C val = line[i];
          val.x *= vpre[rd][q];
          val.y *= vpre[rd][q];
          return val;
        };
        auto stP = [&](int x, C val) {
          const int cidx = xmap[x];
          if (cidx >= 0) P[cidx * LD + y] = val;
        };
        reg::warp_fft_rq<N0, -1>(line, twx, lane, ldv, stP);
      }
    }
    __syncthreads();
    if (OP == XY_VPSI) {
      #pragma unroll 1
    for (int cidx = warp; cidx < ncol; cidx += nw) {
        C* col = P + cidx * LD;
        reg::warp_fft<N1, -1>(col, twy, lane, BufLoad<C>{col}, BufStore<C>{col});
      }
      __syncthreads();
      for (int s = threadIdx.x; s < nvec; s += blockDim.x)
        zp[s] = P[g.stick_col[s] * LD + g.stick_y[s]];
      __syncthreads();
    }
  }
  if constexpr (SACC) {
    __syncthreads();
    const size_t pbase = (size_t)z * N1 * N0;
    for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) atomicAdd(&rho[pbase + t], (double)acc[t]);
  }
}

// ------------------------------------------------------------ xy plane,
// register lanes (FP32)
// The plane pass of kxy with every line transform held in registers by a
// group of lane::lanes_for(N) lanes (fft_lane.cuh): no line buffers, no
// per-stage shared-memory round trips.  Loops over lines run in rounds of
// blockDim/T groups that are uniform across the CTA, so that every lane
// takes part in the shuffles; groups past the end carry zeros.
// shared memory: [twx N0][twy N1][P ncol x pitch(N1)][FP32 density plane
// N1 x N0, density only][xmap N0 ints]
template <int N0, int N1, int OP>
__host__ size_t xyl_smem_bytes(int ncol) {
  size_t b = sizeof(float2) * ((size_t)N0 + N1 + (size_t)ncol * pitch(N1));
  if (OP == XY_DENSITY) b += sizeof(float) * (size_t)N0 * N1;
  return b + sizeof(int) * N0;
}

// CTA shapes of kxy_lane (most threads, CTAs per SM compiled for):
// 0 = 256 x 2 (128 registers), 1 = 256 x 1, 2 = 512 x 1, 3 = 320 x 1,
// 4 = 288 x 2 (113 registers).  Shapes 3 and 4 are launched with just
// enough lanes for one round over the occupied columns (ncol * T rounded up
// to a warp), which for 65 columns is 9 warps.
__host__ __device__ constexpr int lane_threads(int shape) {
  return shape == 2 ? 512 : shape == 3 ? 320 : shape == 4 ? 288 : 256;
}
__host__ __device__ constexpr int lane_minblocks(int shape) { return (shape == 0 || shape == 4) ? 2 : 1; }

// The real-space band pairs psi(r) kept in HBM between the density pass and
// the H*psi pass of the same step (FP32, 8 bytes per point and pair: 11 GB
// at 1 024 bands on a 140^3 grid).  A row's values stay in the register
// layout of the x transform's output: the value at x = MX*bitrev(tx) + k of
// lane tx is stored at k*TX + tx, so a warp's 8 rows x 4 lanes write 8 full
// 32-byte sectors per store, and the H*psi kernel reads each lane's values
// back into the registers it needs them in.
template <int N0, int N1, int TX, int MX>
__device__ __forceinline__ void store_psir(float2* __restrict__ psir, int pair, int n2, int z,
                                           int y, int tx, const float2 (&val)[MX]) {
  float2* row = psir + (((size_t)pair * n2 + z) * N1 + y) * N0 + tx;
#pragma unroll
  for (int k = 0; k < MX; ++k) row[k * TX] = val[k];
}

// L2 prefetch of a contiguous range (16-byte aligned start, size a multiple
// of 16 bytes): one instruction streams it from HBM while the CTA works on
// something else.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// H*psi plane pass from the stored psi(r): times V(r), forward x, forward y
// on the occupied columns, outputs to the sticks through the column map (the
// second half of kxy_lane_map; the backward z and xy transforms of the
// density pass are not repeated).  A CTA takes pairs_per_cta band pairs of
// one plane; while it works on one pair, the next pair's psi(r) plane (one
// contiguous N0*N1*8-byte block) is prefetched into L2 by one bulk
// instruction, so the x rows' loads find it there.
template <int N0, int N1>
__global__ void __maxnreg__(112)
kxy_lane_fwd(float2* __restrict__ zbuf, DeviceSticks g, const double2* __restrict__ twx_g,
             const double2* __restrict__ twy_g, const float* __restrict__ v,
             const float2* __restrict__ psir, int pair0, int npairs, int pairs_per_cta) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  int* xmap = reinterpret_cast<int*>(P + (size_t)ncol * LD);
  const int z = blockIdx.x;
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
  constexpr size_t kPlane = (size_t)N1 * N0;
  auto psir_plane = [&](int pl) { return psir + ((size_t)(pair0 + pl) * g.n2 + z) * kPlane; };
  if (threadIdx.x == 0 && pbeg < pend) prefetch_l2(psir_plane(pbeg), (unsigned)(kPlane * sizeof(C)));
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  __syncthreads();
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
  if (threadIdx.x == 0 && pl + 1 < pend)
    prefetch_l2(psir_plane(pl + 1), (unsigned)(kPlane * sizeof(C)));
  C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
  const C* pp = psir_plane(pl) + tx;
#pragma unroll 1
  for (int base = 0; base < N1; base += sx) {
    const int y = base + gx;
    const bool ok = y < N1;
    C val[MX];
    const C* prow = pp + (size_t)(ok ? y : 0) * N0;
    const float* vrow = v + ((size_t)z * N1 + (ok ? y : 0)) * N0 + MX * mrx;
#pragma unroll
    for (int k = 0; k < MX; ++k) {
      const C p = ok ? prow[k * TX] : cmk<C>(0.0, 0.0);
      const float vv = ok ? vrow[k] : 0.f;
      val[k] = cmk<C>(p.x * vv, p.y * vv);
    }
    lane::line_r2n<TX, MX, -1>(val, tx, twx);
    if (ok) {
      int txh = tx;
      asm volatile("" : "+r"(txh));
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        if (cidx >= 0) P[cidx * LD + y] = val[k];
      }
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int base = 0; base < ncol; base += sy) {
    const int cidx = base + gy;
    const bool ok = cidx < ncol;
    const C* col = P + (ok ? cidx : 0) * LD;
    C val[MY];
#pragma unroll
    for (int k2 = 0; k2 < MY; ++k2) val[k2] = ok ? col[k2 + MY * mry] : cmk<C>(0.0, 0.0);
    lane::line_r2n<TY, MY, -1>(val, ty, twy);
    if (ok) {
      const int* cm = g.colmap + (size_t)cidx * N1;
#pragma unroll
      for (int k = 0; k < MY; ++k) {
        const int s = __ldg(cm + ty + TY * k);
        if (s >= 0) zp[s] = val[k];
      }
    }
  }
  __syncthreads();   // the y columns are read out of P before the next pair's x rows
  }
}

// The same H*psi pass with each round of x rows (blockDim/T rows of psi(r)
// and of V(r)) staged in shared memory by cp.async: while a round's line
// transforms run from registers, the next round's rows (or the next band
// pair's first rows) stream in, so the loads of psi(r) no longer stall the
// transforms.  One CTA per SM (at 140^3 the tables, the column tile and a
// 72-row stage take 197 080 bytes).
template <int N0, int N1>
__host__ size_t xyfs_smem_bytes(int ncol, int rows) {
  return sizeof(float2) * ((size_t)N0 + N1 + (size_t)ncol * pitch(N1)) + sizeof(int) * (size_t)N0 +
         (sizeof(float2) + sizeof(float)) * (size_t)N0 * rows;
}

template <int N0, int N1, bool PRUNE = false>
__global__ void __launch_bounds__(288, 1)
kxy_lane_fwd_staged(float2* __restrict__ zbuf, DeviceSticks g, const double2* __restrict__ twx_g,
                    const double2* __restrict__ twy_g, const float* __restrict__ v,
                    const float2* __restrict__ psir, int pair0, int npairs, int pairs_per_cta) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  static_assert((N0 * sizeof(float)) % 16 == 0, "rows of V(r) must be whole 16-byte chunks");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  const int sx = blockDim.x / TX;                 // rows per round
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* Sp = twy + N1;                               // staged psi(r) rows: sx x N0
  float* Sv = reinterpret_cast<float*>(Sp + (size_t)sx * N0);   // staged V rows
  C* P = reinterpret_cast<C*>(Sv + (size_t)sx * N0);
  int* xmap = reinterpret_cast<int*>(P + (size_t)ncol * LD);
  const int z = blockIdx.x;
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
  constexpr size_t kPlane = (size_t)N1 * N0;
  constexpr int kChunkP = N0 * (int)sizeof(C) / 16, kChunkV = N0 * (int)sizeof(float) / 16;
  // rows y0 .. y0+sx-1 of pair pl into the stage (16-byte chunks)
  auto stage = [&](int pl, int y0) {
    const int nr = min(sx, N1 - y0);
    const char* gp = reinterpret_cast<const char*>(psir + ((size_t)(pair0 + pl) * g.n2 + z) * kPlane +
                                                   (size_t)y0 * N0);
    const char* gv = reinterpret_cast<const char*>(v + ((size_t)z * N1 + y0) * N0);
    char* sp = reinterpret_cast<char*>(Sp);
    char* sv = reinterpret_cast<char*>(Sv);
    for (int i = threadIdx.x; i < nr * kChunkP; i += blockDim.x) {
      const unsigned s = (unsigned)__cvta_generic_to_shared(sp + 16 * (size_t)i);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gp + 16 * (size_t)i)
                   : "memory");
    }
    for (int i = threadIdx.x; i < nr * kChunkV; i += blockDim.x) {
      const unsigned s = (unsigned)__cvta_generic_to_shared(sv + 16 * (size_t)i);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gv + 16 * (size_t)i)
                   : "memory");
    }
    cp_async_commit();
  };
  if (pbeg < pend) stage(pbeg, 0);
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
#pragma unroll 1
    for (int y0 = 0; y0 < N1; y0 += sx) {
      cp_async_wait_all();
      __syncthreads();   // the round is staged; P and xmap are ready
      const int y = y0 + gx;
      const bool ok = y < N1;
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const C p = ok ? Sp[gx * N0 + tx + TX * k] : cmk<C>(0.0, 0.0);
        const float vv = ok ? Sv[gx * N0 + MX * mrx + k] : 0.f;
        val[k] = cmk<C>(p.x * vv, p.y * vv);
      }
      __syncthreads();   // the stage is free: queue the next round under this one's transforms
      if (y0 + sx < N1) stage(pl, y0 + sx);
      else if (pl + 1 < pend) stage(pl + 1, 0);
      lane::line_r2n<TX, MX, -1>(val, tx, twx);
      if (ok) {
        int txh = tx;
        asm volatile("" : "+r"(txh));
#pragma unroll
        for (int k = 0; k < MX; ++k) {
          if (PRUNE && !keep_reg<N0, TX>(k)) continue;   // no column there
          const int cidx = xmap[txh + TX * k];
          if (cidx >= 0) P[cidx * LD + y] = val[k];
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      const C* col = P + (ok ? cidx : 0) * LD;
      C val[MY];
#pragma unroll
      for (int k2 = 0; k2 < MY; ++k2) val[k2] = ok ? col[k2 + MY * mry] : cmk<C>(0.0, 0.0);
      lane::line_r2n<TY, MY, -1>(val, ty, twy);
      if (ok) {
        const int* cm = g.colmap + (size_t)cidx * N1;
#pragma unroll
        for (int k = 0; k < MY; ++k) {
          if (PRUNE && !keep_reg<N1, TY>(k)) continue;   // no stick there
          const int s = __ldg(cm + ty + TY * k);
          if (s >= 0) zp[s] = val[k];
        }
      }
    }
  }
  cp_async_wait_all();
}

template <int N0, int N1, int OP, int SHAPE>
__global__ void __launch_bounds__(lane_threads(SHAPE), lane_minblocks(SHAPE))
kxy_lane(
float2* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
         const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
         const float* __restrict__ v, double* __restrict__ rho, const double* __restrict__ w,
         int pair0, int nst, float2* __restrict__ psir) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  constexpr bool DENS = (OP == XY_DENSITY);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  float* acc = reinterpret_cast<float*>(P + (size_t)ncol * LD);
  int* xmap = reinterpret_cast<int*>(acc + (DENS ? (size_t)N0 * N1 : 0));
  const int z = blockIdx.x;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  if constexpr (DENS)
    for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
    for (int t = threadIdx.x; t < ncol * LD; t += blockDim.x) P[t] = cmk<C>(0.0, 0.0);
    __syncthreads();
    for (int s = threadIdx.x; s < nvec; s += blockDim.x)
      P[g.stick_col[s] * LD + g.stick_y[s]] = zp[s];
    __syncthreads();
    // backward y on the occupied columns, natural in, m-distributed out
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      C* col = P + (ok ? cidx : 0) * LD;
      C val[MY];
#pragma unroll
      for (int k = 0; k < MY; ++k) val[k] = ok ? col[ty + TY * k] : cmk<C>(0.0, 0.0);
      lane::line_n2r<TY, MY, +1>(val, ty, twy);
      if (ok) {
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) col[k2 + MY * mry] = val[k2];
      }
    }
    __syncthreads();
    double w1 = 0.0, w2 = 0.0;
    if (DENS) {
      const int b1 = 2 * (pair0 + pl);
      w1 = w[b1];
      w2 = (b1 + 1 < nst) ? w[b1 + 1] : 0.0;
    }
    const float f1 = (float)w1, f2 = (float)w2;
    // x rows
#pragma unroll 1
    for (int base = 0; base < N1; base += sx) {
      const int y = base + gx;
      const bool ok = y < N1;
      // the column map lookups depend only on the lane: hidden from the
      // optimiser so that they are not kept in MX registers across rows
      int txh = tx;
      asm volatile("" : "+r"(txh));
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        val[k] = (ok && cidx >= 0) ? P[cidx * LD + y] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TX, MX, +1>(val, tx, twx);
      if constexpr (DENS) {
        if (psir && ok) store_psir<N0, N1, TX, MX>(psir, pair0 + pl, g.n2, z, y, tx, val);
        if (ok) {
          float* arow = acc + y * N0 + MX * mrx;
#pragma unroll
          for (int k2 = 0; k2 < MX; ++k2)
            arow[k2] += f1 * val[k2].x * val[k2].x + f2 * val[k2].y * val[k2].y;
        }
      } else {
        const float* vrow = v + ((size_t)z * N1 + (ok ? y : 0)) * N0 + MX * mrx;
        // keep the V loads after the transform: hoisted above it they would
        // hold MX more registers through it
        asm volatile("" ::: "memory");
#pragma unroll
        for (int k2 = 0; k2 < MX; ++k2) {
          const float vv = ok ? vrow[k2] : 0.f;
          val[k2].x *= vv;
          val[k2].y *= vv;
        }
        lane::line_r2n<TX, MX, -1>(val, tx, twx);
        if (ok) {
          asm volatile("" : "+r"(txh));
#pragma unroll
          for (int k = 0; k < MX; ++k) {
            const int cidx = xmap[txh + TX * k];
            if (cidx >= 0) P[cidx * LD + y] = val[k];
          }
        }
      }
    }
    __syncthreads();
    if constexpr (!DENS) {
      // forward y, m-distributed in, natural out
#pragma unroll 1
      for (int base = 0; base < ncol; base += sy) {
        const int cidx = base + gy;
        const bool ok = cidx < ncol;
        C* col = P + (ok ? cidx : 0) * LD;
        C val[MY];
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) val[k2] = ok ? col[k2 + MY * mry] : cmk<C>(0.0, 0.0);
        lane::line_r2n<TY, MY, -1>(val, ty, twy);
        if (ok) {
#pragma unroll
          for (int k = 0; k < MY; ++k) col[ty + TY * k] = val[k];
        }
      }
      __syncthreads();
      for (int s = threadIdx.x; s < nvec; s += blockDim.x)
        zp[s] = P[g.stick_col[s] * LD + g.stick_y[s]];
      __syncthreads();
    }
  }
  if constexpr (DENS) {
    __syncthreads();
    const size_t pbase = (size_t)z * N1 * N0;
    for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) atomicAdd(&rho[pbase + t], (double)acc[t]);
  }
}

// ------------------------------------------------------------ H*psi,
// sticks read and written through the column map
// The H*psi plane pass of kxy_lane<VPSI> with the tile's traffic to the
// sticks taken out: the backward y transform of each occupied column loads
// its inputs straight from the stick buffer through the (column, y) ->
// stick map, and the forward y transform stores its outputs straight back
// the same way.  Per band pair this drops the zero fill of the tile, the
// scatter of the sticks into it and the gather out of it, and three of the
// six CTA barriers.  288 threads, MINB CTAs per SM (2: registers capped at
// 113, lane shape 5; 1: uncapped, lane shape 6).
template <int N0, int N1, int MINB>
__global__ void __launch_bounds__(288, MINB)
kxy_lane_map(float2* __restrict__ zbuf, int npairs, DeviceSticks g,
             const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
             const float* __restrict__ v) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  int* xmap = reinterpret_cast<int*>(P + (size_t)ncol * LD);
  const int z = blockIdx.x, pl = blockIdx.y;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
  (void)npairs;
  // backward y on the occupied columns, inputs from the sticks
#pragma unroll 1
  for (int base = 0; base < ncol; base += sy) {
    const int cidx = base + gy;
    const bool ok = cidx < ncol;
    const int* cm = g.colmap + (size_t)(ok ? cidx : 0) * N1;
    C val[MY];
#pragma unroll
    for (int k = 0; k < MY; ++k) {
      const int s = ok ? __ldg(cm + ty + TY * k) : -1;
      val[k] = s >= 0 ? zp[s] : cmk<C>(0.0, 0.0);
    }
    lane::line_n2r<TY, MY, +1>(val, ty, twy);
    if (ok) {
      C* col = P + cidx * LD;
#pragma unroll
      for (int k2 = 0; k2 < MY; ++k2) col[k2 + MY * mry] = val[k2];
    }
  }
  __syncthreads();
  // x rows: backward, times V(r), forward
#pragma unroll 1
  for (int base = 0; base < N1; base += sx) {
    const int y = base + gx;
    const bool ok = y < N1;
    int txh = tx;
    asm volatile("" : "+r"(txh));
    C val[MX];
#pragma unroll
    for (int k = 0; k < MX; ++k) {
      const int cidx = xmap[txh + TX * k];
      val[k] = (ok && cidx >= 0) ? P[cidx * LD + y] : cmk<C>(0.0, 0.0);
    }
    lane::line_n2r<TX, MX, +1>(val, tx, twx);
    const float* vrow = v + ((size_t)z * N1 + (ok ? y : 0)) * N0 + MX * mrx;
    asm volatile("" ::: "memory");
#pragma unroll
    for (int k2 = 0; k2 < MX; ++k2) {
      const float vv = ok ? vrow[k2] : 0.f;
      val[k2].x *= vv;
      val[k2].y *= vv;
    }
    lane::line_r2n<TX, MX, -1>(val, tx, twx);
    if (ok) {
      asm volatile("" : "+r"(txh));
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        if (cidx >= 0) P[cidx * LD + y] = val[k];
      }
    }
  }
  __syncthreads();
  // forward y, outputs to the sticks
#pragma unroll 1
  for (int base = 0; base < ncol; base += sy) {
    const int cidx = base + gy;
    const bool ok = cidx < ncol;
    const C* col = P + (ok ? cidx : 0) * LD;
    C val[MY];
#pragma unroll
    for (int k2 = 0; k2 < MY; ++k2) val[k2] = ok ? col[k2 + MY * mry] : cmk<C>(0.0, 0.0);
    lane::line_r2n<TY, MY, -1>(val, ty, twy);
    if (ok) {
      const int* cm = g.colmap + (size_t)cidx * N1;
#pragma unroll
      for (int k = 0; k < MY; ++k) {
        const int s = __ldg(cm + ty + TY * k);
        if (s >= 0) zp[s] = val[k];
      }
    }
  }
}

template <int N0, int N1>
__host__ size_t xym_smem_bytes(int ncol) {
  return sizeof(float2) * ((size_t)N0 + N1 + (size_t)ncol * pitch(N1)) + sizeof(int) * (size_t)N0;
}

// ------------------------------------------------------------ density,
// sticks read through the column map
// The density pass of kxy_lane<DENSITY> (whole plane, FP32 accumulator in
// shared memory) with the y inputs loaded straight from the stick buffer
// through the column map: no zero fill of the tile and no scatter of the
// sticks per band pair.  320 threads, one CTA per SM (density shape 6).
template <int N0, int N1>
__global__ void __launch_bounds__(320, 1)
kxy_lane_dmap(const float2* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
              const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
              double* __restrict__ rho, const double* __restrict__ w, int pair0, int nst,
              float2* __restrict__ psir) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  float* acc = reinterpret_cast<float*>(P + (size_t)ncol * LD);
  int* xmap = reinterpret_cast<int*>(acc + (size_t)N0 * N1);
  const int z = blockIdx.x;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    const C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      const int* cm = g.colmap + (size_t)(ok ? cidx : 0) * N1;
      C val[MY];
#pragma unroll
      for (int k = 0; k < MY; ++k) {
        const int sidx = ok ? __ldg(cm + ty + TY * k) : -1;
        val[k] = sidx >= 0 ? zp[sidx] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TY, MY, +1>(val, ty, twy);
      if (ok) {
        C* col = P + cidx * LD;
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) col[k2 + MY * mry] = val[k2];
      }
    }
    __syncthreads();
    const int b1 = 2 * (pair0 + pl);
    const float f1 = (float)w[b1];
    const float f2 = (b1 + 1 < nst) ? (float)w[b1 + 1] : 0.f;
#pragma unroll 1
    for (int base = 0; base < N1; base += sx) {
      const int y = base + gx;
      const bool ok = y < N1;
      int txh = tx;
      asm volatile("" : "+r"(txh));
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        val[k] = (ok && cidx >= 0) ? P[cidx * LD + y] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TX, MX, +1>(val, tx, twx);
      if (psir && ok) store_psir<N0, N1, TX, MX>(psir, pair0 + pl, g.n2, z, y, tx, val);
      if (ok) {
        float* arow = acc + y * N0 + MX * mrx;
#pragma unroll
        for (int k2 = 0; k2 < MX; ++k2)
          arow[k2] += f1 * val[k2].x * val[k2].x + f2 * val[k2].y * val[k2].y;
      }
    }
    __syncthreads();
  }
  const size_t pbase = (size_t)z * N1 * N0;
  for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) atomicAdd(&rho[pbase + t], (double)acc[t]);
}

// ------------------------------------------------------------ density,
// next band pair's sticks queued during the x rows
// The density pass of kxy_lane<DENSITY> (whole plane, FP32 accumulator in
// shared memory, psi(r) optionally stored) with two tiles: P holds the
// sticks of a pair at their (column, y) places and zeros everywhere else,
// and the backward y transform writes its output to a second tile Q instead
// of in place.  P's zeros therefore survive, so P is cleared once per CTA
// instead of once per pair, and as soon as the y transform has read P the
// next pair's sticks are copied into it with cp.async (8 bytes per stick,
// straight to its place in the tile) while the x rows of the current pair
// run from Q.  Each thread keeps the tile offsets of its sticks in
// registers (at most kDqSticks per thread).  Density shape 8: 288 threads,
// one CTA per SM; at 140^3 the two tiles, the accumulator and the tables
// take 227 840 of the 232 448 bytes a CTA may hold.
constexpr int kDqSticks = 16;


template <int N0, int N1>
__host__ size_t xydq_smem_bytes(int ncol) {
  return sizeof(float2) * ((size_t)N0 + N1 + (size_t)2 * ncol * pitch(N1)) +
         sizeof(float) * (size_t)N0 * N1 + sizeof(int) * (size_t)N0;
}

template <int N0, int N1, bool PRUNE = false>
__global__ void __launch_bounds__(288, 1)
kxy_lane_dq(const float2* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
            const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
            double* __restrict__ rho, const double* __restrict__ w, int pair0, int nst,
            float2* __restrict__ psir) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  C* Q = P + (size_t)ncol * LD;
  float* acc = reinterpret_cast<float*>(Q + (size_t)ncol * LD);
  int* xmap = reinterpret_cast<int*>(acc + (size_t)N0 * N1);
  const int z = blockIdx.x;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) acc[t] = 0.f;
  for (int t = threadIdx.x; t < ncol * LD; t += blockDim.x) P[t] = cmk<C>(0.0, 0.0);
  // tile offsets of this thread's sticks s = threadIdx.x + j * blockDim.x
  int soff[kDqSticks];
#pragma unroll
  for (int j = 0; j < kDqSticks; ++j) {
    const int s = threadIdx.x + j * blockDim.x;
    soff[j] = s < nvec ? g.stick_col[s] * LD + g.stick_y[s] : -1;
  }
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
  auto queue_sticks = [&](int pl) {
    const C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec + threadIdx.x;
#pragma unroll
    for (int j = 0; j < kDqSticks; ++j)
      if (soff[j] >= 0) cp_async8(P + soff[j], zp + (size_t)j * blockDim.x);
    cp_async_commit();
  };
  if (pbeg < pend) queue_sticks(pbeg);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    cp_async_wait_all();
    __syncthreads();   // P holds pair pl's sticks; the previous x rows are done with Q
    // backward y on the occupied columns: P (natural) -> Q (m-distributed)
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      const C* col = P + (ok ? cidx : 0) * LD;
      C val[MY];
#pragma unroll
      for (int k = 0; k < MY; ++k)
        val[k] = ok && (!PRUNE || keep_reg<N1, TY>(k)) ? col[ty + TY * k] : cmk<C>(0.0, 0.0);
      lane::line_n2r<TY, MY, +1>(val, ty, twy);
      if (ok) {
        C* qcol = Q + cidx * LD;
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) qcol[k2 + MY * mry] = val[k2];
      }
    }
    __syncthreads();   // P is free: the next pair's sticks stream in under the x rows
    if (pl + 1 < pend) queue_sticks(pl + 1);
    const int b1 = 2 * (pair0 + pl);
    const float f1 = (float)w[b1];
    const float f2 = (b1 + 1 < nst) ? (float)w[b1 + 1] : 0.f;
#pragma unroll 1
    for (int base = 0; base < N1; base += sx) {
      const int y = base + gx;
      const bool ok = y < N1;
      int txh = tx;
      asm volatile("" : "+r"(txh));
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        if (PRUNE && !keep_reg<N0, TX>(k)) {   // no column there
          val[k] = cmk<C>(0.0, 0.0);
          continue;
        }
        const int cidx = xmap[txh + TX * k];
        val[k] = (ok && cidx >= 0) ? Q[cidx * LD + y] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TX, MX, +1>(val, tx, twx);
      if (psir && ok) store_psir<N0, N1, TX, MX>(psir, pair0 + pl, g.n2, z, y, tx, val);
      if (ok) {
        float* arow = acc + y * N0 + MX * mrx;
#pragma unroll
        for (int k2 = 0; k2 < MX; ++k2)
          arow[k2] += f1 * val[k2].x * val[k2].x + f2 * val[k2].y * val[k2].y;
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const size_t pbase = (size_t)z * N1 * N0;
  for (int t = threadIdx.x; t < N0 * N1; t += blockDim.x) atomicAdd(&rho[pbase + t], (double)acc[t]);
}

// ------------------------------------------------------------ density,
// accumulator in tensor memory
// The density pass of kxy_lane<DENSITY> with the FP32 accumulator held in
// tensor memory (TMEM) instead of shared memory.  A thread accumulates the
// same points for every band pair (its rows base + gx, its columns
// MX*bitrev(tx) + k), so each thread keeps them in its own TMEM lane: warp w
// owns lanes 32*(w%4) .. +31 and a block of columns chosen by w/4, and
// reads, adds and writes 8 columns at a time (tcgen05.ld/st .32x32b.x8).
// Freed of the 78 KB shared accumulator, two CTAs fit per SM, each
// allocating 256 of the SM's 512 TMEM columns.  Density shape 7.
// load without waiting: r is valid only after tm_wait_ld(r)
__device__ __forceinline__ void tm_ld8_async(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
// waits for this thread's loads; r passes through the wait so that no use of
// it is scheduled before it
__device__ __forceinline__ void tm_wait_ld(uint32_t (&r)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7])
               :
               : "memory");
}
__device__ __forceinline__ void tm_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  tm_ld8_async(taddr, r);
  tm_wait_ld(r);
}
__device__ __forceinline__ void tm_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
               "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void tm_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

constexpr int kTmemCols = 256;   // TMEM columns per density CTA (two CTAs per SM)

// TMEM columns per row round of a thread: MX rounded up to the 8-column access
__host__ __device__ constexpr int tm_round_cols(int mx) { return (mx + 7) / 8 * 8; }

template <int N0, int N1>
__global__ void __maxnreg__(112)
kxy_lane_dtm(const float2* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
             const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
             double* __restrict__ rho, const double* __restrict__ w, int pair0, int nst) {
  using C = float2;
  constexpr int LD = pitch(N1);
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  constexpr int CW = tm_round_cols(MX), NCH = CW / 8;
  static_assert(TY > 0 && TX > 0, "no register plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  int* xmap = reinterpret_cast<int*>(P + (size_t)ncol * LD);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(xmap + N0);
  const int z = blockIdx.x;
  const int warp = threadIdx.x >> 5;
  const int sx = blockDim.x / TX;
  const int R = (N1 + sx - 1) / sx;       // row rounds per thread
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = *tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) +
                         (uint32_t)((warp >> 2) * R * CW);
  {
    const uint32_t zr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = 0; q < R * NCH; ++q) tm_st8(tbase + 8 * q, zr);
    tm_wait_st();
  }
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    const C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
    for (int t = threadIdx.x; t < ncol * LD; t += blockDim.x) P[t] = cmk<C>(0.0, 0.0);
    __syncthreads();
    for (int s2 = threadIdx.x; s2 < nvec; s2 += blockDim.x)
      P[g.stick_col[s2] * LD + g.stick_y[s2]] = zp[s2];
    __syncthreads();
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      C* col = P + (ok ? cidx : 0) * LD;
      C val[MY];
#pragma unroll
      for (int k = 0; k < MY; ++k) val[k] = ok ? col[ty + TY * k] : cmk<C>(0.0, 0.0);
      lane::line_n2r<TY, MY, +1>(val, ty, twy);
      if (ok) {
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) col[k2 + MY * mry] = val[k2];
      }
    }
    __syncthreads();
    const int b1 = 2 * (pair0 + pl);
    const float f1 = (float)w[b1];
    const float f2 = (b1 + 1 < nst) ? (float)w[b1 + 1] : 0.f;
    // every warp runs all R rounds (the TMEM accesses are warp-wide); rows
    // past the end carry zeros
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      const int y = r * sx + gx;
      const bool ok = y < N1;
      int txh = tx;
      asm volatile("" : "+r"(txh));
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        val[k] = (ok && cidx >= 0) ? P[cidx * LD + y] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TX, MX, +1>(val, tx, twx);
      // read-add-write 8 columns at a time, the next chunk's load in
      // flight while this one is added
      const uint32_t trow = tbase + (uint32_t)(r * CW);
      uint32_t a[8], nx[8];
      tm_ld8(trow, a);
#pragma unroll
      for (int c8 = 0; c8 < NCH; ++c8) {
        if (c8 + 1 < NCH) tm_ld8_async(trow + 8 * (c8 + 1), nx);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int k2 = 8 * c8 + j;
          if (k2 < MX)
            a[j] = __float_as_uint(__uint_as_float(a[j]) + f1 * val[k2].x * val[k2].x +
                                   f2 * val[k2].y * val[k2].y);
        }
        tm_st8(trow + 8 * c8, a);
        if (c8 + 1 < NCH) {
          tm_wait_ld(nx);
#pragma unroll
          for (int j = 0; j < 8; ++j) a[j] = nx[j];
        }
      }
    }
    tm_wait_st();
    __syncthreads();
  }
  // add this CTA's accumulators to the density
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    const int y = r * sx + gx;
#pragma unroll
    for (int c8 = 0; c8 < NCH; ++c8) {
      uint32_t a[8];
      tm_ld8(tbase + (uint32_t)(r * CW + 8 * c8), a);
      if (y < N1) {
        double* out = rho + ((size_t)z * N1 + y) * N0 + MX * mrx;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int k2 = 8 * c8 + j;
          if (k2 < MX) atomicAdd(out + k2, (double)__uint_as_float(a[j]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// ------------------------------------------------------------ density,
// half planes
// The density pass of kxy_lane over one half of a plane's rows per CTA
// (blockIdx.z = 0, 1).  Each half transforms every occupied column along y,
// its inputs gathered straight from the stick buffer through the
// (column, y) -> stick map, keeps the rows it owns (whole lanes of the
// register distribution: lane ty holds rows MY*bitrev(ty) + k), transforms
// those rows along x and accumulates f/Omega |psi|^2 into an FP32 half
// plane.  Half the tile and half the accumulator fit two CTAs per SM, for
// about 1.3x the line transforms of the whole-plane kernel.
// shared memory: [twx N0][twy N1][P ncol x pitch(N1/2)][FP32 half plane
// N1/2 x N0][xmap N0 ints]
template <int N0, int N1>
__host__ size_t xyh_smem_bytes(int ncol) {
  constexpr int H = N1 / 2;
  return sizeof(float2) * ((size_t)N0 + N1 + (size_t)ncol * pitch(H)) +
         sizeof(float) * (size_t)H * N0 + sizeof(int) * (size_t)N0;
}

template <int N0, int N1>
__global__ void __launch_bounds__(288, 2)
kxy_lane_dh(const float2* __restrict__ zbuf, int npairs, int pairs_per_cta, DeviceSticks g,
            const double2* __restrict__ twx_g, const double2* __restrict__ twy_g,
            double* __restrict__ rho, const double* __restrict__ w, int pair0, int nst) {
  using C = float2;
  constexpr int TY = lane::lanes_for(N1), MY = N1 / TY;
  constexpr int TX = lane::lanes_for(N0), MX = N0 / TX;
  constexpr int H = N1 / 2, LDH = pitch(H);
  static_assert(TX > 0 && (TY == 2 || TY == 4) && N1 % 2 == 0,
                "no half-plane plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ncol = g.ncol, nvec = g.nvec;
  C* twx = reinterpret_cast<C*>(smem_raw);
  C* twy = twx + N0;
  C* P = twy + N1;
  float* acc = reinterpret_cast<float*>(P + (size_t)ncol * LDH);
  int* xmap = reinterpret_cast<int*>(acc + (size_t)H * N0);
  const int z = blockIdx.x, y0 = blockIdx.z * H;
  load_tw(twx, twx_g, N0);
  load_tw(twy, twy_g, N1);
  for (int x = threadIdx.x; x < N0; x += blockDim.x) xmap[x] = -1;
  for (int t = threadIdx.x; t < H * N0; t += blockDim.x) acc[t] = 0.f;
  __syncthreads();
  for (int cidx = threadIdx.x; cidx < ncol; cidx += blockDim.x) xmap[g.col_x[cidx]] = cidx;
  const int ty = threadIdx.x % TY, gy = threadIdx.x / TY, sy = blockDim.x / TY;
  const int tx = threadIdx.x % TX, gx = threadIdx.x / TX, sx = blockDim.x / TX;
  const int mry = lane::bitrev(ty, TY), mrx = lane::bitrev(tx, TX);
  const bool keep = (MY * mry >= y0) && (MY * mry < y0 + H);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
#pragma unroll 1
  for (int pl = pbeg; pl < pend; ++pl) {
    const C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
    // backward y on the occupied columns, inputs gathered from the sticks
#pragma unroll 1
    for (int base = 0; base < ncol; base += sy) {
      const int cidx = base + gy;
      const bool ok = cidx < ncol;
      const int* cm = g.colmap + (size_t)(ok ? cidx : 0) * N1;
      C val[MY];
#pragma unroll
      for (int k = 0; k < MY; ++k) {
        const int s = ok ? __ldg(cm + ty + TY * k) : -1;
        val[k] = s >= 0 ? zp[s] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TY, MY, +1>(val, ty, twy);
      if (ok && keep) {
        C* col = P + cidx * LDH + (MY * mry - y0);
#pragma unroll
        for (int k2 = 0; k2 < MY; ++k2) col[k2] = val[k2];
      }
    }
    __syncthreads();
    const int b1 = 2 * (pair0 + pl);
    const float f1 = (float)w[b1];
    const float f2 = (b1 + 1 < nst) ? (float)w[b1 + 1] : 0.f;
    // backward x on this half's rows
#pragma unroll 1
    for (int base = 0; base < H; base += sx) {
      const int yl = base + gx;
      const bool ok = yl < H;
      int txh = tx;
      asm volatile("" : "+r"(txh));
      C val[MX];
#pragma unroll
      for (int k = 0; k < MX; ++k) {
        const int cidx = xmap[txh + TX * k];
        val[k] = (ok && cidx >= 0) ? P[cidx * LDH + yl] : cmk<C>(0.0, 0.0);
      }
      lane::line_n2r<TX, MX, +1>(val, tx, twx);
      if (ok) {
        float* arow = acc + yl * N0 + MX * mrx;
#pragma unroll
        for (int k2 = 0; k2 < MX; ++k2)
          arow[k2] += f1 * val[k2].x * val[k2].x + f2 * val[k2].y * val[k2].y;
      }
    }
    __syncthreads();
  }
  const size_t pbase = ((size_t)z * N1 + y0) * N0;
  for (int t = threadIdx.x; t < H * N0; t += blockDim.x) atomicAdd(&rho[pbase + t], (double)acc[t]);
}

// ------------------------------------------------------------ launch
// Arguments of one batch of band pairs through the specialised kernels.
struct StagedArgs {
  int op;                  // XY_DENSITY or XY_VPSI
  const double* c;         // coefficients (device, default order)
  const void* v;           // V(r): float (mixed) or double (FP64); VPSI only
  double* rho;             // density grid (DENSITY)
  const double* w;         // occ/Omega per band (DENSITY)
  double* hc;              // output H*psi (VPSI)
  int nst, pair0, npairs;
  void* zbuf;
  const double2 *twx, *twy, *twz;
  int rods_per_cta;        // z kernels
  int xy_warps;            // requested warps per kxy CTA
  int vpsi_shape;          // FP32 H*psi plane CTA shape (xy_threads / xy_minblocks)
  int lane_shape;          // FP32 register-lane plane kernel shape, -1 = not used
  int density_lane_shape;  // its density-pass shape (2, 3; 5 = half planes)
  int density_chunks;      // CTAs per plane in the density pass
  float2* psir;            // DENSITY: store psi(r) here; VPSI: read it (skip the backward)
  int fwd_pairs_per_cta;   // VPSI from psi(r): band pairs per CTA of kxy_lane_fwd
  int fwd_staged;          // VPSI from psi(r): rounds of rows staged by cp.async
  int prune;               // FP32 lane kernels skip the points beyond prune_width
  int zlane;               // FP32 z sticks in register lanes: 0 off; 1 both directions
                           // (backward capped for 2 CTAs per SM); 2 both, uncapped; 3
                           // forward only
};

// the pruned plane kernels need every stick column and stick row within
// prune_width of 0, the pruned z kernels every rod
template <int N> bool xy_prunable(const StagedArgs& a, const DeviceSticks& g) {
  return a.prune && g.xw <= prune_width(N) && g.yw <= prune_width(N);
}
template <int N> bool z_prunable(const StagedArgs& a, const DeviceSticks& g) {
  return a.prune && g.zw <= prune_width(N);
}

template <typename T, int N, int SH>
void launch_vpsi_xy(Context& ctx, const StagedArgs& a) {
  using C = typename reg::CT<T>::c;
  const DeviceSticks& g = ctx.dws;
  const int nw = std::min(a.xy_warps, xy_threads(SH) / 32);
  const size_t sm = xy_smem_bytes<T, N, N, XY_VPSI>(g.ncol, nw);
  allow_smem(kxy<T, N, N, XY_VPSI, SH>, sm);
  kxy<T, N, N, XY_VPSI, SH><<<dim3(N, a.npairs), 32 * nw, sm, ctx.stream>>>(
      (C*)a.zbuf, a.npairs, 1, g, a.twx, a.twy, (const T*)a.v, nullptr, nullptr, a.pair0, a.nst);
  QBX_LAUNCHED(ctx);
}

template <int N, int OP, int SH>
void launch_lane_xy(Context& ctx, const StagedArgs& a, int chunks, int ppc) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = xyl_smem_bytes<N, N, OP>(g.ncol);
  allow_smem(kxy_lane<N, N, OP, SH>, sm);
  int threads = lane_threads(SH);
  if (SH == 3 || SH == 4) {
    const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
    threads = std::max(64, std::min(threads, want));
  }
  kxy_lane<N, N, OP, SH><<<dim3(N, chunks), threads, sm, ctx.stream>>>(
      (float2*)a.zbuf, a.npairs, ppc, g, a.twx, a.twy, (const float*)a.v, a.rho, a.w, a.pair0,
      a.nst, OP == XY_DENSITY ? a.psir : nullptr);
  QBX_LAUNCHED(ctx);
}

template <int N, int MINB>
void launch_lane_map(Context& ctx, const StagedArgs& a) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = xym_smem_bytes<N, N>(g.ncol);
  allow_smem(kxy_lane_map<N, N, MINB>, sm);
  const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
  const int threads = std::max(64, std::min(288, want));
  kxy_lane_map<N, N, MINB><<<dim3(N, a.npairs), threads, sm, ctx.stream>>>(
      (float2*)a.zbuf, a.npairs, g, a.twx, a.twy, (const float*)a.v);
  QBX_LAUNCHED(ctx);
}

template <int N>
void launch_lane_fwd(Context& ctx, const StagedArgs& a) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = xym_smem_bytes<N, N>(g.ncol);
  allow_smem(kxy_lane_fwd<N, N>, sm);
  const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
  const int threads = std::max(64, std::min(288, want));
  const int ppc = std::max(1, std::min(a.npairs, a.fwd_pairs_per_cta));
  const int chunks = (a.npairs + ppc - 1) / ppc;
  kxy_lane_fwd<N, N><<<dim3(N, chunks), threads, sm, ctx.stream>>>(
      (float2*)a.zbuf, g, a.twx, a.twy, (const float*)a.v, a.psir, a.pair0, a.npairs, ppc);
  QBX_LAUNCHED(ctx);
}

// false (nothing launched) when the length has no 16-byte row chunks or the
// stage does not fit a CTA's shared memory
template <int N>
bool launch_lane_fwd_staged(Context& ctx, const StagedArgs& a) {
  if constexpr (N % 4 != 0) {
    return false;
  } else {
    const DeviceSticks& g = ctx.dws;
    const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
    const int threads = std::max(64, std::min(288, want));
    const size_t sm = xyfs_smem_bytes<N, N>(g.ncol, threads / lane::lanes_for(N));
    int dev = 0, optin = 0;
    QBX_CUDA(cudaGetDevice(&dev));
    QBX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sm > (size_t)optin) return false;
    const int ppc = std::max(1, std::min(a.npairs, a.fwd_pairs_per_cta));
    const int chunks = (a.npairs + ppc - 1) / ppc;
    auto run = [&](auto kern) {
      allow_smem(kern, sm);
      kern<<<dim3(N, chunks), threads, sm, ctx.stream>>>(
          (float2*)a.zbuf, g, a.twx, a.twy, (const float*)a.v, a.psir, a.pair0, a.npairs, ppc);
    };
    if (xy_prunable<N>(a, g)) run(kxy_lane_fwd_staged<N, N, true>);
    else run(kxy_lane_fwd_staged<N, N, false>);
    QBX_LAUNCHED(ctx);
    return true;
  }
}

template <int N>
void launch_density_map(Context& ctx, const StagedArgs& a, int chunks, int ppc) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = xyl_smem_bytes<N, N, XY_DENSITY>(g.ncol);
  allow_smem(kxy_lane_dmap<N, N>, sm);
  const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
  const int threads = std::max(64, std::min(320, want));
  kxy_lane_dmap<N, N><<<dim3(N, chunks), threads, sm, ctx.stream>>>(
      (const float2*)a.zbuf, a.npairs, ppc, g, a.twx, a.twy, a.rho, a.w, a.pair0, a.nst, a.psir);
  QBX_LAUNCHED(ctx);
}

// false (nothing launched) when the two tiles do not fit a CTA's shared
// memory or a thread would hold more than kDqSticks sticks
template <int N>
bool launch_density_dq(Context& ctx, const StagedArgs& a, int chunks, int ppc) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = xydq_smem_bytes<N, N>(g.ncol);
  const int want = (g.ncol * lane::lanes_for(N) + 31) / 32 * 32;
  const int threads = std::max(64, std::min(288, want));
  int dev = 0, optin = 0;
  QBX_CUDA(cudaGetDevice(&dev));
  QBX_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (sm > (size_t)optin || g.nvec > kDqSticks * threads) return false;
  auto run = [&](auto kern) {
    allow_smem(kern, sm);
    kern<<<dim3(N, chunks), threads, sm, ctx.stream>>>((const float2*)a.zbuf, a.npairs, ppc, g,
                                                       a.twx, a.twy, a.rho, a.w, a.pair0, a.nst,
                                                       a.psir);
  };
  if (xy_prunable<N>(a, g)) run(kxy_lane_dq<N, N, true>);
  else run(kxy_lane_dq<N, N, false>);
  QBX_LAUNCHED(ctx);
  return true;
}

// threads of the TMEM density kernel: one lane group per occupied column,
// at most 288
template <int N>
int density_tmem_threads(const Context& ctx) {
  const int want = (ctx.dws.ncol * lane::lanes_for(N) + 31) / 32 * 32;
  return std::max(64, std::min(288, want));
}

// the TMEM columns every warp needs fit the CTA's 256
template <int N>
bool density_tmem_fits(const Context& ctx) {
  constexpr int TX = lane::lanes_for(N);
  if (TX == 0) return false;
  const int threads = density_tmem_threads<N>(ctx);
  const int sx = threads / TX, R = (N + sx - 1) / sx, nw = threads / 32;
  return ((nw + 3) / 4) * R * tm_round_cols(N / TX) <= kTmemCols;
}

template <int N>
void launch_density_tmem(Context& ctx, const StagedArgs& a, int chunks, int ppc) {
  const DeviceSticks& g = ctx.dws;
  const size_t sm = sizeof(float2) * ((size_t)N + N + (size_t)g.ncol * pitch(N)) +
                    sizeof(int) * (size_t)N + 16;
  allow_smem(kxy_lane_dtm<N, N>, sm);
  const int threads = density_tmem_threads<N>(ctx);
  kxy_lane_dtm<N, N><<<dim3(N, chunks), threads, sm, ctx.stream>>>(
      (const float2*)a.zbuf, a.npairs, ppc, g, a.twx, a.twy, a.rho, a.w, a.pair0, a.nst);
  QBX_LAUNCHED(ctx);
}

template <int N>
constexpr bool density_half_ok() {
  return N % 2 == 0 && lane::lanes_for(N) >= 2 && lane::lanes_for(N) <= 4;
}

template <int N>
void launch_density_half(Context& ctx, const StagedArgs& a, int chunks, int ppc) {
  if constexpr (density_half_ok<N>()) {
    const DeviceSticks& g = ctx.dws;
    const size_t sm = xyh_smem_bytes<N, N>(g.ncol);
    allow_smem(kxy_lane_dh<N, N>, sm);
    const int T = lane::lanes_for(N);
    const int want = std::max((g.ncol * T + 31) / 32 * 32, ((N / 2) * T + 31) / 32 * 32);
    const int threads = std::max(64, std::min(288, want));
    kxy_lane_dh<N, N><<<dim3(N, chunks, 2), threads, sm, ctx.stream>>>(
        (const float2*)a.zbuf, a.npairs, ppc, g, a.twx, a.twy, a.rho, a.w, a.pair0, a.nst);
    QBX_LAUNCHED(ctx);
  }
}

template <typename T, int N>
void run_cubic(Context& ctx, const StagedArgs& a) {
  using C = typename reg::CT<T>::c;
  const DeviceSticks& g = ctx.dws;
  cudaStream_t st = ctx.stream;
  const int ngw = ctx.wb.ng;
  const int rpc = a.rods_per_cta;
  const size_t zs = sizeof(C) * ((size_t)N + (size_t)2 * rpc * pitch(N));
  dim3 zgrid((g.nrods + rpc - 1) / rpc, a.npairs);
  constexpr bool LANE = std::is_same<T, float>::value && lane::lanes_for(N) > 0;
  // psi(r) of these pairs is stored: the H*psi pass needs no backward
  const bool from_psir = LANE && a.op == XY_VPSI && a.psir && a.lane_shape >= 0;
  // z sticks in register lanes: one lane group per stick of the CTA's rods
  const bool zlane = LANE && a.zlane;
  const int zl_threads = std::min(256, (lane::lanes_for(N) * 2 * rpc + 31) / 32 * 32);
  if (!from_psir) {
    ProfScope ps(ctx, "zfft_bwd");
    if constexpr (LANE) {
      if (zlane && a.zlane != 3) {
        auto run = [&](auto kern) {
          kern<<<zgrid, zl_threads, 0, st>>>((const double2*)a.c, ngw, a.nst, a.pair0, g, a.twz,
                                             (float2*)a.zbuf, rpc);
        };
        const bool pz = z_prunable<N>(a, g);
        if (a.zlane == 2) {
          if (pz) run(kz_bwd_lane<N, 1, true>);
          else run(kz_bwd_lane<N, 1, false>);
        } else {
          if (pz) run(kz_bwd_lane<N, 2, true>);
          else run(kz_bwd_lane<N, 2, false>);
        }
        QBX_LAUNCHED(ctx);
      }
    }
    if (!zlane || a.zlane == 3) {
      allow_smem(kz_bwd<T, N>, zs);
      kz_bwd<T, N><<<zgrid, kZThreads, zs, st>>>((const double2*)a.c, ngw, a.nst, a.pair0, g,
                                                 a.twz, (C*)a.zbuf, rpc);
      QBX_LAUNCHED(ctx);
    }
  }
  if constexpr (LANE) {
    if (a.lane_shape >= 0) {
      if (a.op == XY_DENSITY) {
        int chunks = std::max(1, std::min(a.npairs, a.density_chunks));
        const int ppc = (a.npairs + chunks - 1) / chunks;
        chunks = (a.npairs + ppc - 1) / ppc;
        ProfScope ps(ctx, "xy_density");
        // psi(r) is stored by the whole-plane kernels (shapes 2, 3, 6, 8)
        if (a.psir && a.density_lane_shape != 6 && a.density_lane_shape != 2 &&
            a.density_lane_shape != 8)
          launch_lane_xy<N, XY_DENSITY, 3>(ctx, a, chunks, ppc);
        else if (a.density_lane_shape == 8) {
          if (!launch_density_dq<N>(ctx, a, chunks, ppc))
            launch_lane_xy<N, XY_DENSITY, 3>(ctx, a, chunks, ppc);
        }
        else if (a.density_lane_shape == 5 && density_half_ok<N>()) launch_density_half<N>(ctx, a, chunks, ppc);
        else if (a.density_lane_shape == 6) launch_density_map<N>(ctx, a, chunks, ppc);
        else if (a.density_lane_shape == 7 && density_tmem_fits<N>(ctx)) launch_density_tmem<N>(ctx, a, chunks, ppc);
        else if (a.density_lane_shape == 3) launch_lane_xy<N, XY_DENSITY, 3>(ctx, a, chunks, ppc);
        else launch_lane_xy<N, XY_DENSITY, 2>(ctx, a, chunks, ppc);
        return;
      }
      {
        ProfScope ps(ctx, "xy_vpsi");
        if (from_psir) {
          if (!a.fwd_staged || !launch_lane_fwd_staged<N>(ctx, a)) launch_lane_fwd<N>(ctx, a);
        }
        else switch (a.lane_shape) {
          case 5: launch_lane_map<N, 2>(ctx, a); break;
          case 6: launch_lane_map<N, 1>(ctx, a); break;
          case 1: launch_lane_xy<N, XY_VPSI, 1>(ctx, a, a.npairs, 1); break;
          case 2: launch_lane_xy<N, XY_VPSI, 2>(ctx, a, a.npairs, 1); break;
          case 3: launch_lane_xy<N, XY_VPSI, 3>(ctx, a, a.npairs, 1); break;
          case 4: launch_lane_xy<N, XY_VPSI, 4>(ctx, a, a.npairs, 1); break;
          default: launch_lane_xy<N, XY_VPSI, 0>(ctx, a, a.npairs, 1); break;
        }
      }
      const double scale = 1.0 / ((double)N * N * N);
      ProfScope ps(ctx, "zfft_fwd");
      if (zlane) {
        const size_t zls = sizeof(float2) * ((size_t)N + (size_t)2 * rpc * pitch(N));
        auto run = [&](auto kern) {
          allow_smem(kern, zls);
          kern<<<zgrid, zl_threads, zls, st>>>((const float2*)a.zbuf, ngw, a.nst, a.pair0, g,
                                               a.twz, scale, (const double2*)a.c, ctx.d_g2_w,
                                               (double2*)a.hc, rpc);
        };
        if (z_prunable<N>(a, g)) run(kz_fwd_lane<N, true>);
        else run(kz_fwd_lane<N, false>);
      } else {
        allow_smem(kz_fwd<T, N>, zs);
        kz_fwd<T, N><<<zgrid, kZThreads, zs, st>>>((const C*)a.zbuf, ngw, a.nst, a.pair0, g,
                                                   a.twz, scale, (const double2*)a.c, ctx.d_g2_w,
                                                   (double2*)a.hc, rpc);
      }
      QBX_LAUNCHED(ctx);
      return;
    }
  }
  if (a.op == XY_DENSITY) {
    constexpr int SH = XYDefault<T, XY_DENSITY>::shape;
    const int nw = std::min(a.xy_warps, xy_threads(SH) / 32);
    const size_t sm = xy_smem_bytes<T, N, N, XY_DENSITY>(g.ncol, nw);
    allow_smem(kxy<T, N, N, XY_DENSITY, SH>, sm);
    int chunks = std::max(1, std::min(a.npairs, a.density_chunks));
    const int ppc = (a.npairs + chunks - 1) / chunks;
    chunks = (a.npairs + ppc - 1) / ppc;
    ProfScope ps(ctx, "xy_density");
    kxy<T, N, N, XY_DENSITY, SH><<<dim3(N, chunks), 32 * nw, sm, st>>>(
        (C*)a.zbuf, a.npairs, ppc, g, a.twx, a.twy, nullptr, a.rho, a.w, a.pair0, a.nst);
    QBX_LAUNCHED(ctx);
    return;
  }
  {
    ProfScope ps(ctx, "xy_vpsi");
    if constexpr (std::is_same<T, float>::value) {
      if (a.vpsi_shape == 1) launch_vpsi_xy<T, N, 1>(ctx, a);
      else if (a.vpsi_shape == 2) launch_vpsi_xy<T, N, 2>(ctx, a);
      else launch_vpsi_xy<T, N, 0>(ctx, a);
    } else {
      launch_vpsi_xy<T, N, 3>(ctx, a);
    }
  }
  allow_smem(kz_fwd<T, N>, zs);
  const double scale = 1.0 / ((double)N * N * N);
  ProfScope ps(ctx, "zfft_fwd");
  kz_fwd<T, N><<<zgrid, kZThreads, zs, st>>>((const C*)a.zbuf, ngw, a.nst, a.pair0, g, a.twz, scale,
                                             (const double2*)a.c, ctx.d_g2_w, (double2*)a.hc, rpc);
  QBX_LAUNCHED(ctx);
}

template <typename T, int N>
size_t smem_need(const Context& ctx, const StagedArgs& a) {
  const int nwd = std::min(a.xy_warps, xy_threads(XYDefault<T, XY_DENSITY>::shape) / 32);
  const int nwv = std::min(a.xy_warps, xy_threads(std::is_same<T, float>::value ? a.vpsi_shape : 3) / 32);
  const size_t x = std::max(xy_smem_bytes<T, N, N, XY_DENSITY>(ctx.dws.ncol, nwd),
                            xy_smem_bytes<T, N, N, XY_VPSI>(ctx.dws.ncol, nwv));
  const size_t z = sizeof(typename reg::CT<T>::c) * ((size_t)N + (size_t)2 * a.rods_per_cta * pitch(N));
  size_t l = 0;
  if constexpr (std::is_same<T, float>::value && lane::lanes_for(N) > 0)
    if (a.lane_shape >= 0)
      l = std::max(xyl_smem_bytes<N, N, XY_DENSITY>(ctx.dws.ncol),
                   xyl_smem_bytes<N, N, XY_VPSI>(ctx.dws.ncol));
  return std::max(std::max(x, z), l);
}

// ------------------------------------------------------------ full grid
// In-place FP64 FFT of every line along one axis of an n0 x n1 x n2 grid (x
// fastest) whose length along that axis is N.  A CTA copies a tile of
// kGridLines lines into shared memory with coalesced accesses (consecutive
// lines for the x axis; lines at consecutive x for the y and z axes, so each
// row of the tile is one contiguous run of the grid), its warps transform
// the tile's lines in place with the compile-time warp FFT, and the tile is
// copied back.
constexpr int kGridLines = 16;
constexpr int kGridThreads = 256;

template <int N, int DIR>
__global__ void __launch_bounds__(kGridThreads)
k_grid_lines(double2* __restrict__ grid, int n0, int n1, int n2, int axis,
             const double2* __restrict__ tw_g) {
  using C = double2;
  constexpr int L = kGridLines, LD = pitch(N);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + N;
  load_tw(tw, tw_g, N);
  size_t base, estride, lstride;
  int nl;
  if (axis == 0) {
    const int l0 = blockIdx.x * L;
    nl = min(L, n1 * n2 - l0);
    base = (size_t)l0 * N;
    estride = 1;
    lstride = N;
  } else {
    const int xt = (n0 + L - 1) / L;
    const int outer = blockIdx.x / xt, x0 = (blockIdx.x % xt) * L;
    nl = min(L, n0 - x0);
    base = (size_t)x0 + (axis == 1 ? (size_t)n0 * n1 * outer : (size_t)n0 * outer);
    estride = axis == 1 ? (size_t)n0 : (size_t)n0 * n1;
    lstride = 1;
  }
  // x lines: the tile is one contiguous run; y and z: runs of nl along x
  for (int t = threadIdx.x; t < nl * N; t += blockDim.x) {
    int line, e;
    if (axis == 0) { line = t / N; e = t - line * N; }
    else { line = t % nl; e = t / nl; }
    tile[line * LD + e] = grid[base + e * estride + line * lstride];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int l = warp; l < nl; l += nw) {
    C* row = tile + l * LD;
    reg::warp_fft<N, DIR>(row, tw, lane, BufLoad<C>{row}, BufStore<C>{row});
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nl * N; t += blockDim.x) {
    int line, e;
    if (axis == 0) { line = t / N; e = t - line * N; }
    else { line = t % nl; e = t / nl; }
    grid[base + e * estride + line * lstride] = tile[line * LD + e];
  }
}

template <int N>
void run_grid_lines(Context& ctx, double2* grid, int n0, int n1, int n2, int axis, int dir,
                    const double2* tw) {
  const int L = kGridLines;
  const int nblocks = axis == 0 ? (n1 * n2 + L - 1) / L
                                : ((n0 + L - 1) / L) * (axis == 1 ? n2 : n1);
  const size_t smem = sizeof(double2) * ((size_t)N + (size_t)L * pitch(N));
  if (dir > 0) {
    allow_smem(k_grid_lines<N, +1>, smem);
    k_grid_lines<N, +1><<<nblocks, kGridThreads, smem, ctx.stream>>>(grid, n0, n1, n2, axis, tw);
  } else {
    allow_smem(k_grid_lines<N, -1>, smem);
    k_grid_lines<N, -1><<<nblocks, kGridThreads, smem, ctx.stream>>>(grid, n0, n1, n2, axis, tw);
  }
  QBX_LAUNCHED(ctx);
}

}  // namespace fast

// Full-grid line FFTs of the lengths compiled in fft_fast_a.cu / fft_fast_b.cu;
// false when the length along `axis` has no specialised kernel.
bool fast_grid_lines_a(Context& ctx, double2* grid, int n0, int n1, int n2, int axis, int dir,
                       const double2* tw);
bool fast_grid_lines_b(Context& ctx, double2* grid, int n0, int n1, int n2, int axis, int dir,
                       const double2* tw);

// Specialised staged transforms for cubic grids of the lengths compiled in
// fft_fast_a.cu / fft_fast_b.cu; each returns false when it has no kernel
// for the grid, or when its shared memory would not fit.
bool fast_staged_a(Context& ctx, const fast::StagedArgs& a, size_t smem_limit);
bool fast_staged_b(Context& ctx, const fast::StagedArgs& a, size_t smem_limit);

}  // namespace qbx

#define QBX_FAST_CASE(N)                                                      \
  case N:                                                                     \
    if (ctx.precision == MIXED) {                                             \
      if (fast::smem_need<float, N>(ctx, a) > smem_limit) return false;       \
      fast::run_cubic<float, N>(ctx, a);                                      \
    } else {                                                                  \
      if (fast::smem_need<double, N>(ctx, a) > smem_limit) return false;      \
      fast::run_cubic<double, N>(ctx, a);                                     \
    }                                                                         \
    return true;

#define QBX_GRID_CASE(N)                                                      \
  case N:                                                                     \
    fast::run_grid_lines<N>(ctx, grid, n0, n1, n2, axis, dir, tw);            \
    return true;
