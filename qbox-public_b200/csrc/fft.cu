// Staged 3-D FFTs of the electronic step on sm_100a.
//
// Wavefunction transforms (the hot path) never build the full 3-D grid in
// HBM.  A band pair psi_1 + i psi_2 (the reference's two-real-functions
// packing, src/BasisMapping.cpp:667-750) goes through three kernels:
//
//   k_zfft_bwd : gather the coefficients of a few rods, expand them into
//                z-sticks (+G and -G columns), inverse FFT along z in shared
//                memory, write the sticks plane-major  zbuf[pair][z][stick].
//   k_xy       : one CTA per z-plane: scatter that plane's stick values into
//                a compact (x-column x y) tile in shared memory, inverse FFT
//                along y on the occupied columns only, then row by row the
//                inverse FFT along x, and the fused real-space operation:
//                  OP_DENSITY: rho += f1/Omega psi_1^2 + f2/Omega psi_2^2
//                  OP_VPSI:    psi *= V(r), forward x FFT, back into the tile;
//                              forward y FFT, write the plane's sticks back.
//   k_zfft_fwd : forward z FFT of the sticks, unpack the two bands
//                (src/BasisMapping.cpp:722-750), scale by 1/N and write
//                hc = 1/2|G|^2 c + result   (kinetic term fused).
//
// Per band pair the HBM traffic is the coefficients, the sticks written and
// read in each direction and the potential plane: the staged floor.
//
// Density-basis transforms (a handful per step) use the full grid with three
// strided line-FFT passes (k_line_fft).
//
// All 1-D FFTs are mixed-radix (2,3,4,5,7,11) self-sorting Stockham passes
// over shared memory with a twiddle table exp(+2 pi i k/n) built in FP64.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "fft_fast.cuh"
#include "qbx_internal.h"

namespace qbx {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using t = float2; };
template <> struct Cplx<double> { using t = double2; };

template <typename C> __device__ __forceinline__ C mk(double x, double y) {
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
// multiply by DIR * i
template <int DIR, typename C> __device__ __forceinline__ C muli(C a) {
  C r;
  if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}
template <int DIR, typename C> __device__ __forceinline__ C twid(const C* tw, int k) {
  C w = tw[k];
  if (DIR < 0) w.y = -w.y;
  return w;
}

// R-point DFT, out[k] = sum_q v[q] exp(DIR 2 pi i q k / R); roots from the
// length-n table at stride n/R.
template <int R, int DIR, typename C>
__device__ __forceinline__ void small_dft(C* v, const C* tw, int rs) {
  if (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const C c = cadd(v[1], v[3]), d = muli<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  } else {
    C out[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      C acc = v[0];
#pragma unroll
      for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(v[q], twid<DIR>(tw, ((q * k) % R) * rs)));
      out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
  }
}

// One Stockham pass over nlines contiguous lines of length n (line stride ls).
template <int R, int DIR, typename C>
__device__ __forceinline__ void stockham_pass(const C* __restrict__ src, C* __restrict__ dst,
                                              int n, int nlines, int ls, int Ns, const C* tw) {
  const int nb = n / R;
  const int total = nlines * nb;
  const int tws = n / (Ns * R);
  const int rs = n / R;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t / nb;
    const int i = t - line * nb;
    const C* s = src + line * ls;
    C* d = dst + line * ls;
    const int j = i % Ns;
    C v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = s[i + q * nb];
    if (Ns > 1) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twid<DIR>(tw, q * j * tws));
    }
    small_dft<R, DIR>(v, tw, rs);
    const int base = (i / Ns) * Ns * R + j;
#pragma unroll
    for (int q = 0; q < R; ++q) d[base + q * Ns] = v[q];
  }
}

// FFT of nlines lines held in a (ping) with b as the pong buffer; every
// thread of the CTA participates.  Returns the buffer holding the result.
template <int DIR, typename C>
__device__ C* fft_lines(C* a, C* b, int nlines, int ls, const RadixPlan& p, const C* tw) {
  int Ns = 1;
  for (int s = 0; s < p.nstage; ++s) {
    const int r = p.radix[s];
    switch (r) {
      case 2: stockham_pass<2, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
      case 3: stockham_pass<3, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
      case 4: stockham_pass<4, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
      case 5: stockham_pass<5, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
      case 7: stockham_pass<7, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
      default: stockham_pass<11, DIR>(a, b, p.n, nlines, ls, Ns, tw); break;
    }
    __syncthreads();
    C* t = a; a = b; b = t;
    Ns *= r;
  }
  return a;
}

template <typename C>
__device__ __forceinline__ void load_twiddles(C* dst, const double2* src, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = mk<C>(src[k].x, src[k].y);
}

// --------------------------------------------------------- z backward
// zbuf layout: [pair][z][stick], stick fastest.
template <typename T>
__global__ void __launch_bounds__(256)
k_zfft_bwd(const double2* __restrict__ c, int ngw, int nst, int pair0,
           DeviceSticks g, const double2* __restrict__ twz,
           typename Cplx<T>::t* __restrict__ zbuf, int rods_per_cta) {
  using C = typename Cplx<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n2 = g.n2;
  C* A = tw + n2;
  C* B = A + 2 * rods_per_cta * n2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const double2* c1 = c + (size_t)b1 * ngw;
  const double2* c2 = (b1 + 1 < nst) ? c + (size_t)(b1 + 1) * ngw : nullptr;
  load_twiddles(tw, twz, n2);
  const int half = (n2 + 1) / 2;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t / n2, z = t - line * n2;
    const int s = s0 + line;
    const int r = (s + 1) >> 1;
    const int lz = z < half ? z : z - n2;
    bool minus;
    int l;
    if (r == 0) { minus = (lz <= 0); l = minus ? -lz : lz; }
    else { minus = ((s & 1) == 0); l = minus ? -lz : lz; }
    const int lmin = g.rod_lmin[r];
    double vx = 0.0, vy = 0.0;
    if (l >= lmin && l < lmin + g.rod_size[r]) {
      const int ig = g.rod_first[r] + (l - lmin);
      const double2 p = c1[ig];
      const double2 q = c2 ? c2[ig] : make_double2(0.0, 0.0);
      // +G: c1 + i c2 ; -G: conj(c1) + i conj(c2)
      if (!minus) { vx = p.x - q.y; vy = p.y + q.x; }
      else        { vx = p.x + q.y; vy = q.x - p.y; }
    }
    A[line * n2 + z] = mk<C>(vx, vy);
  }
  __syncthreads();
  C* res = fft_lines<+1>(A, B, nl, n2, g.pz, tw);
  C* out = zbuf + (size_t)pl * n2 * g.nvec;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    out[(size_t)z * g.nvec + s0 + line] = res[line * n2 + z];
  }
}

// --------------------------------------------------------- z forward
template <typename T>
__global__ void __launch_bounds__(256)
k_zfft_fwd(const typename Cplx<T>::t* __restrict__ zbuf, int ngw, int nst, int pair0,
           DeviceSticks g, const double2* __restrict__ twz, double scale,
           const double2* __restrict__ c, const double* __restrict__ g2,
           double2* __restrict__ hc, int rods_per_cta) {
  using C = typename Cplx<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n2 = g.n2;
  C* A = tw + n2;
  C* B = A + 2 * rods_per_cta * n2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int s0 = (r0 == 0) ? 0 : 2 * r0 - 1;
  const int nl = (2 * r1 - 1) - s0;
  const int pl = blockIdx.y;
  const int b1 = 2 * (pair0 + pl);
  const bool two = (b1 + 1 < nst);
  load_twiddles(tw, twz, n2);
  const C* in = zbuf + (size_t)pl * n2 * g.nvec;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    A[line * n2 + z] = in[(size_t)z * g.nvec + s0 + line];
  }
  __syncthreads();
  C* res = fft_lines<-1>(A, B, nl, n2, g.pz, tw);
  const int ig0 = g.rod_first[r0];
  const int ig1 = g.rod_first[r1 - 1] + g.rod_size[r1 - 1];
  for (int ig = ig0 + threadIdx.x; ig < ig1; ig += blockDim.x) {
    int r = r0;
    while (r + 1 < r1 && g.rod_first[r + 1] <= ig) ++r;
    const int l = g.rod_lmin[r] + (ig - g.rod_first[r]);
    const int zp = ((l % n2) + n2) % n2;
    const int zm = ((-l % n2) + n2) % n2;
    const int sp = (r == 0) ? 0 : 2 * r - 1 - s0;
    const int sm = (r == 0) ? 0 : 2 * r - s0;
    const C P = res[sp * n2 + zp];
    const C M = res[sm * n2 + zm];
    // c1 = (Z(G) + conj Z(-G))/2, c2 = -i (Z(G) - conj Z(-G))/2
    const double px = P.x, py = P.y, mx = M.x, my = M.y;
    const double c1x = 0.5 * (px + mx) * scale, c1y = 0.5 * (py - my) * scale;
    const double c2x = 0.5 * (py + my) * scale, c2y = 0.5 * (mx - px) * scale;
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

// ------------------------------------------------------------ xy plane
enum { OP_DENSITY = 0, OP_VPSI = 1 };

template <int DIR, typename C>
__device__ void y_pass(C* P, C* S, int ncol, int n1, int cc, const RadixPlan& py, const C* twy) {
  for (int c0 = 0; c0 < ncol; c0 += cc) {
    const int nc = min(cc, ncol - c0);
    C* blk = P + c0 * n1;
    C* res = fft_lines<DIR>(blk, S, nc, n1, py, twy);
    if (res != blk) {
      for (int t = threadIdx.x; t < nc * n1; t += blockDim.x) blk[t] = res[t];
      __syncthreads();
    }
  }
}

template <typename T, int OP>
__global__ void __launch_bounds__(512)
k_xy(typename Cplx<T>::t* __restrict__ zbuf, int npairs, int pairs_per_cta,
     DeviceSticks g, const double2* __restrict__ twx, const double2* __restrict__ twy,
     const double* __restrict__ v, double* __restrict__ rho,
     const double* __restrict__ w, int pair0, int nst, int cc, int rr) {
  using C = typename Cplx<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n0 = g.n0, n1 = g.n1, ncol = g.ncol, nvec = g.nvec;
  C* tx = reinterpret_cast<C*>(smem_raw);
  C* ty = tx + n0;
  C* P = ty + n1;
  C* S = P + ncol * n1;
  const int z = blockIdx.x;
  load_twiddles(tx, twx, n0);
  load_twiddles(ty, twy, n1);
  const int pbeg = blockIdx.y * pairs_per_cta;
  const int pend = min(npairs, pbeg + pairs_per_cta);
  for (int pl = pbeg; pl < pend; ++pl) {
    C* zp = zbuf + ((size_t)pl * g.n2 + z) * nvec;
    for (int t = threadIdx.x; t < ncol * n1; t += blockDim.x) P[t] = mk<C>(0.0, 0.0);
    __syncthreads();
    for (int s = threadIdx.x; s < nvec; s += blockDim.x)
      P[g.stick_col[s] * n1 + g.stick_y[s]] = zp[s];
    __syncthreads();
    y_pass<+1>(P, S, ncol, n1, cc, g.py, ty);
    double w1 = 0.0, w2 = 0.0;
    if (OP == OP_DENSITY) {
      const int b1 = 2 * (pair0 + pl);
      w1 = w[b1];
      w2 = (b1 + 1 < nst) ? w[b1 + 1] : 0.0;
    }
    for (int y0 = 0; y0 < n1; y0 += rr) {
      const int nr = min(rr, n1 - y0);
      C* R1 = S;
      C* R2 = S + rr * n0;
      for (int t = threadIdx.x; t < nr * n0; t += blockDim.x) R1[t] = mk<C>(0.0, 0.0);
      __syncthreads();
      for (int t = threadIdx.x; t < nr * ncol; t += blockDim.x) {
        const int r = t / ncol, cidx = t - r * ncol;
        R1[r * n0 + g.col_x[cidx]] = P[cidx * n1 + y0 + r];
      }
      __syncthreads();
      C* res = fft_lines<+1>(R1, R2, nr, n0, g.px, tx);
      const size_t rowbase = ((size_t)z * n1 + y0) * n0;
      if (OP == OP_DENSITY) {
        for (int t = threadIdx.x; t < nr * n0; t += blockDim.x) {
          const C val = res[t];
          const double a = val.x, b = val.y;
          atomicAdd(&rho[rowbase + t], w1 * a * a + w2 * b * b);
        }
        __syncthreads();
      } else {
        for (int t = threadIdx.x; t < nr * n0; t += blockDim.x) {
          const double vv = v[rowbase + t];
          C val = res[t];
          val.x *= vv; val.y *= vv;
          res[t] = val;
        }
        __syncthreads();
        C* other = (res == R1) ? R2 : R1;
        C* res2 = fft_lines<-1>(res, other, nr, n0, g.px, tx);
        for (int t = threadIdx.x; t < nr * ncol; t += blockDim.x) {
          const int r = t / ncol, cidx = t - r * ncol;
          P[cidx * n1 + y0 + r] = res2[r * n0 + g.col_x[cidx]];
        }
        __syncthreads();
      }
    }
    if (OP == OP_VPSI) {
      y_pass<-1>(P, S, ncol, n1, cc, g.py, ty);
      for (int s = threadIdx.x; s < nvec; s += blockDim.x)
        zp[s] = P[g.stick_col[s] * n1 + g.stick_y[s]];
      __syncthreads();
    }
  }
}

// ------------------------------------------------ full-grid line passes
// In-place FFT of all lines along one axis of an n0 x n1 x n2 grid (x
// fastest).  A CTA takes L lines; for the y and z axes these are L adjacent
// x so that global accesses stay coalesced.
template <int DIR>
__global__ void __launch_bounds__(256)
k_line_fft(double2* __restrict__ grid, int n0, int n1, int n2, int axis, RadixPlan p,
           const double2* __restrict__ tw_g, int L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  const int n = p.n;
  double2* A = tw + n;
  double2* B = A + L * n;
  load_twiddles(tw, tw_g, n);
  // line set of this CTA
  size_t base;
  size_t estride, lstride;
  int nl;
  if (axis == 0) {
    const int nlines = n1 * n2;
    const int l0 = blockIdx.x * L;
    nl = min(L, nlines - l0);
    base = (size_t)l0 * n0;
    estride = 1; lstride = n0;
  } else if (axis == 1) {
    const int xt = (n0 + L - 1) / L;
    const int zb = blockIdx.x / xt, x0 = (blockIdx.x % xt) * L;
    nl = min(L, n0 - x0);
    base = (size_t)x0 + (size_t)n0 * n1 * zb;
    estride = n0; lstride = 1;
  } else {
    const int xt = (n0 + L - 1) / L;
    const int yb = blockIdx.x / xt, x0 = (blockIdx.x % xt) * L;
    nl = min(L, n0 - x0);
    base = (size_t)x0 + (size_t)n0 * yb;
    estride = (size_t)n0 * n1; lstride = 1;
  }
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    int line, e;
    if (axis == 0) { line = t / n; e = t - line * n; }
    else { line = t % nl; e = t / nl; }
    A[line * n + e] = grid[base + e * estride + line * lstride];
  }
  __syncthreads();
  double2* res = fft_lines<DIR>(A, B, nl, n, p, tw);
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    int line, e;
    if (axis == 0) { line = t / n; e = t - line * n; }
    else { line = t % nl; e = t / nl; }
    grid[base + e * estride + line * lstride] = res[line * n + e];
  }
}

__global__ void k_scatter_sphere(const double2* __restrict__ c, const int* __restrict__ ip,
                                 const int* __restrict__ im, int ng, double2* __restrict__ grid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 v = c[i];
    grid[ip[i]] = v;
    grid[im[i]] = make_double2(v.x, -v.y);
  }
}

__global__ void k_scatter_pair(const double2* __restrict__ c1, const double2* __restrict__ c2,
                               const int* __restrict__ ip, const int* __restrict__ im, int ng,
                               double2* __restrict__ grid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 p = c1[i];
    const double2 q = c2 ? c2[i] : make_double2(0.0, 0.0);
    grid[ip[i]] = make_double2(p.x - q.y, p.y + q.x);
    grid[im[i]] = make_double2(p.x + q.y, q.x - p.y);
  }
}

__global__ void k_gather_sphere(const double2* __restrict__ grid, const int* __restrict__ ip,
                                int ng, double scale, double2* __restrict__ c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 v = grid[ip[i]];
    c[i] = make_double2(v.x * scale, v.y * scale);
  }
}

// complex basis: only +G is stored (BasisMapping::vector_to_zvec,
// src/BasisMapping.cpp:655-663)
__global__ void k_scatter_plus(const double2* __restrict__ c, const int* __restrict__ ip, int ng,
                               double2* __restrict__ grid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x)
    grid[ip[i]] = c[i];
}

// two real functions out of one complex transform
// (BasisMapping::zvec_to_doublevector, src/BasisMapping.cpp:716-750), with
// the forward transform's 1/N applied to the grid values
__global__ void k_gather_pair(const double2* __restrict__ grid, const int* __restrict__ ip,
                              const int* __restrict__ im, int ng, double scale,
                              double2* __restrict__ c1, double2* __restrict__ c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 p = grid[ip[i]], m = grid[im[i]];
    const double a = p.x * scale, b = p.y * scale, c = m.x * scale, d = m.y * scale;
    c1[i] = make_double2(0.5 * (a + c), 0.5 * (b - d));
    c2[i] = make_double2(0.5 * (b + d), 0.5 * (c - a));
  }
}

__global__ void k_real_to_grid(const double* __restrict__ f, double scale, size_t n,
                               double2* __restrict__ grid) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    grid[i] = make_double2(f[i] * scale, 0.0);
}

__global__ void k_grid_real(const double2* __restrict__ grid, size_t n, double* __restrict__ f) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    f[i] = grid[i].x;
}

// both parts of a grid of two packed real fields
__global__ void k_grid_split(const double2* __restrict__ grid, size_t n, double* __restrict__ f0,
                             double* __restrict__ f1) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = grid[i];
    f0[i] = v.x;
    f1[i] = v.y;
  }
}

// grid = f0 w + i f1 w (f1 may be null)
__global__ void k_real2_mul_to_grid(const double* __restrict__ f0, const double* __restrict__ f1,
                                    const double* __restrict__ w, size_t n,
                                    double2* __restrict__ grid) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double x = w[i];
    grid[i] = make_double2(f0[i] * x, f1 ? f1[i] * x : 0.0);
  }
}

// ------------------------------------------------------------ launchers
static std::vector<double2> twiddle_table(int n) {
  std::vector<double2> t(n);
  for (int k = 0; k < n; k++) {
    const double a = 2.0 * M_PI * (double)k / (double)n;
    t[k] = make_double2(cos(a), sin(a));
  }
  return t;
}

// the twiddle table of one axis of a context's grid
static const double2* twiddles(const Context& ctx, int axis) { return ctx.dws.tw[axis]; }

void upload_sticks(DeviceSticks& d, const Basis& b) {
  free_sticks(d);
  d.n0 = b.n0; d.n1 = b.n1; d.n2 = b.n2;
  d.nrods = b.nrods; d.nvec = b.nvec; d.ncol = b.ncol;
  d.rod_first = dupload(b.rod_first);
  d.rod_lmin = dupload(b.rod_lmin);
  d.rod_size = dupload(b.rod_size);
  d.stick_y = dupload(b.stick_y);
  d.stick_col = dupload(b.stick_col);
  d.col_x = dupload(b.col_x);
  d.ip = dupload(b.ip);
  d.im = dupload(b.im);
  {
    std::vector<int> cm((size_t)b.ncol * b.n1, -1);
    for (int s = 0; s < b.nvec; s++) cm[(size_t)b.stick_col[s] * b.n1 + b.stick_y[s]] = s;
    d.colmap = dupload(cm);
  }
  auto dist = [](int x, int n) { x = ((x % n) + n) % n; return std::min(x, n - x); };
  d.xw = d.yw = d.zw = 0;
  for (int x : b.col_x) d.xw = std::max(d.xw, dist(x, b.n0));
  for (int y : b.stick_y) d.yw = std::max(d.yw, dist(y, b.n1));
  for (int r = 0; r < b.nrods; r++)
    d.zw = std::max({d.zw, std::abs(b.rod_lmin[r]), std::abs(b.rod_lmin[r] + b.rod_size[r] - 1)});
  d.px = make_plan(b.n0);
  d.py = make_plan(b.n1);
  d.pz = make_plan(b.n2);
  const int n[3] = {b.n0, b.n1, b.n2};
  for (int a = 0; a < 3; a++) {
    std::vector<double2> t = twiddle_table(n[a]);
    d.tw[a] = dalloc<double2>(n[a]);
    h2d_sync(d.tw[a], t.data(), n[a] * sizeof(double2));
  }
}

void free_sticks(DeviceSticks& d) {
  for (int a = 0; a < 3; a++) dfree(d.tw[a]);
  dfree(d.rod_first); dfree(d.rod_lmin); dfree(d.rod_size);
  dfree(d.stick_y); dfree(d.stick_col); dfree(d.col_x);
  dfree(d.ip); dfree(d.im);
  dfree(d.colmap);
}

static const int kRodsPerCta = 8;

template <typename T>
static size_t zsmem(int n2) {
  return sizeof(typename Cplx<T>::t) * (size_t)n2 * (1 + 4 * kRodsPerCta);
}

template <typename T>
struct XYConfig {
  size_t smem;
  int cc, rr;
};

static int max_smem_optin(int dev) {
  int v = 0;
  QBX_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return v;
}

template <typename T>
static XYConfig<T> xy_config(const DeviceSticks& g, int dev) {
  using C = typename Cplx<T>::t;
  const size_t fixed = sizeof(C) * ((size_t)g.n0 + g.n1 + (size_t)g.ncol * g.n1);
  const size_t limit = (size_t)max_smem_optin(dev);
  // FP32 tiles leave room for two CTAs per SM
  size_t budget = sizeof(T) == 4 ? std::min(limit, (size_t)112 * 1024) : limit;
  if (budget < fixed + sizeof(C) * 2 * g.n0) budget = limit;
  QBX_REQUIRE(budget >= fixed + sizeof(C) * 2 * g.n0, 20,
              "FFT plane tile does not fit in shared memory");
  const size_t scratch = budget - fixed;
  XYConfig<T> c;
  c.cc = (int)std::min<size_t>(g.ncol, scratch / (sizeof(C) * g.n1));
  c.rr = (int)std::min<size_t>(g.n1, scratch / (sizeof(C) * 2 * g.n0));
  const size_t need = std::max(sizeof(C) * (size_t)c.cc * g.n1, sizeof(C) * 2 * (size_t)c.rr * g.n0);
  c.smem = fixed + need;
  QBX_REQUIRE(c.cc >= 1 && c.rr >= 1, 20, "FFT plane tile does not fit in shared memory");
  return c;
}

template <typename T>
static void staged_batch(Context& ctx, int op, const double* c, const double* v, double* rho,
                         const double* w, double* hc, int pair0, int npairs) {
  using C = typename Cplx<T>::t;
  const DeviceSticks& g = ctx.dws;
  cudaStream_t st = ctx.stream;
  C* zbuf = (C*)ctx.d_zbuf;
  const double2* twz = twiddles(ctx, 2);
  const double2* twx = twiddles(ctx, 0);
  const double2* twy = twiddles(ctx, 1);
  const int ngw = ctx.wb.ng;
  dim3 zgrid((g.nrods + kRodsPerCta - 1) / kRodsPerCta, npairs);
  const size_t zs = zsmem<T>(g.n2);
  allow_smem(k_zfft_bwd<T>, zs);
  {
    ProfScope ps(ctx, "zfft_bwd");
    k_zfft_bwd<T><<<zgrid, 256, zs, st>>>((const double2*)c, ngw, ctx.nst, pair0, g, twz, zbuf,
                                           kRodsPerCta);
    QBX_LAUNCHED(ctx);
  }
  XYConfig<T> xc = xy_config<T>(g, ctx.device);
  int sms = 0;
  QBX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
  // enough (plane, pair-chunk) CTAs to cover every SM a couple of times
  int chunks = std::max(1, (3 * sms + g.n2 - 1) / g.n2);
  chunks = std::min(chunks, npairs);
  const int ppc = (npairs + chunks - 1) / chunks;
  chunks = (npairs + ppc - 1) / ppc;
  dim3 xgrid(g.n2, chunks);
  if (op == OP_DENSITY) {
    allow_smem(k_xy<T, OP_DENSITY>, xc.smem);
    ProfScope ps(ctx, "xy_density");
    k_xy<T, OP_DENSITY><<<xgrid, 512, xc.smem, st>>>(zbuf, npairs, ppc, g, twx, twy, nullptr, rho, w,
                                                   pair0, ctx.nst, xc.cc, xc.rr);
    QBX_LAUNCHED(ctx);
  } else {
    allow_smem(k_xy<T, OP_VPSI>, xc.smem);
    {
      ProfScope ps(ctx, "xy_vpsi");
      k_xy<T, OP_VPSI><<<xgrid, 512, xc.smem, st>>>(zbuf, npairs, ppc, g, twx, twy, v, nullptr,
                                                  nullptr, pair0, ctx.nst, xc.cc, xc.rr);
      QBX_LAUNCHED(ctx);
    }
    allow_smem(k_zfft_fwd<T>, zs);
    const double scale = 1.0 / ((double)g.n0 * g.n1 * g.n2);
    ProfScope ps(ctx, "zfft_fwd");
    k_zfft_fwd<T><<<zgrid, 256, zs, st>>>(zbuf, ngw, ctx.nst, pair0, g, twz, scale,
                                           (const double2*)c, ctx.d_g2_w, (double2*)hc, kRodsPerCta);
    QBX_LAUNCHED(ctx);
  }
}

// ------------------------------------------------ complex basis (k != 0)
// One band per stick line: the basis at k has one rod per (h,k) column and
// no -G half to fill (BasisMapping::vector_to_zvec and zvec_to_vector of a
// complex basis, src/BasisMapping.cpp:585-627, 703-750).  zbuf holds band
// `band0 + slot` in slot, [slot][z][stick] as for band pairs, so the plane
// kernels run unchanged on the complex sticks.
__global__ void __launch_bounds__(256)
k_zfft_bwd_k(const double2* __restrict__ c, int ngw, int band0, DeviceSticks g,
             const double2* __restrict__ twz, double2* __restrict__ zbuf, int rods_per_cta) {
  using C = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n2 = g.n2;
  C* A = tw + n2;
  C* B = A + rods_per_cta * n2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int nl = r1 - r0;
  const int pl = blockIdx.y;
  const double2* cb = c + (size_t)(band0 + pl) * ngw;
  load_twiddles(tw, twz, n2);
  const int half = (n2 + 1) / 2;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t / n2, z = t - line * n2;
    const int r = r0 + line;
    const int l = z < half ? z : z - n2;
    const int lmin = g.rod_lmin[r];
    C v = make_double2(0.0, 0.0);
    if (l >= lmin && l < lmin + g.rod_size[r]) v = cb[g.rod_first[r] + (l - lmin)];
    A[line * n2 + z] = v;
  }
  __syncthreads();
  C* res = fft_lines<+1>(A, B, nl, n2, g.pz, tw);
  C* out = zbuf + (size_t)pl * n2 * g.nvec;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    out[(size_t)z * g.nvec + r0 + line] = res[line * n2 + z];
  }
}

// z transform back and hc = 1/2 |k+G|^2 c + (V psi)(G) / N
__global__ void __launch_bounds__(256)
k_zfft_fwd_k(const double2* __restrict__ zbuf, int ngw, int band0, DeviceSticks g,
             const double2* __restrict__ twz, double scale, const double2* __restrict__ c,
             const double* __restrict__ g2, double2* __restrict__ hc, int rods_per_cta) {
  using C = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  const int n2 = g.n2;
  C* A = tw + n2;
  C* B = A + rods_per_cta * n2;
  const int r0 = blockIdx.x * rods_per_cta;
  const int r1 = min(g.nrods, r0 + rods_per_cta);
  const int nl = r1 - r0;
  const int pl = blockIdx.y;
  load_twiddles(tw, twz, n2);
  const C* in = zbuf + (size_t)pl * n2 * g.nvec;
  for (int t = threadIdx.x; t < nl * n2; t += blockDim.x) {
    const int line = t % nl, z = t / nl;
    A[line * n2 + z] = in[(size_t)z * g.nvec + r0 + line];
  }
  __syncthreads();
  C* res = fft_lines<-1>(A, B, nl, n2, g.pz, tw);
  const int ig0 = g.rod_first[r0];
  const int ig1 = g.rod_first[r1 - 1] + g.rod_size[r1 - 1];
  const size_t boff = (size_t)(band0 + pl) * ngw;
  for (int ig = ig0 + threadIdx.x; ig < ig1; ig += blockDim.x) {
    int r = r0;
    while (r + 1 < r1 && g.rod_first[r + 1] <= ig) ++r;
    const int l = g.rod_lmin[r] + (ig - g.rod_first[r]);
    const int z = ((l % n2) + n2) % n2;
    const C p = res[(r - r0) * n2 + z];
    const double kin = 0.5 * g2[ig];
    const double2 a = c[boff + ig];
    hc[boff + ig] = make_double2(kin * a.x + p.x * scale, kin * a.y + p.y * scale);
  }
}

static constexpr int kRodsPerCtaK = 2 * kRodsPerCta;   // one line per rod

// bands of a k point per pass through the context's stick buffer
static int kbands_per_batch(const Context& ctx, const KPointSet& kp) {
  const size_t per_band = (size_t)kp.dks.n2 * kp.dks.nvec * sizeof(double2);
  const int nb = (int)std::min<size_t>((size_t)ctx.nst, ctx.zbuf_bytes / per_band);
  QBX_REQUIRE(nb >= 1, 20, "stick buffer too small for one band of this k point");
  return nb;
}

static void staged_k(Context& ctx, KPointSet& kp, int op, const double* v, double* rho) {
  const DeviceSticks& g = kp.dks;
  cudaStream_t st = ctx.stream;
  double2* zbuf = (double2*)ctx.d_zbuf;
  const int ngw = kp.kb.ng;
  const size_t zs = zsmem<double>(g.n2);
  allow_smem(k_zfft_bwd_k, zs);
  allow_smem(k_zfft_fwd_k, zs);
  XYConfig<double> xc = xy_config<double>(g, ctx.device);
  allow_smem(k_xy<double, OP_DENSITY>, xc.smem);
  allow_smem(k_xy<double, OP_VPSI>, xc.smem);
  int sms = 0;
  QBX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
  const int nbmax = kbands_per_batch(ctx, kp);
  for (int b0 = 0; b0 < ctx.nst; b0 += nbmax) {
    const int nb = std::min(nbmax, ctx.nst - b0);
    dim3 zgrid((g.nrods + kRodsPerCtaK - 1) / kRodsPerCtaK, nb);
    k_zfft_bwd_k<<<zgrid, 256, zs, st>>>((const double2*)kp.d_c, ngw, b0, g, g.tw[2], zbuf,
                                         kRodsPerCtaK);
    QBX_LAUNCHED(ctx);
    int chunks = std::max(1, (3 * sms + g.n2 - 1) / g.n2);
    chunks = std::min(chunks, nb);
    const int ppc = (nb + chunks - 1) / chunks;
    chunks = (nb + ppc - 1) / ppc;
    dim3 xgrid(g.n2, chunks);
    if (op == OP_DENSITY) {
      // the pair kernel's weights w[2 slot], w[2 slot + 1] are both the band's
      k_xy<double, OP_DENSITY><<<xgrid, 512, xc.smem, st>>>(zbuf, nb, ppc, g, g.tw[0], g.tw[1],
                                                           nullptr, rho, kp.d_w2, b0, 2 * ctx.nst,
                                                           xc.cc, xc.rr);
      QBX_LAUNCHED(ctx);
    } else {
      k_xy<double, OP_VPSI><<<xgrid, 512, xc.smem, st>>>(zbuf, nb, ppc, g, g.tw[0], g.tw[1], v,
                                                        nullptr, nullptr, b0, 2 * ctx.nst, xc.cc,
                                                        xc.rr);
      QBX_LAUNCHED(ctx);
      const double scale = 1.0 / ((double)g.n0 * g.n1 * g.n2);
      k_zfft_fwd_k<<<zgrid, 256, zs, st>>>(zbuf, ngw, b0, g, g.tw[2], scale,
                                           (const double2*)kp.d_c, kp.d_g2, (double2*)kp.d_hc,
                                           kRodsPerCtaK);
      QBX_LAUNCHED(ctx);
    }
  }
}

// rho += sum_n weight occ_n / Omega |psi_nk|^2 (SlaterDet::compute_density,
// complex branch, src/SlaterDet.cpp:280-298)
void launch_density_k(Context& ctx, KPointSet& kp, double* rho) {
  ProfScope ps(ctx, "density_k");
  staged_k(ctx, kp, OP_DENSITY, nullptr, rho);
}

// hc = 1/2 |k+G|^2 c + FFT_fwd(v FFT_bwd(c)) (SlaterDet::rs_mul_add, complex
// branch, src/SlaterDet.cpp:458-475, with the kinetic term of
// EnergyFunctional::energy, src/EnergyFunctional.cpp:789-839)
void launch_vpsi_k(Context& ctx, KPointSet& kp, const double* v) {
  ProfScope ps(ctx, "vpsi_k");
  staged_k(ctx, kp, OP_VPSI, v, nullptr);
}

static int nblk(size_t n);

__global__ void k_to_float(const double* __restrict__ x, size_t n, float* __restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// The specialised kernels of fft_fast_*.cu in batches of band pairs through
// ctx.d_zfast; false when the grid has none.
// the psi(r) buffer (FP32, every band pair on the whole grid), allocated
// outside stream capture when the device has room for it
static bool psir_ready(Context& ctx) {
  if (ctx.psir_mode == 0 || ctx.precision != MIXED || ctx.fast_lane_shape < 0) return false;
  const size_t need = (size_t)((ctx.nst + 1) / 2) * ctx.N() * sizeof(float2);
  if (ctx.d_psir && ctx.psir_bytes >= need) return true;
  if (ctx.capturing) return false;
  size_t freeb = 0, total = 0;
  QBX_CUDA(cudaMemGetInfo(&freeb, &total));
  if (freeb < need + ((size_t)4 << 30)) {
    if (ctx.psir_mode < 0) ctx.psir_mode = 0;   // no room: recompute psi(r) from now on
    return false;
  }
  if (ctx.d_psir) cudaFree(ctx.d_psir);
  QBX_CUDA(cudaMalloc(&ctx.d_psir, need));
  ctx.psir_bytes = need;
  return true;
}

static bool staged_fast(Context& ctx, int op, const double* c, const double* v, double* rho,
                        const double* w, double* hc) {
  if (!ctx.fast_fft || !ctx.d_zfast) return false;
  const DeviceSticks& g = ctx.dws;
  fast::StagedArgs a{};
  a.op = (op == OP_DENSITY) ? fast::XY_DENSITY : fast::XY_VPSI;
  a.c = c;
  a.rho = rho;
  a.w = w;
  a.hc = hc;
  a.nst = ctx.nst;
  a.zbuf = ctx.d_zfast;
  a.twx = twiddles(ctx, 0);
  a.twy = twiddles(ctx, 1);
  a.twz = twiddles(ctx, 2);
  a.rods_per_cta = ctx.fast_rods;
  a.xy_warps = ctx.fast_warps;
  a.vpsi_shape = ctx.fast_vpsi_shape;
  a.lane_shape = ctx.fast_lane_shape;
  a.density_lane_shape = ctx.fast_density_lane_shape;
  a.density_chunks = ctx.fast_chunks;
  a.fwd_pairs_per_cta = ctx.fast_fwd_ppc;
  a.zlane = ctx.fast_zlane;
  a.fwd_staged = ctx.fast_fwd_staged;
  a.prune = ctx.fast_prune;
  a.v = v;
  a.psir = nullptr;
  if (op == OP_DENSITY) {
    ctx.psir_valid = false;
    if (ctx.psir_store && psir_ready(ctx)) a.psir = ctx.d_psir;
  } else if (ctx.psir_use && ctx.psir_valid && ctx.psir_src == c) {
    a.psir = ctx.d_psir;
  }
  if (op == OP_VPSI && ctx.precision == MIXED) {
    const size_t N = ctx.N();
    k_to_float<<<nblk(N), 256, 0, ctx.stream>>>(v, N, ctx.d_vr32);
    QBX_LAUNCHED(ctx);
    a.v = ctx.d_vr32;
  }
  const size_t limit = (size_t)max_smem_optin(ctx.device);
  int plo = 0, phi = 0;
  shard_pairs(ctx, plo, phi);            // this GPU's band pairs
  const int npairs = phi - plo;
  const size_t per_pair = (ctx.precision == MIXED ? sizeof(float2) : sizeof(double2)) *
                          (size_t)g.n2 * g.nvec;
  int batch = (int)std::min<size_t>(std::max(npairs, 1), ctx.zfast_bytes / per_pair);
  if (ctx.fast_batch > 0) batch = std::min(batch, ctx.fast_batch);
  QBX_REQUIRE(batch >= 1, 21, "stick buffer of the specialised FFTs holds no band pair");
  bool first = true;
  for (int p0 = plo; p0 < phi; p0 += batch) {
    a.pair0 = p0;
    a.npairs = std::min(batch, phi - p0);
    const bool ok = fast_staged_a(ctx, a, limit) || fast_staged_b(ctx, a, limit);
    if (!ok) {
      QBX_REQUIRE(first, 21, "specialised FFT kernels unavailable after the first batch");
      return false;
    }
    first = false;
  }
  if (op == OP_DENSITY && a.psir) {
    ctx.psir_valid = true;
    ctx.psir_src = c;
  }
  return true;
}

static void staged(Context& ctx, int op, const double* c, const double* v, double* rho,
                   const double* w, double* hc) {
  if (staged_fast(ctx, op, c, v, rho, w, hc)) return;
  int plo = 0, phi = 0;
  shard_pairs(ctx, plo, phi);
  for (int p0 = plo; p0 < phi; p0 += ctx.pair_batch) {
    const int np = std::min(ctx.pair_batch, phi - p0);
    if (ctx.precision == MIXED)
      staged_batch<float>(ctx, op, c, v, rho, w, hc, p0, np);
    else
      staged_batch<double>(ctx, op, c, v, rho, w, hc, p0, np);
  }
}

// With the band pairs split over GPUs (qbx_set_band_shard) each GPU
// transforms its own pairs; the density is then summed over the GPUs and
// the H*psi blocks gathered, so every GPU continues with the whole of both.
void launch_density(Context& ctx, const double* c, double* rho) {
  QBX_CUDA(cudaMemsetAsync(rho, 0, ctx.N() * sizeof(double), ctx.stream));
  staged(ctx, OP_DENSITY, c, nullptr, rho, density_weights(ctx), nullptr);
  if (ctx.shard_comm) shard_sum(ctx, rho, ctx.N());
}

void launch_vpsi(Context& ctx, const double* c, const double* v, double* hc) {
  staged(ctx, OP_VPSI, c, v, nullptr, nullptr, hc);
  if (ctx.shard_comm) shard_gather_bands(ctx, hc);
}

// full-grid transform of `grid` on the geometry of d (sizes, twiddles)
static void grid_fft_on(Context& ctx, const DeviceSticks& b, double2* grid, int dir) {
  ProfScope ps(ctx, "grid_fft");
  const int n[3] = {b.n0, b.n1, b.n2};
  const int L = 16;
  for (int axis = 0; axis < 3; axis++) {
    const double2* tw = b.tw[axis];
    // compile-time lengths: warp FFTs on coalesced tiles (fft_fast.cuh)
    if (ctx.fast_fft &&
        (fast_grid_lines_a(ctx, grid, b.n0, b.n1, b.n2, axis, dir, tw) ||
         fast_grid_lines_b(ctx, grid, b.n0, b.n1, b.n2, axis, dir, tw)))
      continue;
    const RadixPlan p = make_plan(n[axis]);
    int nblocks;
    if (axis == 0) nblocks = (b.n1 * b.n2 + L - 1) / L;
    else if (axis == 1) nblocks = ((b.n0 + L - 1) / L) * b.n2;
    else nblocks = ((b.n0 + L - 1) / L) * b.n1;
    const size_t smem = sizeof(double2) * (size_t)n[axis] * (1 + 2 * L);
    if (dir > 0) {
      allow_smem(k_line_fft<+1>, smem);
      k_line_fft<+1><<<nblocks, 256, smem, ctx.stream>>>(grid, b.n0, b.n1, b.n2, axis, p, tw, L);
    } else {
      allow_smem(k_line_fft<-1>, smem);
      k_line_fft<-1><<<nblocks, 256, smem, ctx.stream>>>(grid, b.n0, b.n1, b.n2, axis, p, tw, L);
    }
    QBX_LAUNCHED(ctx);
  }
}

// full-grid transform of the density-basis grid held in ctx.d_grid
static void grid_fft(Context& ctx, int dir) { grid_fft_on(ctx, ctx.dvs, (double2*)ctx.d_grid, dir); }

// One band c (ng coefficients of the half sphere) to its real values on the
// grid of d (FourierTransform::backward, one band), x fastest, into f.
void wfgrid_backward(Context& ctx, const DeviceSticks& d, int ng, const double* c, double* f) {
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  QBX_REQUIRE(N <= ctx.N(), 1, "grid larger than the density grid's workspace");
  QBX_CUDA(cudaMemsetAsync(ctx.d_grid, 0, N * sizeof(double2), ctx.stream));
  k_scatter_sphere<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)c, d.ip, d.im, ng,
                                                     (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft_on(ctx, d, (double2*)ctx.d_grid, +1);
  k_grid_real<<<nblk(N), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, N, f);
  QBX_LAUNCHED(ctx);
}

// The inverse: real values f on the grid of d to the band's coefficients
// (FourierTransform::forward with its 1/N, then the half sphere).
void wfgrid_forward(Context& ctx, const DeviceSticks& d, int ng, const double* f, double* c) {
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  QBX_REQUIRE(N <= ctx.N(), 1, "grid larger than the density grid's workspace");
  k_real_to_grid<<<nblk(N), 256, 0, ctx.stream>>>(f, 1.0, N, (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft_on(ctx, d, (double2*)ctx.d_grid, -1);
  k_gather_sphere<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, d.ip, ng,
                                                    1.0 / (double)N, (double2*)c);
  QBX_LAUNCHED(ctx);
}

static int nblk(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// ----------------------------------------------- a caller's basis and grid
// The grid of a FourierTransform built on any basis (its Miller indices in
// the caller's order): sizes, twiddle tables, radix plans and the grid
// index of +G and (real basis) -G of each coefficient.  The transforms are
// full-grid line passes; the staged z-stick kernels serve the contexts'
// own bases.
void upload_grid_map(DeviceSticks& d, int n0, int n1, int n2, const std::vector<int>& ip,
                     const std::vector<int>& im) {
  free_sticks(d);
  d = DeviceSticks{};
  d.n0 = n0; d.n1 = n1; d.n2 = n2;
  d.ip = dupload(ip);
  if (!im.empty()) d.im = dupload(im);
  d.px = make_plan(n0);
  d.py = make_plan(n1);
  d.pz = make_plan(n2);
  const int n[3] = {n0, n1, n2};
  for (int a = 0; a < 3; a++) {
    std::vector<double2> t = twiddle_table(n[a]);
    d.tw[a] = dalloc<double2>(n[a]);
    h2d_sync(d.tw[a], t.data(), n[a] * sizeof(double2));
  }
}

// FourierTransform::backward (src/FourierTransform.cpp:159-200): one band
// (c2 == nullptr) or the pair c1 + i c2 (real basis) from the basis to the
// complex grid, unscaled synthesis
void basis_ft_backward(Context& ctx, const DeviceSticks& d, int ng, bool real_basis,
                       const double* c1, const double* c2, double* grid) {
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  QBX_CUDA(cudaMemsetAsync(grid, 0, N * sizeof(double2), ctx.stream));
  if (!real_basis) {
    k_scatter_plus<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)c1, d.ip, ng,
                                                     (double2*)grid);
  } else if (c2) {
    k_scatter_pair<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)c1, (const double2*)c2, d.ip,
                                                     d.im, ng, (double2*)grid);
  } else {
    k_scatter_sphere<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)c1, d.ip, d.im, ng,
                                                       (double2*)grid);
  }
  QBX_LAUNCHED(ctx);
  grid_fft_on(ctx, d, (double2*)grid, +1);
}

// FourierTransform::forward (src/FourierTransform.cpp:147-196): the grid is
// transformed in place (the reference also overwrites f), scaled by 1/N and
// gathered onto the basis; with c2 the two real functions are unpacked
void basis_ft_forward(Context& ctx, const DeviceSticks& d, int ng, bool real_basis, double* grid,
                      double* c1, double* c2) {
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  grid_fft_on(ctx, d, (double2*)grid, -1);
  const double scale = 1.0 / (double)N;
  if (c2) {
    QBX_REQUIRE(real_basis, 1, "the two-band forward transform needs a real basis");
    k_gather_pair<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)grid, d.ip, d.im, ng, scale,
                                                    (double2*)c1, (double2*)c2);
  } else {
    k_gather_sphere<<<nblk(ng), 256, 0, ctx.stream>>>((const double2*)grid, d.ip, ng, scale,
                                                      (double2*)c1);
  }
  QBX_LAUNCHED(ctx);
}

void vb_backward(Context& ctx, const double* coef, double* real_out) {
  const size_t N = ctx.N();
  QBX_CUDA(cudaMemsetAsync(ctx.d_grid, 0, N * sizeof(double2), ctx.stream));
  k_scatter_sphere<<<nblk(ctx.vb.ng), 256, 0, ctx.stream>>>((const double2*)coef, ctx.dvs.ip,
                                                            ctx.dvs.im, ctx.vb.ng, (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft(ctx, +1);
  k_grid_real<<<nblk(N), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, N, real_out);
  QBX_LAUNCHED(ctx);
}

void vb_backward_pair(Context& ctx, const double* a, const double* b, double* out0, double* out1) {
  const size_t N = ctx.N();
  QBX_CUDA(cudaMemsetAsync(ctx.d_grid, 0, N * sizeof(double2), ctx.stream));
  k_scatter_pair<<<nblk(ctx.vb.ng), 256, 0, ctx.stream>>>((const double2*)a, (const double2*)b,
                                                          ctx.dvs.ip, ctx.dvs.im, ctx.vb.ng,
                                                          (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft(ctx, +1);
  k_grid_split<<<nblk(N), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, N, out0, out1);
  QBX_LAUNCHED(ctx);
}

void vb_forward_real_pair(Context& ctx, const double* f0, const double* f1, const double* w,
                          double* c0, double* c1) {
  const size_t N = ctx.N();
  k_real2_mul_to_grid<<<nblk(N), 256, 0, ctx.stream>>>(f0, f1, w, N, (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft(ctx, -1);
  if (f1) {
    k_gather_pair<<<nblk(ctx.vb.ng), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, ctx.dvs.ip,
                                                           ctx.dvs.im, ctx.vb.ng, 1.0 / (double)N,
                                                           (double2*)c0, (double2*)c1);
  } else {
    k_gather_sphere<<<nblk(ctx.vb.ng), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, ctx.dvs.ip,
                                                             ctx.vb.ng, 1.0 / (double)N,
                                                             (double2*)c0);
  }
  QBX_LAUNCHED(ctx);
}

void vb_forward_real(Context& ctx, const double* f, double scale, double* coef) {
  const size_t N = ctx.N();
  k_real_to_grid<<<nblk(N), 256, 0, ctx.stream>>>(f, scale, N, (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft(ctx, -1);
  k_gather_sphere<<<nblk(ctx.vb.ng), 256, 0, ctx.stream>>>((const double2*)ctx.d_grid, ctx.dvs.ip,
                                                           ctx.vb.ng, 1.0 / (double)N, (double2*)coef);
  QBX_LAUNCHED(ctx);
}

void wb_backward_pair(Context& ctx, const double* c1, const double* c2, double* grid_out) {
  const size_t N = ctx.N();
  QBX_CUDA(cudaMemsetAsync(ctx.d_grid, 0, N * sizeof(double2), ctx.stream));
  k_scatter_pair<<<nblk(ctx.wb.ng), 256, 0, ctx.stream>>>((const double2*)c1, (const double2*)c2,
                                                          ctx.dws.ip, ctx.dws.im, ctx.wb.ng,
                                                          (double2*)ctx.d_grid);
  QBX_LAUNCHED(ctx);
  grid_fft(ctx, +1);
  QBX_CUDA(cudaMemcpyAsync(grid_out, ctx.d_grid, N * sizeof(double2), cudaMemcpyDeviceToDevice,
                           ctx.stream));
}

}  // namespace qbx

namespace qbx {

// Density of nst bands of c (device, default order) added into rho, with the
// stick buffer and the three twiddle tables supplied by the caller instead
// of the context's own.  Batches of band pairs are sized to zbuf_bytes.
template <typename T>
static void density_buffers_t(Context& ctx, const double* c, int nst, const double* w,
                              double* rho, void* zbuf, size_t zbuf_bytes, const double2* twx,
                              const double2* twy, const double2* twz) {
  using C = typename Cplx<T>::t;
  const DeviceSticks& g = ctx.dws;
  cudaStream_t st = ctx.stream;
  const size_t per_pair = sizeof(C) * (size_t)g.n2 * g.nvec;
  const int npairs_all = (nst + 1) / 2;
  const int batch = (int)std::min<size_t>(npairs_all, zbuf_bytes / per_pair);
  QBX_REQUIRE(batch >= 1, 60, "stick buffer smaller than one band pair");
  const size_t zs = zsmem<T>(g.n2);
  allow_smem(k_zfft_bwd<T>, zs);
  XYConfig<T> xc = xy_config<T>(g, ctx.device);
  allow_smem(k_xy<T, OP_DENSITY>, xc.smem);
  int sms = 0;
  QBX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
  for (int p0 = 0; p0 < npairs_all; p0 += batch) {
    const int npairs = std::min(batch, npairs_all - p0);
    dim3 zgrid((g.nrods + kRodsPerCta - 1) / kRodsPerCta, npairs);
    k_zfft_bwd<T><<<zgrid, 256, zs, st>>>((const double2*)c, ctx.wb.ng, nst, p0, g, twz, (C*)zbuf,
                                           kRodsPerCta);
    QBX_LAUNCHED(ctx);
    int chunks = std::max(1, (3 * sms + g.n2 - 1) / g.n2);
    chunks = std::min(chunks, npairs);
    const int ppc = (npairs + chunks - 1) / chunks;
    chunks = (npairs + ppc - 1) / ppc;
    dim3 xgrid(g.n2, chunks);
    k_xy<T, OP_DENSITY><<<xgrid, 512, xc.smem, st>>>((C*)zbuf, npairs, ppc, g, twx, twy, nullptr,
                                                     rho, w, p0, nst, xc.cc, xc.rr);
    QBX_LAUNCHED(ctx);
  }
}

size_t density_stick_bytes_per_pair(const Context& ctx) {
  const size_t e = ctx.precision == MIXED ? sizeof(float2) : sizeof(double2);
  return e * (size_t)ctx.dws.n2 * ctx.dws.nvec;
}

void density_with_buffers(Context& ctx, const double* c, int nst, const double* w, double* rho,
                          void* zbuf, size_t zbuf_bytes, const double2* twx, const double2* twy,
                          const double2* twz) {
  if (ctx.precision == MIXED)
    density_buffers_t<float>(ctx, c, nst, w, rho, zbuf, zbuf_bytes, twx, twy, twz);
  else
    density_buffers_t<double>(ctx, c, nst, w, rho, zbuf, zbuf_bytes, twx, twy, twz);
}

}  // namespace qbx

namespace qbx {

// ------------------------------------------------------------ autotuner
// Picks the staged-FFT launch configuration (plane-kernel family and CTA
// shape for H*psi and for the density, band pairs per launch, rods per z
// CTA) for this context's grid, basis and precision by timing the
// candidates on the context's own wavefunctions and potential, one
// parameter at a time in that order.  Results go to ctx.fast_*; the chosen
// values and timings are appended to `log`.
void autotune_fft(Context& ctx, std::vector<std::pair<std::string, double>>* log) {
  QBX_REQUIRE(ctx.have_cell && ctx.d_zfast, 7, "autotune needs a cell");
  const size_t N = ctx.N();
  double* rho_tmp = dalloc<double>(N);
  double* hc_tmp = ctx.d_ctmp;
  cudaEvent_t e0, e1;
  QBX_CUDA(cudaEventCreate(&e0));
  QBX_CUDA(cudaEventCreate(&e1));
  auto time_ms = [&](auto fn) {
    fn();   // warm-up (function attributes, caches)
    QBX_CUDA(cudaEventRecord(e0, ctx.stream));
    fn();
    QBX_CUDA(cudaEventRecord(e1, ctx.stream));
    QBX_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    QBX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return (double)ms;
  };
  auto vpsi = [&]() { launch_vpsi(ctx, ctx.d_c, ctx.d_vr, hc_tmp); };
  auto dens = [&]() { launch_density(ctx, ctx.d_c, rho_tmp); };
  auto note = [&](const std::string& what, double ms) {
    if (log) log->push_back({what, ms});
  };
  try {
    // 1. H*psi plane kernel: register-lane shapes (FP32 lengths with a
    // register plan), then the warp-per-line kernel
    {
      std::vector<std::pair<int, int>> cand;   // (lane shape, warp shape)
      if (ctx.precision == MIXED) {
        for (int s : {4, 0, 3, 5, 6}) cand.push_back({s, ctx.fast_vpsi_shape});
        for (int s : {0, 1}) cand.push_back({-1, s});
      } else {
        cand.push_back({-1, ctx.fast_vpsi_shape});
      }
      double best = 1e30;
      std::pair<int, int> pick = cand[0];
      for (auto cv : cand) {
        ctx.fast_lane_shape = cv.first;
        ctx.fast_vpsi_shape = cv.second;
        const double t = time_ms(vpsi);
        note("vpsi lane " + std::to_string(cv.first) + " warp " + std::to_string(cv.second), t);
        if (t < best) { best = t; pick = cv; }
      }
      ctx.fast_lane_shape = pick.first;
      ctx.fast_vpsi_shape = pick.second;
    }
    // 2. density plane kernel shape
    if (ctx.precision == MIXED && ctx.fast_lane_shape >= 0) {
      double best = 1e30;
      int pick = ctx.fast_density_lane_shape;
      for (int s : {3, 2, 5, 6, 7, 8}) {
        ctx.fast_density_lane_shape = s;
        const double t = time_ms(dens);
        note("density lane " + std::to_string(s), t);
        if (t < best) { best = t; pick = s; }
      }
      ctx.fast_density_lane_shape = pick;
      // CTAs per plane (each accumulates its share of the band pairs)
      int pick_c = ctx.fast_chunks;
      for (int ch : {4, 8, 12, 16}) {
        ctx.fast_chunks = ch;
        const double t = time_ms(dens);
        note("density CTAs per plane " + std::to_string(ch), t);
        if (t < best) { best = t; pick_c = ch; }
      }
      ctx.fast_chunks = pick_c;
    }
    // 3. band pairs per launch (the stick buffer stays in L2 for small batches)
    {
      const size_t per_pair = (ctx.precision == MIXED ? sizeof(float2) : sizeof(double2)) *
                              (size_t)ctx.dws.n2 * ctx.dws.nvec;
      const int cap = (int)std::max<size_t>(1, ctx.zfast_bytes / per_pair);
      double best = 1e30;
      int pick = ctx.fast_batch;
      for (int b : {16, 32, 64, 0}) {
        if (b > cap) continue;
        ctx.fast_batch = b;
        const double t = time_ms(vpsi) + time_ms(dens);
        note("pairs per launch " + std::to_string(b == 0 ? cap : b), t);
        if (t < best) { best = t; pick = b; }
      }
      ctx.fast_batch = pick;
    }
    // 4. z-stick kernels (register lanes or a warp per stick) and rods per CTA
    {
      double best = 1e30;
      int pick = ctx.fast_rods, pick_z = ctx.fast_zlane;
      for (int zl : {1, 0}) {
        if (zl == 0 && ctx.precision != MIXED) continue;
        if (ctx.precision == MIXED) ctx.fast_zlane = zl;
        for (int r : {8, 16, 24, 32}) {
          ctx.fast_rods = r;
          const double t = time_ms(vpsi);
          note("z lanes " + std::to_string(ctx.fast_zlane) + " rods per z CTA " + std::to_string(r), t);
          if (t < best) { best = t; pick = r; pick_z = ctx.fast_zlane; }
        }
      }
      ctx.fast_rods = pick;
      ctx.fast_zlane = pick_z;
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dfree(rho_tmp);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(rho_tmp);
}

}  // namespace qbx
