// Deterministic reductions for the device scalar slots: fixed-size partial
// sums per CTA, then one CTA adds the partials in order, so a sum does not
// depend on scheduling.  Shared by the kernel files of the electronic step.
#pragma once

#include "qbx_internal.h"

namespace qbx {
namespace red {

constexpr int kRedBlocks = 592;   // 4 x 148 SMs
constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r += sh[i];
  return r;   // valid in thread 0
}

// sum of up to 4 quantities produced by functor F(i, out[4]) over i < n
template <int K, typename F>
__global__ void __launch_bounds__(kThreads) k_reduce(F f, size_t n, double* partial) {
  __shared__ double sh[32];
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    f(i, acc);
#pragma unroll
  for (int k = 0; k < K; k++) {
    const double s = block_sum(acc[k], sh);
    if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = s;
  }
}

template <int K>
__global__ void k_reduce_final(const double* partial, int nb, double* out) {
  __shared__ double sh[32];
  for (int k = 0; k < K; k++) {
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partial[k * nb + i];
    const double s = block_sum(a, sh);
    if (threadIdx.x == 0) out[k] = s;
  }
}

// K sums of f over [0, n) into the scalar slots [slot, slot + K); no host
// synchronisation (the host reads the slots after the step)
template <int K, typename F>
inline void reduce(Context& ctx, F f, size_t n, int slot) {
  const int nb = (int)std::max<size_t>(1, std::min<size_t>(kRedBlocks, (n + kThreads - 1) / kThreads));
  k_reduce<K><<<nb, kThreads, 0, ctx.stream>>>(f, n, ctx.d_red);
  QBX_LAUNCHED(ctx);
  k_reduce_final<K><<<1, kThreads, 0, ctx.stream>>>(ctx.d_red, nb, ctx.d_scalars + slot);
  QBX_LAUNCHED(ctx);
}

// as reduce, but adds weight x the sums into the slots instead of storing them
template <int K>
__global__ void k_reduce_final_acc(const double* partial, int nb, double weight, double* out) {
  __shared__ double sh[32];
  for (int k = 0; k < K; k++) {
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partial[k * nb + i];
    const double s = block_sum(a, sh);
    if (threadIdx.x == 0) out[k] += weight * s;
  }
}

template <int K, typename F>
inline void reduce_acc(Context& ctx, F f, size_t n, int slot, double weight) {
  const int nb = (int)std::max<size_t>(1, std::min<size_t>(kRedBlocks, (n + kThreads - 1) / kThreads));
  k_reduce<K><<<nb, kThreads, 0, ctx.stream>>>(f, n, ctx.d_red);
  QBX_LAUNCHED(ctx);
  k_reduce_final_acc<K><<<1, kThreads, 0, ctx.stream>>>(ctx.d_red, nb, weight, ctx.d_scalars + slot);
  QBX_LAUNCHED(ctx);
}

}  // namespace red
}  // namespace qbx
