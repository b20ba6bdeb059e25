// Device helpers of the hi/lo splits of the mixed path, shared by the split
// kernels and the kernels that write a split as a by-product of their pass.
#pragma once

#include <cuda_bf16.h>

namespace qbx {

// round an FP32 value to TF32 (10 explicit mantissa bits), nearest with
// ties away from zero; finite inputs only
__device__ __forceinline__ float tf32_round(float x) {
  unsigned u = __float_as_uint(x);
  u = (u + 0x1000u) & 0xffffe000u;
  return __uint_as_float(u);
}

// hi = round(v), lo = round(v - hi) in BF16 and in TF32 (held in FP32)
__device__ __forceinline__ void split_bf16(double v, __nv_bfloat16& h, __nv_bfloat16& l) {
  h = __double2bfloat16(v);
  l = __double2bfloat16(v - (double)__bfloat162float(h));
}
__device__ __forceinline__ void split_tf32(double v, float& h, float& l) {
  h = tf32_round((float)v);
  l = tf32_round((float)(v - (double)h));
}

// The splits of rows r .. r + 3 (r a multiple of 4) of column c of an FP64
// block, given as v: BF16 hi/lo at ld ldb when r < ldb (8-byte stores; rows
// past the block's end come in as zeros and fill the padding) and/or TF32
// hi/lo at ld ldt for the rows below `rows` (one 16-byte store when all four
// are).  hi = round(x), lo = round(x - hi) in each format.
template <bool BF, bool TF>
__device__ __forceinline__ void store_splits4(const double (&v)[4], int r, int rows, int c,
                                              __nv_bfloat16* __restrict__ bhi,
                                              __nv_bfloat16* __restrict__ blo, int ldb,
                                              float* __restrict__ thi, float* __restrict__ tlo,
                                              int ldt) {
  if constexpr (BF) {
    __nv_bfloat16 h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) split_bf16(v[q], h[q], l[q]);
    if (r < ldb) {
      *reinterpret_cast<uint2*>(bhi + (size_t)c * ldb + r) = *reinterpret_cast<uint2*>(h);
      *reinterpret_cast<uint2*>(blo + (size_t)c * ldb + r) = *reinterpret_cast<uint2*>(l);
    }
  }
  if constexpr (TF) {
    float h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) split_tf32(v[q], h[q], l[q]);
    if (r + 3 < rows) {
      *reinterpret_cast<float4*>(thi + (size_t)c * ldt + r) = make_float4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<float4*>(tlo + (size_t)c * ldt + r) = make_float4(l[0], l[1], l[2], l[3]);
    } else {
      for (int q = 0; q < 4 && r + q < rows; ++q) {
        thi[(size_t)c * ldt + r + q] = h[q];
        tlo[(size_t)c * ldt + r + q] = l[q];
      }
    }
  }
}

}  // namespace qbx
