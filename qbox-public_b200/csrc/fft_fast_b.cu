// Specialised staged FFT kernels, grid lengths of the larger cells
// (64-atom cell 84, water 112, 512-atom cell 140, and neighbours).
#include "fft_fast.cuh"

namespace qbx {

bool fast_staged_b(Context& ctx, const fast::StagedArgs& a, size_t smem_limit) {
  const DeviceSticks& g = ctx.dws;
  if (g.n0 != g.n1 || g.n0 != g.n2) return false;
  switch (g.n0) {
    QBX_FAST_CASE(80)
    QBX_FAST_CASE(84)
    QBX_FAST_CASE(96)
    QBX_FAST_CASE(112)
    QBX_FAST_CASE(120)
    QBX_FAST_CASE(128)
    QBX_FAST_CASE(140)
    QBX_FAST_CASE(144)
    default:
      return false;
  }
}

}  // namespace qbx
