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

bool fast_grid_lines_b(Context& ctx, double2* grid, int n0, int n1, int n2, int axis, int dir,
                       const double2* tw) {
  const int n = axis == 0 ? n0 : axis == 1 ? n1 : n2;
  switch (n) {
    QBX_GRID_CASE(80)
    QBX_GRID_CASE(84)
    QBX_GRID_CASE(96)
    QBX_GRID_CASE(112)
    QBX_GRID_CASE(120)
    QBX_GRID_CASE(128)
    QBX_GRID_CASE(140)
    QBX_GRID_CASE(144)
    default:
      return false;
  }
}

}  // namespace qbx
