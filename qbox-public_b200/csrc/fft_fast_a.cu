// Specialised staged FFT kernels, grid lengths of the small cells
// (8-atom cell and the 32-system batch: 36 ... 72).
#include "fft_fast.cuh"

namespace qbx {

bool fast_staged_a(Context& ctx, const fast::StagedArgs& a, size_t smem_limit) {
  const DeviceSticks& g = ctx.dws;
  if (g.n0 != g.n1 || g.n0 != g.n2) return false;
  switch (g.n0) {
    QBX_FAST_CASE(36)
    QBX_FAST_CASE(40)
    QBX_FAST_CASE(42)
    QBX_FAST_CASE(48)
    QBX_FAST_CASE(56)
    QBX_FAST_CASE(60)
    QBX_FAST_CASE(64)
    QBX_FAST_CASE(66)
    QBX_FAST_CASE(70)
    QBX_FAST_CASE(72)
    default:
      return false;
  }
}

bool fast_grid_lines_a(Context& ctx, double2* grid, int n0, int n1, int n2, int axis, int dir,
                       const double2* tw) {
  const int n = axis == 0 ? n0 : axis == 1 ? n1 : n2;
  switch (n) {
    QBX_GRID_CASE(36)
    QBX_GRID_CASE(40)
    QBX_GRID_CASE(42)
    QBX_GRID_CASE(48)
    QBX_GRID_CASE(56)
    QBX_GRID_CASE(60)
    QBX_GRID_CASE(64)
    QBX_GRID_CASE(66)
    QBX_GRID_CASE(70)
    QBX_GRID_CASE(72)
    default:
      return false;
  }
}

}  // namespace qbx
