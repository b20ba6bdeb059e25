// Scalars of the electronic step on the host side.
//
// The step's reductions leave their sums in device slots (SLOT_* of
// qbx_internal.h) and the solvers their info codes in status words; nothing
// is read back while the step runs.  enqueue_readback copies all of them (and
// the ionic forces) to pinned host mirrors as the last operation of a step,
// inside a captured graph as well, and the finish_* functions derive the
// energies the reference's EnergyFunctional reports from that copy.
#include <cmath>
#include <cstring>
#include <string>

#include "qbx_internal.h"

namespace qbx {

void enqueue_readback(Context& ctx, bool fion) {
  QBX_CUDA(cudaMemcpyAsync(ctx.h_scalars, ctx.d_scalars, kSlots * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx.stream));
  QBX_CUDA(cudaMemcpyAsync(ctx.h_status, ctx.d_status, kStatus * sizeof(int),
                           cudaMemcpyDeviceToHost, ctx.stream));
  if (fion && ctx.h_fion) {
    size_t natoms = 0;
    for (auto& t : ctx.tau) natoms += t.size() / 3;
    QBX_CUDA(cudaMemcpyAsync(ctx.h_fion, ctx.d_fion, 3 * natoms * sizeof(double),
                             cudaMemcpyDeviceToHost, ctx.stream));
  }
}

void readback(Context& ctx, bool fion) {
  enqueue_readback(ctx, fion);
  QBX_CUDA(cudaStreamSynchronize(ctx.stream));
}

double read_slot(Context& ctx, int slot) {
  QBX_REQUIRE(!ctx.capturing, 56, "host read of a device scalar inside a captured step");
  QBX_CUDA(cudaMemcpyAsync(ctx.h_scalars + slot, ctx.d_scalars + slot, sizeof(double),
                           cudaMemcpyDeviceToHost, ctx.stream));
  QBX_CUDA(cudaStreamSynchronize(ctx.stream));
  return ctx.h_scalars[slot];
}

// ChargeDensity::update_density (src/ChargeDensity.cpp:173-191): the total
// charge is the grid sum times Omega / N
void finish_density(Context& ctx) {
  ctx.total_charge = ctx.h_scalars[SLOT_CHARGE] * ctx.vb.omega / (double)ctx.N();
}

// XCPotential::update and EnergyFunctional::update_vhxc
// (src/EnergyFunctional.cpp:231-394): E_xc = Omega/N sum e_xc, E_ps and E_H
// from the G-space sums
void finish_vhxc(Context& ctx) {
  const double om = ctx.vb.omega;
  ctx.exc = ctx.h_scalars[SLOT_EXC] * om / (double)ctx.N();
  ctx.xc_rhov1 = ctx.xc == "LDA" ? 0.0 : ctx.h_scalars[SLOT_EXC + 1];
  // dxc = Omega/N sum rho (e_xc - v_xc) (src/XCPotential.cpp:199-229, 376-423)
  ctx.dxc = ctx.exc - ctx.h_scalars[SLOT_EXC + 2] * om / (double)ctx.N();
  ctx.eps = ctx.h_scalars[SLOT_EPS_EH] * om;
  ctx.ehart = om * 4.0 * M_PI * ctx.h_scalars[SLOT_EPS_EH + 1];
  ctx.ehart_e = om * 4.0 * M_PI * ctx.h_scalars[SLOT_EPS_EH + 2];
  ctx.ehart_p = om * 4.0 * M_PI * ctx.h_scalars[SLOT_EPS_EH + 3];
}

// EnergyFunctional::energy (src/EnergyFunctional.cpp:397-1044): the total
// energy and, with forces, the ionic forces (electronic part from the device
// plus the short-range ion-ion part from the host)
void finish_energy(Context& ctx, bool forces) {
  ctx.ekin = ctx.h_scalars[SLOT_EKIN];
  ctx.enl = ctx.nproj ? ctx.h_scalars[SLOT_ENL] : 0.0;
  ctx.ecoul = ctx.ehart + ctx.esr - ctx.eself;
  ctx.etotal = ctx.ekin + ctx.eps + ctx.enl + ctx.ecoul + ctx.exc;
  if (forces) {
    size_t natoms = 0;
    for (auto& t : ctx.tau) natoms += t.size() / 3;
    ctx.fion.assign(ctx.h_fion, ctx.h_fion + 3 * natoms);
    size_t a = 0;
    for (size_t is = 0; is < ctx.tau.size(); is++)
      for (size_t i = 0; i < ctx.tau[is].size(); i++) ctx.fion[a++] += ctx.fion_esr[is][i];
  }
}

void finish_eigsum(Context& ctx) { ctx.eigsum = ctx.h_scalars[SLOT_EIG]; }

void finish_theta(Context& ctx) { ctx.theta = ctx.h_scalars[SLOT_THETA]; }

void check_status(Context& ctx) {
  const int* s = ctx.h_status;
  QBX_REQUIRE(s[ST_TC_ERR] == 0, 55, "tcgen05 GEMM pipeline wait timed out");
  QBX_REQUIRE(s[ST_INFO_GRAM] == 0, 40, "Cholesky of the overlap matrix: matrix not positive "
                                        "definite (info=" + std::to_string(s[ST_INFO_GRAM]) + ")");
  QBX_REQUIRE(s[ST_INFO_ORTHO] == 0, 40, "Cholesky of the overlap matrix: matrix not positive "
                                         "definite (info=" + std::to_string(s[ST_INFO_ORTHO]) + ")");
  QBX_REQUIRE(s[ST_INFO_POLAR] == 0, 42, "LU factor of the polar iterate is singular (info=" +
                                             std::to_string(s[ST_INFO_POLAR]) + ")");
}

void bind_stream(Context& ctx, cudaStream_t s) {
  QBX_BLAS(cublasSetStream(ctx.blas, s));
  // cublasSetStream falls back to the library's default workspace; the
  // context's own keeps captured GEMMs independent of that pool
  if (ctx.d_blas_ws) QBX_BLAS(cublasSetWorkspace(ctx.blas, ctx.d_blas_ws, ctx.blas_ws_bytes));
  QBX_SOLVER(cusolverDnSetStream(ctx.solver, s));
}

}  // namespace qbx
