// Molecular dynamics on the device-resident wavefunctions: the reference's
// BOSampleStepper::step with atoms_dyn = MD (src/BOSampleStepper.cpp:412-1420)
// and MDIonicStepper (src/MDIonicStepper.cpp:8-273) without thermostat.
//
// Per ionic step: density, potential and energy with forces at the current
// positions; velocity Verlet on the host (3 doubles per atom); the new
// positions update the structure factors, local potential and projectors in
// place (the buffers keep their addresses, so captured electronic steps stay
// valid); the wavefunctions are extrapolated on the device (linear, with the
// previous wavefunctions aligned by a polar factor and the result Lowdin
// orthonormalised: align_to_c and lowdin of step.cu, split precision in the
// mixed path); then nitscf electronic steps.  Only positions, forces and
// energies cross to the host.
#include <cmath>
#include <cstring>
#include <vector>

#include "qbx.h"
#include "qbx_internal.h"

namespace qbx {

namespace {

constexpr double kAmu = 1822.89;   // atomic mass unit in electron masses, src/IonicStepper.cpp:40
constexpr int kThreads = 256;

int blocks(size_t n) { return (int)std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 16); }

// mode 0 (first ionic step): c <- c + dt cv, cv <- old c
// mode 1 (later steps):      c <- 2 c - cv, cv <- old c
// mode 2 (after the run):    cv <- (c - cv) / dt   (s = 1/dt)
__global__ void k_extrapolate(double* __restrict__ c, double* __restrict__ cv, size_t n, double s,
                              int mode) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double x = c[i], v = cv[i];
    if (mode == 0) {
      c[i] = x + s * v;
      cv[i] = x;
    } else if (mode == 1) {
      c[i] = 2.0 * x - v;
      cv[i] = x;
    } else {
      cv[i] = (x - v) * s;
    }
  }
}

void extrapolate(Context& c, double s, int mode) {
  const size_t n = 2 * (size_t)c.wb.ng * c.nst;
  k_extrapolate<<<blocks(n), kThreads, 0, c.stream>>>(c.d_c, c.d_wfv, n, s, mode);
  QBX_LAUNCHED(c);
}

int natoms_of(const Context& c) {
  int n = 0;
  for (auto& t : c.tau) n += (int)t.size() / 3;
  return n;
}

}  // namespace

// AtomSet::set_positions + EnergyFunctional::atoms_moved
// (src/EnergyFunctional.cpp:1047-1197) for the same atoms at new positions
// (species-major, 3 per atom): structure factors, local potential and
// pseudocharge sums, projector phases (and their split copies), E_sr with
// its forces and stress.  Buffers are updated in place.
void move_atoms(Context& c, const double* tau) {
  size_t off = 0;
  for (auto& t : c.tau) {
    std::memcpy(t.data(), tau + off, t.size() * sizeof(double));
    off += t.size();
  }
  QBX_CUDA(cudaMemcpyAsync(c.d_tau_all, tau, off * sizeof(double), cudaMemcpyHostToDevice,
                           c.stream));
  QBX_CUDA(cudaStreamSynchronize(c.stream));
  launch_setup_atoms(c);
  split_projectors(c);
  for (KPointSet& kp : c.kpts) kp.anl_ready = false;   // phases at k+G rebuilt on use
  std::vector<double> zv(c.species.size());
  for (size_t is = 0; is < c.species.size(); is++) zv[is] = c.species[is].zval;
  c.esr = esr_energy_forces(c.wb.cell, c.tau, zv, 1.5, c.fion_esr, c.sigma_esr);
  c.have_stress = false;
  QBX_CUDA(cudaStreamSynchronize(c.stream));
}

// BOSampleStepper::step(niter) with atoms_dyn = MD, wf_dyn = PSDA, nite = 0,
// the default (linear) wavefunction extrapolation and no thermostat.
// vel: initial velocities in, final velocities out (may be NULL: start at
// rest); tau_out: final positions (may be NULL); ionic: niter x 3 values
// (etotal, ekin_ion, econst) of each ionic step (may be NULL); scf: the
// QBX_NENERGY energies of each electronic step (may be NULL).
void md_run(Context& c, int niter, int nitscf, double dt, const double* mass_amu, double* vel,
            double* tau_out, double* ionic, double* scf) {
  const int nsp = (int)c.species.size();
  const int na = natoms_of(c);
  std::vector<double> pm(3 * (size_t)na);   // mass of each coordinate
  {
    size_t k = 0;
    for (int is = 0; is < nsp; is++)
      for (size_t i = 0; i < c.tau[is].size(); i++) pm[k++] = mass_amu[is] * kAmu;
  }
  std::vector<double> r0, rm, v0(3 * (size_t)na, 0.0), f;
  for (auto& t : c.tau) r0.insert(r0.end(), t.begin(), t.end());
  if (vel) std::memcpy(v0.data(), vel, v0.size() * sizeof(double));
  const size_t wf = 2 * (size_t)c.wb.ng * c.nst;
  if (!c.d_wfv) {
    // the wavefunction velocity starts at zero and persists across runs
    c.d_wfv = dalloc<double>(wf);
    QBX_CUDA(cudaMemsetAsync(c.d_wfv, 0, wf * sizeof(double), c.stream));
  }
  // energy and forces at the current positions with the current C
  auto forces_here = [&]() {
    ProfScope ps(c, "md_forces");
    update_density(c);
    update_vhxc(c);
    energy(c, false, true);
    readback(c, true);
    check_status(c);
    finish_density(c);
    finish_vhxc(c);
    finish_energy(c, true);
    f = c.fion;
  };
  auto compute_v = [&]() {
    for (size_t i = 0; i < v0.size(); i++)
      v0[i] = (r0[i] - rm[i]) / dt + dt / (2.0 * pm[i]) * f[i];
  };
  auto ekin_ion = [&]() {
    double e = 0.0;
    for (size_t i = 0; i < v0.size(); i++) e += 0.5 * pm[i] * v0[i] * v0[i];
    return e;
  };
  for (int it = 0; it < niter; it++) {
    forces_here();
    if (it > 0) compute_v();
    const double ek = ekin_ion();
    if (ionic) {
      ionic[3 * it] = c.etotal;
      ionic[3 * it + 1] = ek;
      ionic[3 * it + 2] = c.etotal + ek;
    }
    // velocity Verlet: r0 <- r0 + v0 dt + dt^2/(2m) f (MDIonicStepper::compute_r)
    std::vector<double> rp(r0.size());
    for (size_t i = 0; i < r0.size(); i++)
      rp[i] = r0[i] + v0[i] * dt + dt * dt / (2.0 * pm[i]) * f[i];
    rm = r0;
    r0 = rp;
    {
      ProfScope ps(c, "md_move_atoms");
      move_atoms(c, r0.data());
    }
    // wavefunction extrapolation (src/BOSampleStepper.cpp:731-779)
    {
      ProfScope ps(c, "md_extrapolate");
      if (it == 0) {
        extrapolate(c, dt, 0);
        gram(c, true);
      } else {
        align_to_c(c, c.d_wfv);
        extrapolate(c, 0.0, 1);
        lowdin(c);
      }
    }
    readback(c, false);
    check_status(c);
    c.extrapolate = false;   // wf_stepper->preprocess()
    for (int s = 0; s < nitscf; s++)
      scf_step_any(c, false, false,
                   scf ? scf + ((size_t)it * nitscf + s) * QBX_NENERGY : nullptr, nullptr);
  }
  // wavefunction velocity and the forces at the last positions
  // (src/BOSampleStepper.cpp:1351-1420)
  align_to_c(c, c.d_wfv);
  extrapolate(c, 1.0 / dt, 2);
  gram(c, true);
  forces_here();
  compute_v();
  if (vel) std::memcpy(vel, v0.data(), v0.size() * sizeof(double));
  if (tau_out) std::memcpy(tau_out, r0.data(), r0.size() * sizeof(double));
}

}  // namespace qbx
