// EnergyFunctional::update_vhxc and EnergyFunctional::energy on the GPU
// (src/EnergyFunctional.h:82-84,111; src/EnergyFunctional.cpp:231-1044):
// the bodies that replace the reference's in a GPU build.  The potential,
// the energy terms, H*psi (kinetic, local and nonlocal, written into dwf),
// the forces (local, nonlocal and E_sr) and the stress tensor come from the
// attached context of the Sample's SlaterDet.  Gamma, one spin, one k point,
// no confinement, external or electric-field terms.
#include <valarray>
#include <vector>

#include "EnergyFunctional.h"
#include "Sample.h"
#include "SlaterDet.h"
#include "Wavefunction.h"
#include "qbx_shim.h"

using namespace std;

void EnergyFunctional::update_vhxc(bool compute_stress, bool update_vh, bool update_vxc) {
  (void)compute_stress;
  if (!update_vh && !update_vxc) return;
  const SlaterDet& sd = *s_.wf.sd(0, 0);
  qbx_context* q = qbx_shim::context_of(sd);
  qbx_shim::check(q, qbx_update_vhxc(q));
  qbx_shim::check(q, qbx_get_vr(q, &v_r[0][0]));
}

double EnergyFunctional::energy(bool compute_hpsi, Wavefunction& dwf, bool compute_forces,
                                vector<vector<double> >& fion, bool compute_stress,
                                valarray<double>& sigma_out) {
  const SlaterDet& sd = *s_.wf.sd(0, 0);
  qbx_context* q = qbx_shim::context_of(sd);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)sd.c().cvalptr()));
  size_t natoms = 0;
  for (size_t is = 0; is < fion.size(); is++) natoms += fion[is].size() / 3;
  vector<double> f(3 * natoms + 3, 0.0);
  double e[QBX_NENERGY];
  qbx_shim::check(q, qbx_energy(q, compute_hpsi, compute_forces, e, f.data()));
  ekin_ = e[0];
  eps_ = e[1];
  enl_ = e[2];
  ehart_ = e[3];
  ecoul_ = e[4];
  exc_ = e[5];
  esr_ = e[6];
  eself_ = e[7];
  etotal_ = e[8];
  econf_ = ets_ = eexf_ = eext_ = epv_ = eefield_ = 0.0;
  enthalpy_ = etotal_;
  if (compute_hpsi) qbx_shim::check(q, qbx_get_hpsi(q, (double*)dwf.sd(0, 0)->c().valptr()));
  if (compute_forces) {
    size_t a = 0;
    for (size_t is = 0; is < fion.size(); is++)
      for (size_t i = 0; i < fion[is].size(); i++) fion[is][i] = f[a++];
  }
  if (compute_stress) {
    double sig[6], parts[36];
    qbx_shim::check(q, qbx_stress(q, sig, parts));
    // parts: ekin, eps, enl, ehart, exc, esr, six components each
    valarray<double>* part[6] = {&sigma_ekin, &sigma_eps, &sigma_enl,
                                 &sigma_ehart, &sigma_exc, &sigma_esr};
    for (int p = 0; p < 6; p++) {
      part[p]->resize(6);
      for (int k = 0; k < 6; k++) (*part[p])[k] = parts[6 * p + k];
    }
    sigma_econf.resize(6);
    sigma_econf = 0.0;
    sigma.resize(6);
    sigma_out.resize(6);
    for (int k = 0; k < 6; k++) sigma[k] = sigma_out[k] = sig[k];
  }
  return etotal_;
}
