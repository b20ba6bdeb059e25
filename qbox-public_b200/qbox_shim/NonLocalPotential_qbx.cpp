// NonLocalPotential::energy on the GPU (src/NonLocalPotential.h:65-67): the
// body that replaces src/NonLocalPotential.cpp:1258-2069 in a GPU build.
// The projectors were built on the device when the atoms were set
// (qbx_set_atoms / qbx_move_atoms, the work of update_twnl); this call
// projects the attached SlaterDet's coefficients, adds the nonlocal H*psi
// into dsd, and returns E_nl, the nonlocal forces and sigma_enl.
#include <valarray>
#include <vector>

#include "AtomSet.h"
#include "NonLocalPotential.h"
#include "SlaterDet.h"
#include "qbx_shim.h"

using namespace std;

double NonLocalPotential::energy(bool compute_hpsi, SlaterDet& dsd, bool compute_forces,
                                 vector<vector<double> >& fion, bool compute_stress,
                                 valarray<double>& sigma_enl) {
  qbx_context* q = qbx_shim::context_of(sd_);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)sd_.c().cvalptr()));
  size_t natoms = 0;
  for (size_t is = 0; is < fion.size(); is++) natoms += fion[is].size() / 3;
  vector<double> f(3 * natoms + 3, 0.0);
  double sig[6] = {0, 0, 0, 0, 0, 0};
  double enl = 0.0;
  qbx_shim::check(q, qbx_nonlocal_energy(q, compute_hpsi, (double*)dsd.c().valptr(),
                                         compute_forces, f.data(), compute_stress, sig, &enl));
  if (compute_forces) {
    // species-major, as the reference's fion[is][3*ia+j]
    size_t a = 0;
    for (size_t is = 0; is < fion.size(); is++)
      for (size_t i = 0; i < fion[is].size(); i++) fion[is][i] = f[a++];
  }
  if (compute_stress) {
    sigma_enl.resize(6);
    for (int i = 0; i < 6; i++) sigma_enl[i] = sig[i];
  }
  return enl;
}
