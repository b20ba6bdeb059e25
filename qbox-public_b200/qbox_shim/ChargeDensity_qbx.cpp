// ChargeDensity::update_density on the GPU (src/ChargeDensity.h:58,
// src/ChargeDensity.cpp:136-198): the body that replaces the reference's in
// a GPU build.  rho(r) is formed on the device from the attached
// SlaterDet's coefficients and copied into rhor[0]; rho(G) on the density
// basis follows through the density FourierTransform (vft_, itself on the
// GPU when FourierTransform.cpp is the replacement in this directory).
// Gamma, one spin, one k point, one task.
#include <complex>
#include <stdexcept>

#include "Basis.h"
#include "ChargeDensity.h"
#include "FourierTransform.h"
#include "SlaterDet.h"
#include "UnitCell.h"
#include "Wavefunction.h"
#include "qbx_shim.h"

using namespace std;

void ChargeDensity::update_density(void) {
  if (wf_.nspin() != 1 || wf_.nkp() != 1)
    throw runtime_error("ChargeDensity on the GPU: one spin and the Gamma point only");
  const SlaterDet& sd = *wf_.sd(0, 0);
  qbx_context* q = qbx_shim::context_of(sd);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)sd.c().cvalptr()));
  double charge = 0.0;
  qbx_shim::check(q, qbx_update_density(q, &charge));
  qbx_shim::check(q, qbx_get_density(q, &rhor[0][0]));
  total_charge_[0] = charge;
  const double omega = vbasis_->cell().volume();
  for (size_t i = 0; i < rhor[0].size(); i++) rhotmp[i] = complex<double>(omega * rhor[0][i], 0.0);
  vft_->forward(&rhotmp[0], &rhog[0][0]);
}
