// PSDAWavefunctionStepper::update on the GPU (src/PSDAWavefunctionStepper.h:
// 38, src/PSDAWavefunctionStepper.cpp:46-249): residual, preconditioner,
// Anderson extrapolation and ortho_align on the device from the H*psi of the
// last EnergyFunctional::energy; the new coefficients are copied back into
// the SlaterDet.  preprocess() (the header's inline body) clears the
// extrapolation flag of this object; the device history restarts with it
// through qbx_psda_reset when the flag is seen cleared.
#include "PSDAWavefunctionStepper.h"
#include "SlaterDet.h"
#include "Wavefunction.h"
#include "qbx_shim.h"

void PSDAWavefunctionStepper::update(Wavefunction& dwf) {
  (void)dwf;   // H*psi stays on the device since the last energy()
  SlaterDet& sd = *wf_.sd(0, 0);
  qbx_context* q = qbx_shim::context_of(sd);
  if (!extrapolate_) qbx_shim::check(q, qbx_psda_reset(q));
  qbx_shim::check(q, qbx_psda_update(q));
  qbx_shim::check(q, qbx_get_coeffs(q, (double*)sd.c().valptr()));
  extrapolate_ = true;
}
