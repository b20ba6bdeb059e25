// The Qbox side of the drop-in: replacement bodies for the reference's
// classes on the electronic-step path, compiled inside a Qbox build against
// its unchanged headers (FourierTransform.h, SlaterDet.h,
// NonLocalPotential.h, ChargeDensity.h, EnergyFunctional.h,
// PSDAWavefunctionStepper.h) and linked with libqbx.
//
// Ownership: a SlaterDet whose methods run on the GPU has a qbx_context
// attached (attach(), after SlaterDet::resize and the species and atoms are
// known).  That context holds the device copy of the coefficients; the
// replacement bodies upload the host coefficients before an operation that
// reads them and download them after one that changes them, so the
// reference's host ComplexMatrix stays valid for the code around them.
// Errors come back from the C ABI as status codes and leave as the
// reference's exceptions (SlaterDetException, std::runtime_error).
#ifndef QBX_SHIM_H
#define QBX_SHIM_H

#include <qbx.h>

class SlaterDet;

namespace qbx_shim {

// The GPU context of a SlaterDet (one per SlaterDet; single task, the
// reference's Context collapsed to one process).
void attach(const SlaterDet& sd, qbx_context* q);
void detach(const SlaterDet& sd);
qbx_context* context_of(const SlaterDet& sd);

// Throws the reference's SlaterDetException with qbx_last_error on rc != 0.
void check(qbx_context* q, int rc);

// The device index the FourierTransform objects use (QBX_DEVICE, else 0).
int device();

}  // namespace qbx_shim

#endif
