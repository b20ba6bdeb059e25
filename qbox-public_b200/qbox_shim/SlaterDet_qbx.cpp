// SlaterDet methods of the electronic step on the GPU (src/SlaterDet.h:
// 66-77): bodies that replace those of src/SlaterDet.cpp in a GPU build.
// The SlaterDet's coefficients are uploaded to its attached context before
// each operation and, where the operation changes them, downloaded after.
// The FourierTransform argument of compute_density / rs_mul_add names the
// grid; the context transforms on its own dense grid, which is the grid of
// ChargeDensity's wavefunction transforms (src/ChargeDensity.cpp:44-49,98).
#include <complex>
#include <stdexcept>

#include "FourierTransform.h"
#include "SlaterDet.h"
#include "qbx_shim.h"

using namespace std;

namespace {

void require_grid(qbx_context* q, const FourierTransform& ft) {
  int ngw = 0, ngv = 0, np[3] = {0, 0, 0};
  qbx_shim::check(q, qbx_basis_sizes(q, &ngw, &ngv, np));
  if (np[0] != ft.np0() || np[1] != ft.np1() || np[2] != ft.np2())
    throw SlaterDetException("SlaterDet on the GPU: the transform's grid is not the context's");
}

}  // namespace

void SlaterDet::compute_density(FourierTransform& ft, double weight, double* rho) const {
  qbx_context* q = qbx_shim::context_of(*this);
  require_grid(q, ft);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)c_.cvalptr()));
  qbx_shim::check(q, qbx_compute_density(q, weight, rho));
}

void SlaterDet::rs_mul_add(FourierTransform& ft, const double* v, SlaterDet& sdp) const {
  qbx_context* q = qbx_shim::context_of(*this);
  require_grid(q, ft);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)c_.cvalptr()));
  qbx_shim::check(q, qbx_rs_mul_add(q, v, (double*)sdp.c().valptr()));
}

void SlaterDet::gram(void) {
  qbx_context* q = qbx_shim::context_of(*this);
  qbx_shim::check(q, qbx_set_coeffs(q, (const double*)c_.cvalptr()));
  qbx_shim::check(q, qbx_gram(q));
  qbx_shim::check(q, qbx_get_coeffs(q, (double*)c_.valptr()));
}

void SlaterDet::ortho_align(const SlaterDet& sd) {
  qbx_context* q = qbx_shim::context_of(*this);
  qbx_shim::check(q, qbx_set_coeffs(q, (const double*)c_.cvalptr()));
  qbx_shim::check(q, qbx_ortho_align(q, (const double*)sd.c().cvalptr()));
  qbx_shim::check(q, qbx_get_coeffs(q, (double*)c_.valptr()));
}

complex<double> SlaterDet::dot(const SlaterDet& sd) const {
  qbx_context* q = qbx_shim::context_of(*this);
  qbx_shim::check(q, qbx_set_coeffs_async(q, (const double*)c_.cvalptr()));
  double d = 0.0;
  qbx_shim::check(q, qbx_dot(q, (const double*)sd.c().cvalptr(), &d));
  return complex<double>(d, 0.0);
}
