// FourierTransform on the GPU: a drop-in replacement of the reference's
// src/FourierTransform.cpp behind its unchanged header
// (src/FourierTransform.h:52-170).  Every public member keeps its meaning:
// backward = unscaled synthesis on the grid, forward = analysis with 1/N,
// single and two-band (real basis) forms, grids x fastest.  The transforms
// are the qbx_ft_* entry points of libqbx (include/qbx.h); the object keeps
// its BasisMapping member for the inline accessors (np2_loc, ...) of the
// header.  Single task only: the basis must not be distributed.
#include "FourierTransform.h"

#include <cstdlib>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "Basis.h"
#include "qbx_shim.h"

using namespace std;

namespace {

mutex g_mu;
map<const FourierTransform*, qbx_ft*>& handles() {
  static map<const FourierTransform*, qbx_ft*> h;
  return h;
}

qbx_ft* handle(const FourierTransform* t) {
  lock_guard<mutex> lock(g_mu);
  auto it = handles().find(t);
  if (it == handles().end()) throw runtime_error("FourierTransform: no GPU transform");
  return it->second;
}

void check(qbx_ft* h, int rc, const char* what) {
  if (rc) throw runtime_error(string("FourierTransform::") + what + ": " + qbx_ft_last_error(h));
}

}  // namespace

FourierTransform::FourierTransform(const Basis& basis, int np0, int np1, int np2)
    : basis_(basis), bm_(BasisMapping(basis, np0, np1, np2)), np0_(np0), np1_(np1), np2_(np2),
      nvec_(bm_.nvec()) {
  if (basis.npes() != 1)
    throw runtime_error("FourierTransform on the GPU: the basis must not be distributed");
  ntrans0_ = max(abs(basis_.idxmax(1)), abs(basis_.idxmin(1))) + 1;
  ntrans1_ = np0_;
  ntrans2_ = nvec_;
  qbx_ft* h = nullptr;
  const int rc = qbx_ft_create(&h, qbx_shim::device(), basis.localsize(), basis.idx_ptr(),
                               basis.real() ? 1 : 0, np0, np1, np2);
  if (rc) throw runtime_error("FourierTransform: qbx_ft_create failed, code " + to_string(rc));
  lock_guard<mutex> lock(g_mu);
  handles()[this] = h;
}

FourierTransform::~FourierTransform() {
  qbx_ft* h = nullptr;
  {
    lock_guard<mutex> lock(g_mu);
    auto it = handles().find(this);
    if (it != handles().end()) {
      h = it->second;
      handles().erase(it);
    }
  }
  qbx_ft_destroy(h);
}

void FourierTransform::backward(const complex<double>* c, complex<double>* f) {
  qbx_ft* h = handle(this);
  check(h, qbx_ft_backward(h, (const double*)c, (double*)f), "backward");
}

void FourierTransform::backward(const complex<double>* c1, const complex<double>* c2,
                                complex<double>* f) {
  qbx_ft* h = handle(this);
  check(h, qbx_ft_backward2(h, (const double*)c1, (const double*)c2, (double*)f), "backward");
}

void FourierTransform::forward(complex<double>* f, complex<double>* c) {
  qbx_ft* h = handle(this);
  check(h, qbx_ft_forward(h, (double*)f, (double*)c), "forward");
}

void FourierTransform::forward(complex<double>* f, complex<double>* c1, complex<double>* c2) {
  qbx_ft* h = handle(this);
  check(h, qbx_ft_forward2(h, (double*)f, (double*)c1, (double*)c2), "forward");
}

void FourierTransform::reset_timers(void) {
  for (Timer* t : {&tm_fwd, &tm_bwd, &tm_map_fwd, &tm_map_bwd, &tm_trans_fwd, &tm_trans_bwd,
                   &tm_fxy, &tm_fxy_inv, &tm_fz, &tm_fz_inv, &tm_init})
    t->reset();
}
