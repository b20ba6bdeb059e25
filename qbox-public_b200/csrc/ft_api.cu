// FourierTransform on a caller's basis and grid (src/FourierTransform.h:
// 105-121): the four transforms of the reference's class on host arrays.
//
// A qbx_ft is built from what the reference's constructor reads off its
// Basis: the Miller index (h, k, l) of each local coefficient, in the
// caller's own order, whether the basis is real (the Gamma half sphere,
// each coefficient also standing for -G with the conjugate value) and the
// grid sizes np0, np1, np2.  Grids are x fastest, index i + np0*(j + np1*k)
// (FourierTransform::index).  The transforms run on the device as full-grid
// line passes (the same radix kernels as the density-basis transforms of
// the electronic step); coefficients and grids cross the host link on each
// call, as the class's host arrays require.
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/qbx.h"
#include "qbx_internal.h"

struct qbx_ft {
  qbx::Context c;             // device, stream and launch bookkeeping only
  qbx::DeviceSticks d{};
  int ng = 0;
  bool real_basis = true;
  double* d_grid = nullptr;   // np012 complex
  double* d_c = nullptr;      // two bands of ng complex
};

namespace {

template <typename F>
int ft_guarded(qbx_ft* h, F f) {
  if (!h) return 1;
  try {
    QBX_CUDA(cudaSetDevice(h->c.device));
    f(*h);
    h->c.last_error.clear();
    return 0;
  } catch (const qbx::Error& e) {
    h->c.last_error = e.msg;
    return e.code > 0 ? e.code : 1;
  } catch (const std::exception& e) {
    h->c.last_error = e.what();
    return 6;
  }
}

size_t grid_size(const qbx_ft& f) { return (size_t)f.d.n0 * f.d.n1 * f.d.n2; }

void free_ft(qbx_ft* h) {
  qbx::free_sticks(h->d);
  qbx::dfree(h->d_grid);
  qbx::dfree(h->d_c);
  if (h->c.stream) cudaStreamDestroy(h->c.stream);
  h->c.stream = nullptr;
}

}  // namespace

extern "C" {

int qbx_ft_create(qbx_ft** out, int device, int ngw, const int* hkl, int real_basis, int np0,
                  int np1, int np2) {
  if (!out) return 1;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return 8;
  if (device < 0 || device >= ndev) return 9;
  if (ngw < 1 || !hkl || np0 < 1 || np1 < 1 || np2 < 1) return 1;
  qbx_ft* h = new (std::nothrow) qbx_ft();
  if (!h) return 5;
  h->c.device = device;
  h->ng = ngw;
  h->real_basis = real_basis != 0;
  if (const char* e = std::getenv("QBX_FAST_FFT")) h->c.fast_fft = std::atoi(e) != 0;
  const int rc = ft_guarded(h, [&](qbx_ft& f) {
    QBX_CUDA(cudaStreamCreateWithFlags(&f.c.stream, cudaStreamNonBlocking));
    auto md = [](int v, int n) { return ((v % n) + n) % n; };
    std::vector<int> ip(ngw), im;
    if (f.real_basis) im.resize(ngw);
    for (int ig = 0; ig < ngw; ig++) {
      const int h0 = hkl[3 * ig], k0 = hkl[3 * ig + 1], l0 = hkl[3 * ig + 2];
      // Basis::fits_in_grid (src/Basis.cpp:139-144): -np/2 <= index < np/2
      // on each axis, for -G as well on a real basis
      auto fits = [&](int v, int n) {
        return v < n / 2 && v >= -(n / 2) && (!f.real_basis || (-v < n / 2 && -v >= -(n / 2)));
      };
      QBX_REQUIRE(fits(h0, np0) && fits(k0, np1) && fits(l0, np2), 12,
                  "basis does not fit in the FFT grid");
      ip[ig] = md(h0, np0) + np0 * (md(k0, np1) + np1 * md(l0, np2));
      if (f.real_basis) im[ig] = md(-h0, np0) + np0 * (md(-k0, np1) + np1 * md(-l0, np2));
    }
    qbx::upload_grid_map(f.d, np0, np1, np2, ip, im);
    f.d_grid = qbx::dalloc<double>(2 * grid_size(f));
    f.d_c = qbx::dalloc<double>(4 * (size_t)ngw);
  });
  if (rc) {
    free_ft(h);
    delete h;
    return rc;
  }
  *out = h;
  return 0;
}

void qbx_ft_destroy(qbx_ft* h) {
  if (!h) return;
  cudaSetDevice(h->c.device);
  if (h->c.stream) cudaStreamSynchronize(h->c.stream);
  free_ft(h);
  delete h;
}

const char* qbx_ft_last_error(qbx_ft* h) { return h ? h->c.last_error.c_str() : "null handle"; }

int qbx_ft_backward(qbx_ft* h, const double* c, double* f) {
  return ft_guarded(h, [&](qbx_ft& t) {
    QBX_REQUIRE(c && f, 1, "null coefficient or grid array");
    const size_t N = grid_size(t);
    QBX_CUDA(cudaMemcpyAsync(t.d_c, c, 2 * sizeof(double) * t.ng, cudaMemcpyHostToDevice,
                             t.c.stream));
    qbx::basis_ft_backward(t.c, t.d, t.ng, t.real_basis, t.d_c, nullptr, t.d_grid);
    QBX_CUDA(cudaMemcpyAsync(f, t.d_grid, 2 * sizeof(double) * N, cudaMemcpyDeviceToHost,
                             t.c.stream));
    QBX_CUDA(cudaStreamSynchronize(t.c.stream));
  });
}

int qbx_ft_backward2(qbx_ft* h, const double* c1, const double* c2, double* f) {
  return ft_guarded(h, [&](qbx_ft& t) {
    QBX_REQUIRE(c1 && c2 && f, 1, "null coefficient or grid array");
    QBX_REQUIRE(t.real_basis, 1, "the two-band transform needs a real basis");
    const size_t N = grid_size(t);
    const size_t nb = 2 * sizeof(double) * t.ng;
    QBX_CUDA(cudaMemcpyAsync(t.d_c, c1, nb, cudaMemcpyHostToDevice, t.c.stream));
    QBX_CUDA(cudaMemcpyAsync(t.d_c + 2 * (size_t)t.ng, c2, nb, cudaMemcpyHostToDevice, t.c.stream));
    qbx::basis_ft_backward(t.c, t.d, t.ng, true, t.d_c, t.d_c + 2 * (size_t)t.ng, t.d_grid);
    QBX_CUDA(cudaMemcpyAsync(f, t.d_grid, 2 * sizeof(double) * N, cudaMemcpyDeviceToHost,
                             t.c.stream));
    QBX_CUDA(cudaStreamSynchronize(t.c.stream));
  });
}

int qbx_ft_forward(qbx_ft* h, double* f, double* c) {
  return ft_guarded(h, [&](qbx_ft& t) {
    QBX_REQUIRE(c && f, 1, "null coefficient or grid array");
    const size_t N = grid_size(t);
    QBX_CUDA(cudaMemcpyAsync(t.d_grid, f, 2 * sizeof(double) * N, cudaMemcpyHostToDevice,
                             t.c.stream));
    qbx::basis_ft_forward(t.c, t.d, t.ng, t.real_basis, t.d_grid, t.d_c, nullptr);
    QBX_CUDA(cudaMemcpyAsync(c, t.d_c, 2 * sizeof(double) * t.ng, cudaMemcpyDeviceToHost,
                             t.c.stream));
    QBX_CUDA(cudaStreamSynchronize(t.c.stream));
  });
}

int qbx_ft_forward2(qbx_ft* h, double* f, double* c1, double* c2) {
  return ft_guarded(h, [&](qbx_ft& t) {
    QBX_REQUIRE(c1 && c2 && f, 1, "null coefficient or grid array");
    QBX_REQUIRE(t.real_basis, 1, "the two-band transform needs a real basis");
    const size_t N = grid_size(t);
    const size_t nb = 2 * sizeof(double) * t.ng;
    QBX_CUDA(cudaMemcpyAsync(t.d_grid, f, 2 * sizeof(double) * N, cudaMemcpyHostToDevice,
                             t.c.stream));
    qbx::basis_ft_forward(t.c, t.d, t.ng, true, t.d_grid, t.d_c, t.d_c + 2 * (size_t)t.ng);
    QBX_CUDA(cudaMemcpyAsync(c1, t.d_c, nb, cudaMemcpyDeviceToHost, t.c.stream));
    QBX_CUDA(cudaMemcpyAsync(c2, t.d_c + 2 * (size_t)t.ng, nb, cudaMemcpyDeviceToHost, t.c.stream));
    QBX_CUDA(cudaStreamSynchronize(t.c.stream));
  });
}

}  // extern "C"
