// qbx_density_static: the band-pair charge density for callers that cannot
// allocate device memory.
//
// Some callers of this library cannot call cudaMalloc at the point where
// they need the density: code that runs inside a host callback or a driver
// plug-in where allocation is forbidden, a process whose device memory is
// carved up ahead of time by another framework's pool, or a long-running
// service that must not grow its footprint after start-up.  They own the
// coefficients and the density grid, but not the stick scratch buffer that
// the staged FFT needs.  This entry point takes that scratch, and the twiddle
// and weight tables, from one file-scope device array instead.
//
// The array is QBX_STATIC_SCRATCH_BYTES long and lives on every GPU that
// loads the library until the process exits.  All calls on a device share
// it and it keeps the previous call's contents; every region a call reads is
// written by that call first.  Two calls whose work overlaps on one GPU (two
// host threads, or two contexts on different streams) race on it.
#include <string>

#include "../../include/qbx.h"
#include "qbx_internal.h"

struct qbx_context;   // defined in capi.cu
namespace qbx {
Context& context_of(qbx_context* h);
}

namespace {

constexpr size_t kScratchBytes = QBX_STATIC_SCRATCH_BYTES;
// [0, kTableBytes): twiddle tables (x, y, z) then the band weights;
// [kTableBytes, kScratchBytes): the stick buffer.
constexpr size_t kTableBytes = (size_t)1 << 20;
constexpr int kMaxLen = 4096;   // longest FFT length whose table fits

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch in the CUDA context current on the calling
// thread.  A __device__ symbol's address belongs to a context, not to a
// device ordinal (a plug-in's own driver-API context on the same device, or
// the context made after a cudaDeviceReset, places the array elsewhere), so
// it is looked up on every call; the lookup allocates nothing.
void* scratch_address() {
  void* p = nullptr;
  QBX_CUDA(cudaGetSymbolAddress(&p, g_scratch));
  QBX_REQUIRE(p != nullptr, 61, "no device address for the static scratch array");
  return p;
}

// exp(+2 pi i k/n) for the three axis lengths, and the band weights
// w_n = occ_n / Omega (w holds occ_n on entry, or is filled with 2/Omega
// when have_occ is 0).
__global__ void k_static_tables(double2* tw, int n0, int n1, int n2, double* w, int nst,
                                int have_occ, double inv_omega) {
  const int total = n0 + n1 + n2;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total + nst;
       t += gridDim.x * blockDim.x) {
    if (t < total) {
      const int n = t < n0 ? n0 : (t < n0 + n1 ? n1 : n2);
      const int k = t < n0 ? t : (t < n0 + n1 ? t - n0 : t - n0 - n1);
      double s, c;
      sincospi(2.0 * (double)k / (double)n, &s, &c);
      tw[t] = make_double2(c, s);
    } else {
      const int b = t - total;
      w[b] = (have_occ ? w[b] : 2.0) * inv_omega;
    }
  }
}

}  // namespace

extern "C" int qbx_density_static(qbx_context* h, const double* d_c, int nst, const double* occ,
                                  double* d_rho) {
  if (!h) return 1;
  qbx::Context& c = qbx::context_of(h);
  try {
    QBX_CUDA(cudaSetDevice(c.device));
    QBX_REQUIRE(c.have_cell, 7, "qbx_set_cell has not been called");
    QBX_REQUIRE(d_c && d_rho && nst > 0, 1, "null coefficient or density pointer, or nst < 1");
    const int n0 = c.wb.n0, n1 = c.wb.n1, n2 = c.wb.n2;
    QBX_REQUIRE(n0 <= kMaxLen && n1 <= kMaxLen && n2 <= kMaxLen, 62,
                "FFT length exceeds the static table limit of 4096");
    const size_t table_bytes = sizeof(double2) * ((size_t)n0 + n1 + n2) + sizeof(double) * nst;
    QBX_REQUIRE(table_bytes <= kTableBytes, 62,
                "band count too large for the static weight table");
    const size_t per_pair = qbx::density_stick_bytes_per_pair(c);
    QBX_REQUIRE(per_pair <= kScratchBytes - kTableBytes, 62,
                "one band pair's z-sticks (" + std::to_string(per_pair) +
                    " bytes) exceed the static scratch of " +
                    std::to_string(kScratchBytes - kTableBytes) + " bytes");
    unsigned char* base = (unsigned char*)scratch_address();
    double2* twx = (double2*)base;
    double2* twy = twx + n0;
    double2* twz = twy + n1;
    double* w = (double*)(twz + n2);
    // tables, rewritten on every call: the array keeps whatever the last
    // call (of any context on this device) left in it
    if (occ)
      QBX_CUDA(cudaMemcpyAsync(w, occ, sizeof(double) * nst, cudaMemcpyHostToDevice, c.stream));
    k_static_tables<<<32, 256, 0, c.stream>>>(twx, n0, n1, n2, w, nst, occ ? 1 : 0,
                                              1.0 / c.wb.omega);
    QBX_LAUNCHED(c);
    QBX_CUDA(cudaMemsetAsync(d_rho, 0, c.N() * sizeof(double), c.stream));
    qbx::density_with_buffers(c, d_c, nst, w, d_rho, base + kTableBytes,
                              kScratchBytes - kTableBytes, twx, twy, twz);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    c.last_error.clear();
    return 0;
  } catch (const qbx::Error& e) {
    c.last_error = e.msg;
    return e.code > 0 ? e.code : 1;
  } catch (const std::exception& e) {
    c.last_error = e.what();
    return 6;
  }
}
