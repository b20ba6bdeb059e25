// The SCF loop of BOSampleStepper::step with nite > 0 (ground state):
// charge mixing of rho(G) with the Anderson mixer and Kerker weights,
// src/BOSampleStepper.cpp:318-410 and 781-1114, src/AndersonMixer.cpp.
//
// rho(G) and the mixer's history live on the device (2 ng_v doubles per
// vector); one reduction pass forms the mixer's normal matrix and right-hand
// side from the history, the n x n (n <= the history length) eigenproblem is
// solved on the host, and one kernel forms the next input density.  The
// electronic steps inside each SCF iteration are those of qbx_scf_step
// without the density update (energy, eigenvalue sum, PSDA update).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "qbx.h"
#include "qbx_internal.h"

namespace qbx {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxHist = 8;     // longest Anderson history supported here

int blocks(size_t n) { return (int)std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 16); }

// w_ls(G) = sqrt(G^2 / (G^2 + q1^2)), q1 = 2 pi / rc1 with rc1 = 3 bohr, and the
// Kerker weight G^2 / (G^2 + q0^2), q0 = 2 pi / rcut (1 at G = 0 and without a
// Kerker radius) (src/BOSampleStepper.cpp:344-407)
__global__ void k_mix_weights(const double* __restrict__ g2, int ng, double rcut,
                              double* __restrict__ wls, double* __restrict__ wk) {
  const double q1 = 2.0 * M_PI / 3.0;
  const double q0 = rcut > 0.0 ? 2.0 * M_PI / rcut : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double g = g2[i];
    wls[i] = g != 0.0 ? sqrt(g / (g + q1 * q1)) : 1.0;
    wk[i] = (rcut > 0.0 && g != 0.0) ? g / (g + q0 * q0) : 1.0;
  }
}

// x_k <- rho_in, f_k <- (rho - rho_in) / w_ls (the newest history entry)
__global__ void k_mix_push(const double* __restrict__ rhog, const double* __restrict__ rhog_in,
                           const double* __restrict__ wls, size_t m, double* __restrict__ xk,
                           double* __restrict__ fk) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < m;
       l += (size_t)gridDim.x * blockDim.x) {
    xk[l] = rhog_in[l];
    fk[l] = (rhog[l] - rhog_in[l]) / wls[l >> 1];
  }
}

// History vectors of the mixer: f_k and the n earlier f (k - 1 - i).
struct MixHist {
  const double* fk;
  const double* f[kMaxHist];
  int n;
};

// a(i, j) = sum_l (f_k - f_i)(f_k - f_j) for j <= i < n, packed as
// i (i + 1) / 2 + j, then b(i) = sum_l (f_k - f_i) f_k
// (src/AndersonMixer.cpp:66-95)
__global__ void k_mix_normal(MixHist h, size_t m, double* __restrict__ partial) {
  constexpr int NA = kMaxHist * (kMaxHist + 1) / 2;
  constexpr int K = NA + kMaxHist;
  __shared__ double sh[32];
  double acc[K];
#pragma unroll
  for (int q = 0; q < K; ++q) acc[q] = 0.0;
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < m;
       l += (size_t)gridDim.x * blockDim.x) {
    const double fk = h.fk[l];
    double d[kMaxHist];
#pragma unroll
    for (int i = 0; i < kMaxHist; ++i) d[i] = i < h.n ? fk - h.f[i][l] : 0.0;
#pragma unroll
    for (int i = 0; i < kMaxHist; ++i) {
#pragma unroll
      for (int j = 0; j <= i; ++j) acc[i * (i + 1) / 2 + j] += d[i] * d[j];
      acc[NA + i] += d[i] * fk;
    }
  }
#pragma unroll 1
  for (int q = 0; q < K; ++q) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) partial[(size_t)q * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

__global__ void k_mix_final(const double* __restrict__ partial, int nb, int K,
                            double* __restrict__ out) {
  __shared__ double sh[32];
  for (int q = 0; q < K; ++q) {
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += partial[(size_t)q * nb + i];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x < 32) {
      double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) out[q] = t;
    }
    __syncthreads();
  }
}

struct MixCoef {
  const double* x[kMaxHist];
  const double* f[kMaxHist];
  double theta[kMaxHist];
  int n;
};

// xbar = x_k - sum_i theta_i (x_k - x_i), fbar = f_k - sum_i theta_i (f_k - f_i)
// (src/AndersonMixer.cpp:241-256); then the next input density
// rho_in = xbar + alpha (fbar w_ls) w_kerker (src/BOSampleStepper.cpp:838-863)
__global__ void k_mix_apply(const double* __restrict__ xk, const double* __restrict__ fk,
                            MixCoef mc, const double* __restrict__ wls,
                            const double* __restrict__ wk, double alpha, size_t m,
                            double* __restrict__ rhog_in) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < m;
       l += (size_t)gridDim.x * blockDim.x) {
    const double x = xk[l], f = fk[l];
    double xb = x, fb = f;
#pragma unroll
    for (int i = 0; i < kMaxHist; ++i)
      if (i < mc.n) {
        xb -= mc.theta[i] * (x - mc.x[i][l]);
        fb -= mc.theta[i] * (f - mc.f[i][l]);
      }
    const size_t g = l >> 1;
    rhog_in[l] = xb + alpha * (fb * wls[g]) * wk[g];
  }
}

// simple mixing: rho_in += alpha (rho - rho_in) w_kerker
__global__ void k_mix_simple(const double* __restrict__ rhog, const double* __restrict__ wk,
                             double alpha, size_t m, double* __restrict__ rhog_in) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < m;
       l += (size_t)gridDim.x * blockDim.x)
    rhog_in[l] += alpha * (rhog[l] - rhog_in[l]) * wk[l >> 1];
}

__global__ void k_scale(double* __restrict__ x, size_t n, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

// Eigen-decomposition of a symmetric n x n matrix (column-major, full) by
// cyclic Jacobi rotations: w ascending, columns of v the eigenvectors.
void jacobi_eigen(int n, std::vector<double> a, std::vector<double>& w, std::vector<double>& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) v[i + i * n] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += a[p + q * n] * a[p + q * n];
    if (off == 0.0) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a[p + q * n];
        if (apq == 0.0) continue;
        const double app = a[p + p * n], aqq = a[q + q * n];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; k++) {
          const double akp = a[k + p * n], akq = a[k + q * n];
          a[k + p * n] = c * akp - s * akq;
          a[k + q * n] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          const double apk = a[p + k * n], aqk = a[q + k * n];
          a[p + k * n] = c * apk - s * aqk;
          a[q + k * n] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = v[k + p * n], vkq = v[k + q * n];
          v[k + p * n] = c * vkp - s * vkq;
          v[k + q * n] = s * vkp + c * vkq;
        }
      }
  }
  // ascending order
  std::vector<int> idx(n);
  for (int i = 0; i < n; i++) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return a[x + x * n] < a[y + y * n]; });
  std::vector<double> v2((size_t)n * n);
  w.assign(n, 0.0);
  for (int j = 0; j < n; j++) {
    w[j] = a[idx[j] + idx[j] * n];
    for (int k = 0; k < n; k++) v2[k + j * n] = v[k + idx[j] * n];
  }
  v.swap(v2);
}

// The Anderson mixer's history on the device (AndersonMixer with diag = true
// and eig_ratio = 0, src/AndersonMixer.cpp:28-256).
struct Mixer {
  int nmax = 0, n = -1, k = -1;
  size_t m = 0;
  double* x(Context& c, int i) const { return c.d_mix + (size_t)i * m; }
  double* f(Context& c, int i) const { return c.d_mix + (size_t)(nmax + 1 + i) * m; }
};

void ensure_mix_buffers(Context& c, int ndim, double rcut) {
  const int ngv = c.vb.ng;
  const size_t m = 2 * (size_t)ngv;
  if (c.mix_ndim != ndim) {
    dfree(c.d_mix);
    if (ndim > 0) c.d_mix = dalloc<double>(2 * (size_t)(ndim + 1) * m);
    c.mix_ndim = ndim;
  }
  if (!c.d_rhog_in) c.d_rhog_in = dalloc<double>(m);
  if (!c.d_wmix) {
    c.d_wmix = dalloc<double>(2 * (size_t)ngv);
    c.mix_rcut = -1.0;
  }
  if (c.mix_rcut != rcut) {
    double* d_g2 = dupload(c.vb.g2);   // |G|^2 of the density basis
    k_mix_weights<<<blocks(ngv), kThreads, 0, c.stream>>>(d_g2, ngv, rcut, c.d_wmix,
                                                          c.d_wmix + ngv);
    QBX_LAUNCHED(c);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    dfree(d_g2);
    c.mix_rcut = rcut;
  }
}

// rho(r) = Re FFT_bwd(rho(G)) / Omega and its charge (ChargeDensity::update_rhor,
// src/ChargeDensity.cpp:201-240)
void update_rhor(Context& c) {
  vb_backward(c, c.d_rhog, c.d_rhor);
  k_scale<<<blocks(c.N()), kThreads, 0, c.stream>>>(c.d_rhor, c.N(), 1.0 / c.vb.omega);
  QBX_LAUNCHED(c);
  launch_sum(c, c.d_rhor, c.N(), SLOT_CHARGE);
}

// AndersonMixer::update followed by the Kerker step of the input density.
void mix_update(Context& c, Mixer& mx, double alpha) {
  const int ngv = c.vb.ng;
  const size_t m = mx.m;
  const double* wls = c.d_wmix;
  const double* wk = c.d_wmix + ngv;
  mx.k = (mx.k + 1) % (mx.nmax + 1);
  if (mx.n < mx.nmax) mx.n++;
  const int k = mx.k, n = mx.n;
  k_mix_push<<<blocks(m), kThreads, 0, c.stream>>>(c.d_rhog, c.d_rhog_in, wls, m, mx.x(c, k),
                                                   mx.f(c, k));
  QBX_LAUNCHED(c);
  MixCoef mc{};
  mc.n = n;
  if (n > 0) {
    MixHist h{};
    h.fk = mx.f(c, k);
    h.n = n;
    for (int i = 0; i < n; i++) {
      const int kmi = (k - i + mx.nmax) % (mx.nmax + 1);
      h.f[i] = mx.f(c, kmi);
      mc.f[i] = mx.f(c, kmi);
      mc.x[i] = mx.x(c, kmi);
    }
    constexpr int K = kMaxHist * (kMaxHist + 1) / 2 + kMaxHist;
    static_assert(SLOT_MIX + K <= kSlots, "mixer slots");
    // partials of K sums per block in the 4096-double reduction buffer
    const int nb = (int)std::max<size_t>(1, std::min<size_t>(4 * 1024 / K, (m + kThreads - 1) / kThreads));
    k_mix_normal<<<nb, kThreads, 0, c.stream>>>(h, m, c.d_red);
    QBX_LAUNCHED(c);
    k_mix_final<<<1, kThreads, 0, c.stream>>>(c.d_red, nb, K, c.d_scalars + SLOT_MIX);
    QBX_LAUNCHED(c);
    readback(c, false);
    const double* r = c.h_scalars + SLOT_MIX;
    constexpr int NA = kMaxHist * (kMaxHist + 1) / 2;
    std::vector<double> a((size_t)n * n), b(n), w, u;
    for (int i = 0; i < n; i++) {
      for (int j = 0; j <= i; j++) a[i + j * n] = a[j + i * n] = r[i * (i + 1) / 2 + j];
      b[i] = r[NA + i];
    }
    jacobi_eigen(n, a, w, u);
    for (int i = 0; i < n; i++) mc.theta[i] = 0.0;
    for (int q = 0; q < n; q++)
      if (w[q] > 0.0 * w[n - 1]) {
        double ub = 0.0;
        for (int j = 0; j < n; j++) ub += u[j + q * n] * b[j];
        for (int i = 0; i < n; i++) mc.theta[i] += (ub / w[q]) * u[i + q * n];
      }
  }
  k_mix_apply<<<blocks(m), kThreads, 0, c.stream>>>(mx.x(c, k), mx.f(c, k), mc, wls, wk, alpha,
                                                    m, c.d_rhog_in);
  QBX_LAUNCHED(c);
}

}  // namespace

void free_mix(Context& c) {
  dfree(c.d_rhog_in);
  dfree(c.d_mix);
  dfree(c.d_wmix);
  c.mix_ndim = -1;
  c.mix_rcut = -1.0;
}

// BOSampleStepper::step(0) (ground state, atoms fixed) with wf_dyn = PSDA:
// nitscf SCF iterations; with nite > 0 each mixes the new density into the
// input density, rebuilds the potentials and runs up to nite electronic
// steps (stopping once the eigenvalue sum moves less than 0.01 of the
// Hartree energy change); etotal_int[it] is the Harris-Foulkes estimate of
// iteration it, eigsum[it * max(nite, 1) + ite] the eigenvalue sum of each
// electronic step, nite_done[it] the steps run.  Stops early when the
// spread of the last three etotal_int is below scf_tol.
void scf_run(Context& c, int nitscf, int nite, double mix_coeff, double mix_rcut, int mix_ndim,
             double scf_tol, double* etotal_int, double* eigsum, int* nite_done,
             int* nitscf_done) {
  QBX_REQUIRE(mix_ndim >= 0 && mix_ndim <= kMaxHist, 1, "charge_mix_ndim must be 0 .. 8");
  const int ngv = c.vb.ng;
  const size_t m = 2 * (size_t)ngv;
  if (nite > 0) ensure_mix_buffers(c, mix_ndim, mix_rcut);
  Mixer mx;
  mx.nmax = mix_ndim;
  mx.m = m;
  c.extrapolate = false;                 // wf_stepper->preprocess()
  double ehart = 0.0, ehart_m = 0.0, delta_ehart = 0.0;
  double etot = 0.0, etot_m = 0.0, etot_mm = 0.0;
  const int nsteps = std::max(nite, 1);
  int it = 0;
  for (; it < nitscf; it++) {
    update_density(c);
    if (nite > 0) {
      if (it == 0) {
        QBX_CUDA(cudaMemcpyAsync(c.d_rhog_in, c.d_rhog, m * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c.stream));
      } else {
        if (mix_ndim > 0) {
          mix_update(c, mx, mix_coeff);
        } else {
          k_mix_simple<<<blocks(m), kThreads, 0, c.stream>>>(c.d_rhog, c.d_wmix + ngv, mix_coeff,
                                                             m, c.d_rhog_in);
          QBX_LAUNCHED(c);
        }
        QBX_CUDA(cudaMemcpyAsync(c.d_rhog, c.d_rhog_in, m * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c.stream));
        update_rhor(c);
      }
    }
    update_vhxc(c);
    readback(c, false);
    finish_density(c);
    finish_vhxc(c);
    if (nite > 0) c.extrapolate = false;   // preprocess of each SCF iteration
    if (it == 0) {
      ehart = c.ehart;
      delta_ehart = 0.0;
    } else if (it == 1) {
      ehart_m = ehart;
      ehart = c.ehart;
      delta_ehart = std::fabs(ehart - ehart_m);
    } else {
      ehart_m = ehart;
      ehart = c.ehart;
      delta_ehart = std::min(delta_ehart, std::fabs(ehart - ehart_m));
    }
    double eig = 0.0, eig_m = 0.0;
    bool conv = false;
    int ite = 0;
    while (!conv && ite < nsteps) {
      energy(c, true, false);
      launch_eigsum(c);
      readback(c, false);
      check_status(c);
      finish_energy(c, false);
      finish_eigsum(c);
      if (ite > 0) eig_m = eig;
      eig = c.eigsum;
      if (eigsum) eigsum[(size_t)it * nsteps + ite] = eig;
      psda_update(c, PSDA_PREC_FROM_ENERGY);   // energy() ran on this C
      if (ite > 0) conv = std::fabs(eig - eig_m) < 0.01 * delta_ehart;
      ite++;
    }
    readback(c, false);
    check_status(c);
    finish_theta(c);
    if (nite_done) nite_done[it] = ite;
    // Harris-Foulkes estimate (src/BOSampleStepper.cpp:1075-1077), two
    // electrons per band
    const double eint = 2.0 * eig - c.ehart_e + c.ehart_p + c.esr - c.eself + c.dxc;
    if (etotal_int) etotal_int[it] = eint;
    etot_mm = etot_m;
    etot_m = etot;
    etot = eint;
    double d = std::fabs(etot - etot_m);
    d = std::max(d, std::fabs(etot - etot_mm));
    d = std::max(d, std::fabs(etot_m - etot_mm));
    if (d < scf_tol) {
      it++;
      break;
    }
  }
  if (nitscf_done) *nitscf_done = it;
}

}  // namespace qbx
