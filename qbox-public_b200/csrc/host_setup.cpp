// Host-side setup of the electronic step: plane-wave basis and staged-FFT
// stick geometry, species G-space tables, and the pseudocharge repulsion
// energy.  These are per-geometry (not per-step) computations that the
// reference performs in Basis::resize, BasisMapping, Species::initialize_slpp
// and EnergyFunctional::atoms_moved.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <stdexcept>
#include <thread>

#include "qbx_internal.h"

namespace qbx {

// ---------------------------------------------------------------- sizes
bool factorizable(int n) {
  // Basis::factorizable, src/Basis.cpp:105-133
  if (n % 11 == 0) n /= 11;
  if (n % 7 == 0) n /= 7;
  if (n % 5 == 0) n /= 5;
  if (n % 3 == 0) n /= 3;
  if (n % 3 == 0) n /= 3;
  while (n % 2 == 0) n /= 2;
  return n == 1;
}

static double norm3(const double* v) {
  return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

static int hmax_of(const double cell[9], double ecut, int dir) {
  const double fac = std::sqrt(2.0 * ecut) / (2.0 * M_PI);
  return (int)(1.5 + fac * norm3(cell + 3 * dir));
}

int fft_size(const double cell[9], double ecut, int dir) {
  // src/Basis.cpp:513-521
  int n = 2 * hmax_of(cell, ecut, dir);
  while (!factorizable(n)) n += 2;
  return n;
}

void dense_grid(const double cell[9], double ecut_wf, int np[3]) {
  // src/ChargeDensity.cpp:36-49: density basis at 4 ecut, grid size + 2
  for (int i = 0; i < 3; i++) {
    int n = fft_size(cell, 4.0 * ecut_wf, i) + 2;
    while (!factorizable(n)) n += 2;
    np[i] = n;
  }
}

RadixPlan make_plan(int n) {
  RadixPlan p;
  p.n = n;
  int m = n;
  // radix 4 for the power-of-two part, then 2, then the odd factors
  while (m % 4 == 0) { p.radix[p.nstage++] = 4; m /= 4; }
  while (m % 2 == 0) { p.radix[p.nstage++] = 2; m /= 2; }
  const int odd[4] = {3, 5, 7, 11};
  for (int f : odd)
    while (m % f == 0) { p.radix[p.nstage++] = f; m /= f; }
  QBX_REQUIRE(m == 1, 10, "FFT length " + std::to_string(n) + " has an unsupported factor");
  QBX_REQUIRE(p.nstage <= 12, 10, "too many FFT stages");
  return p;
}

// ---------------------------------------------------------------- basis
void build_basis(Basis& b, const double cell[9], double ecut) {
  std::memcpy(b.cell, cell, 9 * sizeof(double));
  // reciprocal vectors b_i = 2 pi (a_j x a_k) / omega
  const double* a0 = cell;
  const double* a1 = cell + 3;
  const double* a2 = cell + 6;
  auto cross = [](const double* u, const double* v, double* w) {
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
  };
  double c12[3], c20[3], c01[3];
  cross(a1, a2, c12);
  cross(a2, a0, c20);
  cross(a0, a1, c01);
  const double vol = a0[0] * c12[0] + a0[1] * c12[1] + a0[2] * c12[2];
  QBX_REQUIRE(vol > 0, 11, "cell volume must be positive");
  b.omega = vol;
  for (int i = 0; i < 3; i++) {
    b.recip[i] = 2.0 * M_PI * c12[i] / vol;
    b.recip[3 + i] = 2.0 * M_PI * c20[i] / vol;
    b.recip[6 + i] = 2.0 * M_PI * c01[i] / vol;
  }
  b.ecut = ecut;
  const double two_ecut = 2.0 * ecut;
  const int hmax = hmax_of(cell, ecut, 0);
  const int kmax = hmax_of(cell, ecut, 1);
  const int lmax = hmax_of(cell, ecut, 2);
  const double* B0 = b.recip;
  const double* B1 = b.recip + 3;
  const double* B2 = b.recip + 6;
  auto gnorm2 = [&](int h, int k, int l) {
    double x = h * B0[0] + k * B1[0] + l * B2[0];
    double y = h * B0[1] + k * B1[1] + l * B2[1];
    double z = h * B0[2] + k * B1[2] + l * B2[2];
    return x * x + y * y + z * z;
  };
  b.rod_h.clear(); b.rod_k.clear(); b.rod_lmin.clear(); b.rod_size.clear();
  // Gamma half sphere: rod (0,0,l>=0), rods (0,k>0,l), rods (h>0,k,l)
  // (the rod set of src/Basis.cpp:357-447), here in sorted (h,k) order.
  for (int h = 0; h <= hmax; h++) {
    for (int k = (h == 0 ? 0 : -kmax); k <= kmax; k++) {
      int lstart = lmax + 1, lend = -lmax - 1;
      const int lfrom = (h == 0 && k == 0) ? 0 : -lmax;
      for (int l = lfrom; l <= lmax; l++)
        if (gnorm2(h, k, l) < two_ecut) {
          lstart = std::min(lstart, l);
          lend = std::max(lend, l);
        }
      if (lend >= lstart) {
        b.rod_h.push_back(h);
        b.rod_k.push_back(k);
        b.rod_lmin.push_back(lstart);
        b.rod_size.push_back(lend - lstart + 1);
      }
    }
  }
  b.nrods = (int)b.rod_h.size();
  QBX_REQUIRE(b.nrods > 0 && b.rod_h[0] == 0 && b.rod_k[0] == 0 && b.rod_lmin[0] == 0,
              11, "basis has no G=0 rod");
  b.rod_first.resize(b.nrods);
  int ng = 0;
  for (int r = 0; r < b.nrods; r++) { b.rod_first[r] = ng; ng += b.rod_size[r]; }
  b.ng = ng;
  b.hkl.resize(3 * ng);
  b.gx.resize(3 * ng);
  b.g2.resize(ng); b.g.resize(ng); b.gi.resize(ng); b.g2i.resize(ng);
  for (int r = 0; r < b.nrods; r++)
    for (int i = 0; i < b.rod_size[r]; i++) {
      const int ig = b.rod_first[r] + i;
      const int h = b.rod_h[r], k = b.rod_k[r], l = b.rod_lmin[r] + i;
      b.hkl[3 * ig] = h; b.hkl[3 * ig + 1] = k; b.hkl[3 * ig + 2] = l;
      // Basis::update_g, src/Basis.cpp:646-690
      const double x = h * B0[0] + k * B1[0] + l * B2[0];
      const double y = h * B0[1] + k * B1[1] + l * B2[1];
      const double z = h * B0[2] + k * B1[2] + l * B2[2];
      b.gx[ig] = x; b.gx[ng + ig] = y; b.gx[2 * ng + ig] = z;
      b.g2[ig] = x * x + y * y + z * z;
      b.g[ig] = std::sqrt(b.g2[ig]);
      b.gi[ig] = b.g[ig] > 0.0 ? 1.0 / b.g[ig] : 0.0;
      b.g2i[ig] = b.gi[ig] * b.gi[ig];
    }
  b.g0 = 0;
}

// The complex basis at k (units of the reciprocal vectors): the rods of
// every (h,k) column with some |k+G|^2 < 2 ecut over the whole sphere
// (src/Basis.cpp:449-486), here in sorted (h,k) order, l ascending; gx, g2,
// g, gi, g2i hold k+G and its norms (Basis::update_g kpg*, :646-690).
void build_kbasis(Basis& b, const double cell[9], double ecut, const double kp[3]) {
  build_basis(b, cell, ecut);   // cell, reciprocal vectors, volume
  b.complex_basis = true;
  b.kpoint[0] = kp[0]; b.kpoint[1] = kp[1]; b.kpoint[2] = kp[2];
  const double two_ecut = 2.0 * ecut;
  const int hmax = hmax_of(cell, ecut, 0);
  const int kmax = hmax_of(cell, ecut, 1);
  const int lmax = hmax_of(cell, ecut, 2);
  const double* B0 = b.recip;
  const double* B1 = b.recip + 3;
  const double* B2 = b.recip + 6;
  auto q = [&](double h, double k, double l, double* out) {
    for (int i = 0; i < 3; i++) out[i] = h * B0[i] + k * B1[i] + l * B2[i];
  };
  b.rod_h.clear(); b.rod_k.clear(); b.rod_lmin.clear(); b.rod_size.clear();
  for (int h = -hmax; h <= hmax; h++)
    for (int k = -kmax; k <= kmax; k++) {
      int lstart = lmax + 1, lend = -lmax - 1;
      for (int l = -lmax; l <= lmax; l++) {
        double v[3];
        q(kp[0] + h, kp[1] + k, kp[2] + l, v);
        if (v[0] * v[0] + v[1] * v[1] + v[2] * v[2] < two_ecut) {
          lstart = std::min(lstart, l);
          lend = std::max(lend, l);
        }
      }
      if (lend >= lstart) {
        b.rod_h.push_back(h);
        b.rod_k.push_back(k);
        b.rod_lmin.push_back(lstart);
        b.rod_size.push_back(lend - lstart + 1);
      }
    }
  b.nrods = (int)b.rod_h.size();
  QBX_REQUIRE(b.nrods > 0, 11, "empty basis at this k point");
  b.rod_first.resize(b.nrods);
  int ng = 0;
  for (int r = 0; r < b.nrods; r++) { b.rod_first[r] = ng; ng += b.rod_size[r]; }
  b.ng = ng;
  b.hkl.resize(3 * ng);
  b.gx.resize(3 * ng);
  b.g2.resize(ng); b.g.resize(ng); b.gi.resize(ng); b.g2i.resize(ng);
  b.first = -1;
  for (int r = 0; r < b.nrods; r++)
    for (int i = 0; i < b.rod_size[r]; i++) {
      const int ig = b.rod_first[r] + i;
      const int h = b.rod_h[r], k = b.rod_k[r], l = b.rod_lmin[r] + i;
      b.hkl[3 * ig] = h; b.hkl[3 * ig + 1] = k; b.hkl[3 * ig + 2] = l;
      double v[3];
      q(kp[0] + h, kp[1] + k, kp[2] + l, v);
      b.gx[ig] = v[0]; b.gx[ng + ig] = v[1]; b.gx[2 * ng + ig] = v[2];
      b.g2[ig] = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      b.g[ig] = std::sqrt(b.g2[ig]);
      b.gi[ig] = b.g[ig] > 0.0 ? 1.0 / b.g[ig] : 0.0;
      b.g2i[ig] = b.gi[ig] * b.gi[ig];
      // the reference moves rod (0,0) to the front of its local basis
      // (src/Basis.cpp:587-597): its lowest l is the first coefficient
      if (h == 0 && k == 0 && i == 0) b.first = ig;
    }
  QBX_REQUIRE(b.first >= 0, 11, "the basis at this k point has no (0,0) rod");
  b.g0 = -1;   // no G = 0 coefficient constraint on a complex basis
}

// Stick geometry of a complex basis on the grid: one stick per rod.
void set_grid_complex(Basis& b, int n0, int n1, int n2) {
  b.n0 = n0; b.n1 = n1; b.n2 = n2;
  b.nvec = b.nrods;
  b.stick_x.assign(b.nvec, 0);
  b.stick_y.assign(b.nvec, 0);
  auto md = [](int v, int n) { return ((v % n) + n) % n; };
  for (int r = 0; r < b.nrods; r++) {
    const int h = b.rod_h[r], k = b.rod_k[r];
    QBX_REQUIRE(2 * std::abs(h) < n0 && 2 * std::abs(k) < n1, 12,
                "basis does not fit in the FFT grid");
    QBX_REQUIRE(2 * std::max(std::abs(b.rod_lmin[r]),
                             std::abs(b.rod_lmin[r] + b.rod_size[r] - 1)) < n2,
                12, "basis does not fit in the FFT grid");
    b.stick_x[r] = md(h, n0);
    b.stick_y[r] = md(k, n1);
  }
  std::map<int, int> cols;
  for (int s = 0; s < b.nvec; s++) cols[b.stick_x[s]] = 0;
  b.col_x.clear();
  for (auto& kv : cols) { kv.second = (int)b.col_x.size(); b.col_x.push_back(kv.first); }
  b.ncol = (int)b.col_x.size();
  b.stick_col.resize(b.nvec);
  for (int s = 0; s < b.nvec; s++) b.stick_col[s] = cols[b.stick_x[s]];
  b.ip.resize(b.ng);
  b.im.assign(b.ng, 0);
  for (int ig = 0; ig < b.ng; ig++) {
    const int h = b.hkl[3 * ig], k = b.hkl[3 * ig + 1], l = b.hkl[3 * ig + 2];
    b.ip[ig] = md(h, n0) + n0 * (md(k, n1) + n1 * md(l, n2));
  }
}

void set_grid(Basis& b, int n0, int n1, int n2) {
  b.n0 = n0; b.n1 = n1; b.n2 = n2;
  b.nvec = 2 * b.nrods - 1;
  b.stick_x.assign(b.nvec, 0);
  b.stick_y.assign(b.nvec, 0);
  auto md = [](int v, int n) { return ((v % n) + n) % n; };
  for (int r = 0; r < b.nrods; r++) {
    const int h = b.rod_h[r], k = b.rod_k[r];
    // the basis must fit in the grid (BasisMapping ctor assert)
    QBX_REQUIRE(2 * std::abs(h) < n0 && 2 * std::abs(k) < n1, 12,
                "basis does not fit in the FFT grid");
    QBX_REQUIRE(2 * std::max(std::abs(b.rod_lmin[r]),
                             std::abs(b.rod_lmin[r] + b.rod_size[r] - 1)) < n2,
                12, "basis does not fit in the FFT grid");
    if (r == 0) {
      b.stick_x[0] = 0; b.stick_y[0] = 0;
    } else {
      b.stick_x[2 * r - 1] = md(h, n0); b.stick_y[2 * r - 1] = md(k, n1);
      b.stick_x[2 * r] = md(-h, n0);    b.stick_y[2 * r] = md(-k, n1);
    }
  }
  std::map<int, int> cols;
  for (int s = 0; s < b.nvec; s++) cols[b.stick_x[s]] = 0;
  b.col_x.clear();
  for (auto& kv : cols) { kv.second = (int)b.col_x.size(); b.col_x.push_back(kv.first); }
  b.ncol = (int)b.col_x.size();
  b.stick_col.resize(b.nvec);
  for (int s = 0; s < b.nvec; s++) b.stick_col[s] = cols[b.stick_x[s]];
  b.ip.resize(b.ng);
  b.im.resize(b.ng);
  for (int ig = 0; ig < b.ng; ig++) {
    const int h = b.hkl[3 * ig], k = b.hkl[3 * ig + 1], l = b.hkl[3 * ig + 2];
    b.ip[ig] = md(h, n0) + n0 * (md(k, n1) + n1 * md(l, n2));
    b.im[ig] = md(-h, n0) + n0 * (md(-k, n1) + n1 * md(-l, n2));
  }
}

// ------------------------------------------------------------- species
// Radix-2 complex FFT with the e^{-i} sign, used by the radial sine and
// cosine transforms below (length 2*ndft, a power of two).
static void fft_pow2(std::vector<std::complex<double>>& a) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * M_PI / (double)len;
    for (size_t i = 0; i < n; i += len)
      for (size_t j = 0; j < len / 2; j++) {
        const std::complex<double> w(std::cos(ang * j), std::sin(ang * j));
        const std::complex<double> u = a[i + j], v = a[i + j + len / 2] * w;
        a[i + j] = u + v;
        a[i + j + len / 2] = u - v;
      }
  }
}

// y_k = sum_{j=1}^{n-1} y_j sin(pi j k / n)  (src/sinft.cpp sinft)
static void sinft(std::vector<double>& y) {
  const int n = (int)y.size();
  std::vector<std::complex<double>> z(2 * n, 0.0);
  for (int i = 1; i < n; i++) { z[i] = y[i]; z[2 * n - i] = -y[i]; }
  fft_pow2(z);
  for (int i = 0; i < n; i++) y[i] = -0.5 * z[i].imag();
}

// y has n+1 entries on input; the first n are replaced by
// 0.5 y_0 + sum_{j=1}^{n-1} y_j cos(pi j k/n) + 0.5 (-1)^k y_n  (cosft1)
static void cosft1(std::vector<double>& y, int n) {
  std::vector<std::complex<double>> z(2 * n, 0.0);
  z[0] = y[0];
  for (int i = 1; i < n + 1; i++) { z[i] = y[i]; z[2 * n - i] = y[i]; }
  fft_pow2(z);
  for (int i = 0; i < n; i++) y[i] = 0.5 * z[i].real();
}

// end-corrected trapezoid rule of src/Species.cpp:34-48
static double simpsn(const std::vector<double>& t) {
  const int n = (int)t.size();
  const double c0 = 17.0 / 48.0, c1 = 59.0 / 48.0, c2 = 43.0 / 48.0, c3 = 49.0 / 48.0;
  double s = c0 * (t[0] + t[n - 1]) + c1 * (t[1] + t[n - 2]) + c2 * (t[2] + t[n - 3]) +
             c3 * (t[3] + t[n - 4]);
  for (int i = 4; i < n - 4; i++) s += t[i];
  return s;
}

// cubic spline second derivatives (src/spline.cpp spline/tridsolve)
static void spline(const std::vector<double>& x, const std::vector<double>& y,
                   double ypl, double ypr, int natl, int natr,
                   std::vector<double>& y2) {
  const int n = (int)x.size();
  std::vector<double> d(n), e(n), f(n);
  y2.assign(n, 0.0);
  const double third = 1.0 / 3.0, sixth = 1.0 / 6.0;
  if (natl == 0) {
    const double h = x[1] - x[0];
    d[0] = third * h; e[0] = sixth * h; f[0] = 0.0;
    y2[0] = (y[1] - y[0]) / h - ypl;
  } else { d[0] = 1.0; e[0] = 0.0; f[0] = 0.0; y2[0] = 0.0; }
  if (natr == 0) {
    const double h = x[n - 1] - x[n - 2];
    d[n - 1] = third * h; e[n - 1] = 0.0; f[n - 1] = sixth * h;
    y2[n - 1] = ypr - (y[n - 1] - y[n - 2]) / h;
  } else { d[n - 1] = 1.0; e[n - 1] = 0.0; f[n - 1] = 0.0; y2[n - 1] = 0.0; }
  for (int i = 1; i < n - 1; i++) {
    const double hp = x[i + 1] - x[i], hm = x[i] - x[i - 1];
    d[i] = third * (hp + hm);
    e[i] = sixth * hp;
    f[i] = sixth * hm;
    y2[i] = (y[i + 1] - y[i]) / hp - (y[i] - y[i - 1]) / hm;
  }
  for (int i = 1; i < n; i++) { f[i] /= d[i - 1]; d[i] -= f[i] * e[i - 1]; }
  for (int i = 1; i < n; i++) y2[i] -= f[i] * y2[i - 1];
  y2[n - 1] /= d[n - 1];
  for (int i = n - 2; i >= 0; i--) y2[i] = (y2[i] - e[i] * y2[i + 1]) / d[i];
}

// value and derivative of the spline (src/spline.cpp splintd)
static void splintd(const std::vector<double>& xa, const std::vector<double>& ya,
                    const std::vector<double>& y2a, double x, double& y, double& dy) {
  int kl = 0, kh = (int)xa.size() - 1;
  while (kh - kl > 1) {
    const int k = (kh + kl) / 2;
    if (xa[k] > x) kh = k; else kl = k;
  }
  const double h = xa[kh] - xa[kl];
  const double a = (xa[kh] - x) / h, b = (x - xa[kl]) / h;
  y = a * ya[kl] + b * ya[kh] +
      h * h * (1.0 / 6.0) * ((a * a * a - a) * y2a[kl] + (b * b * b - b) * y2a[kh]);
  dy = (ya[kh] - ya[kl]) / h +
       h * (((1.0 / 6.0) - 0.5 * a * a) * y2a[kl] + (0.5 * b * b - (1.0 / 6.0)) * y2a[kh]);
}

double SpeciesTables::eself() const {
  return zval * zval / (std::sqrt(2.0 * M_PI) * rcps);
}

void SpeciesTables::dvlocg(double g, double& v, double& dv) const {
  if (g > gspl[ndft - 1]) { v = 0.0; dv = 0.0; return; }
  splintd(gspl, vlocg, vlocg2, g, v, dv);
}

void SpeciesTables::dvnlg(int iop, double g, double& v, double& dv) const {
  if (g > gspl[ndft - 1]) { v = 0.0; dv = 0.0; return; }
  splintd(gspl, vnlg[iop], vnlg2[iop], g, v, dv);
}

double SpeciesTables::rhopsg(double g) const {
  return -zval * std::exp(-0.25 * rcps * rcps * g * g);
}

// Species::initialize_slpp (src/Species.cpp:510-1055) for s and p projectors:
// extend V_loc with -Z/r, subtract the Gaussian pseudocharge potential
// Z erf(r/rcps)/r, sine-transform to G, spline; projectors by the l=0 sine
// transform and the l=1 sine/cosine combination of j_1.
void species_from_radial(SpeciesTables& s, int zval, double dr, int np,
                         const double* vlocal, int nproj, const int* proj_l,
                         const double* proj, const double* proj_d) {
  QBX_REQUIRE(dr > 0.0001 && np > 8, 13, "bad radial mesh");
  const double fpi = 4.0 * M_PI;
  s.zval = zval;
  s.rcps = 1.5;
  int ndft = 1;
  while (ndft * dr < 40.0) ndft *= 2;
  QBX_REQUIRE(np <= ndft, 13, "radial mesh longer than the transform length");
  s.ndft = ndft;
  std::vector<double> r(ndft);
  for (int i = 0; i < ndft; i++) r[i] = i * dr;
  std::vector<double> vlocr(ndft);
  for (int i = 0; i < np; i++) vlocr[i] = vlocal[i];
  for (int i = np; i < ndft; i++) vlocr[i] = -zval / r[i];
  const double z = zval;
  vlocr[0] += (z / s.rcps) * (2.0 / std::sqrt(M_PI));
  for (int i = 1; i < ndft; i++) vlocr[i] += (z / r[i]) * std::erf(r[i] / s.rcps);
  for (int i = 0; i < ndft; i++) vlocr[i] *= fpi * r[i] * dr;
  std::vector<double> fint(ndft);
  for (int i = 0; i < ndft; i++) fint[i] = vlocr[i] * r[i];
  const double v0 = simpsn(fint);
  s.vlocg = vlocr;
  sinft(s.vlocg);
  s.gspl.resize(ndft);
  const double fac = M_PI / (ndft * dr);
  s.gspl[0] = 0.0;
  s.vlocg[0] = v0;
  for (int i = 1; i < ndft; i++) {
    s.gspl[i] = i * fac;
    s.vlocg[i] /= s.gspl[i];
  }
  spline(s.gspl, s.vlocg, 0.0, 0.0, 0, 1, s.vlocg2);

  s.proj_l.clear(); s.proj_d.clear(); s.vnlg.clear(); s.vnlg2.clear();
  for (int iop = 0; iop < nproj; iop++) {
    const int l = proj_l[iop];
    QBX_REQUIRE(l == 0 || l == 1, 13, "only s and p projectors are supported");
    std::vector<double> vnlr(ndft, 0.0);
    for (int i = 0; i < np; i++) vnlr[i] = fpi * dr * proj[(size_t)iop * np + i];
    std::vector<double> t(ndft), t2;
    if (l == 0) {
      for (int i = 0; i < ndft; i++) fint[i] = vnlr[i] * r[i] * r[i];
      const double p0 = simpsn(fint);
      for (int i = 0; i < ndft; i++) t[i] = vnlr[i] * r[i];
      sinft(t);
      t[0] = p0;
      for (int i = 1; i < ndft; i++) t[i] /= s.gspl[i];
      spline(s.gspl, t, 0.0, 0.0, 0, 1, t2);
    } else {
      std::vector<double> sp = vnlr;
      sinft(sp);
      fint[0] = 0.0;
      for (int i = 1; i < ndft; i++) fint[i] = sp[i] / (s.gspl[i] * s.gspl[i]);
      std::vector<double> cp(ndft + 1, 0.0);
      for (int i = 0; i < ndft; i++) cp[i] = vnlr[i] * r[i];
      cosft1(cp, ndft);
      t[0] = 0.0;
      for (int i = 1; i < ndft; i++) t[i] = fint[i] - cp[i] / s.gspl[i];
      spline(s.gspl, t, 0.0, 0.0, 1, 1, t2);
    }
    s.proj_l.push_back(l);
    s.proj_d.push_back(proj_d ? proj_d[iop] : 1.0);
    s.vnlg.push_back(t);
    s.vnlg2.push_back(t2);
  }
}

// --------------------------------------------------------------- E_sr
// UnitCell::fold_in_ws (src/UnitCell.cpp:157-187)
static void fold_in_ws(const double cell[9], double v[3]) {
  double an[13][3];
  const double* a = cell;
  for (int j = 0; j < 3; j++) {
    an[0][j] = a[j]; an[1][j] = a[3 + j]; an[2][j] = a[6 + j];
    an[3][j] = a[j] + a[3 + j]; an[4][j] = a[j] - a[3 + j];
    an[5][j] = a[3 + j] + a[6 + j]; an[6][j] = a[3 + j] - a[6 + j];
    an[7][j] = a[6 + j] + a[j]; an[8][j] = a[6 + j] - a[j];
    an[9][j] = a[j] + a[3 + j] + a[6 + j]; an[10][j] = a[j] - a[3 + j] - a[6 + j];
    an[11][j] = a[j] + a[3 + j] - a[6 + j]; an[12][j] = a[j] - a[3 + j] + a[6 + j];
  }
  const double eps = 1.e-10;
  for (int iter = 0; iter < 10; iter++) {
    bool done = true;
    for (int i = 0; i < 13; i++) {
      const double h = 0.5 * (an[i][0] * an[i][0] + an[i][1] * an[i][1] + an[i][2] * an[i][2]);
      auto dot = [&]() { return v[0] * an[i][0] + v[1] * an[i][1] + v[2] * an[i][2]; };
      const double sp = dot();
      if (sp > h + eps) {
        done = false;
        do { for (int j = 0; j < 3; j++) v[j] -= an[i][j]; } while (dot() > h + eps);
      } else if (sp < -h - eps) {
        done = false;
        do { for (int j = 0; j < 3; j++) v[j] += an[i][j]; } while (dot() < -h - eps);
      }
    }
    if (done) return;
  }
}

// Pseudocharge repulsion energy and forces, lattice sum over neighbouring
// cells (EnergyFunctional::atoms_moved, src/EnergyFunctional.cpp:1112-1192).
double esr_energy_forces(const double cell[9],
                         const std::vector<std::vector<double>>& tau,
                         const std::vector<double>& zv, double rcps,
                         std::vector<std::vector<double>>& f, double* sigma) {
  // Voigt pairs xx yy zz xy yz xz; sigma_esr = -(1/Omega) sum dedr x_i x_j
  // (src/EnergyFunctional.cpp:1173-1194)
  static const int vi[6] = {0, 1, 2, 0, 1, 0}, vj[6] = {0, 1, 2, 1, 2, 2};
  double sig[6] = {0, 0, 0, 0, 0, 0};
  const int nsp = (int)tau.size();
  f.assign(nsp, std::vector<double>());
  for (int is = 0; is < nsp; is++) f[is].assign(tau[is].size(), 0.0);
  // distance between opposite planes of the cell: 2 pi / |b_i|
  double recip[9];
  {
    Basis b;
    build_basis(b, cell, 0.01);
    std::memcpy(recip, b.recip, sizeof(recip));
  }
  double d[3];
  for (int i = 0; i < 3; i++) d[i] = 2.0 * M_PI / norm3(recip + 3 * i);
  // Pairs (is1 <= is2; ia2 >= ia1 within a species) in the reference's order,
  // the outer atom index split over host threads with private sums that are
  // added at the end (only the summation order differs from one thread).
  struct Part {
    double esr = 0.0;
    double sig[6] = {0, 0, 0, 0, 0, 0};
    std::vector<std::vector<double>> f;
  };
  const double rc12 = std::sqrt(rcps * rcps + rcps * rcps);
  const int nc0 = (int)(8.0 * rc12 / d[0]);
  const int nc1 = (int)(8.0 * rc12 / d[1]);
  const int nc2 = (int)(8.0 * rc12 / d[2]);
  int natoms = 0;
  for (int is = 0; is < nsp; is++) natoms += (int)tau[is].size() / 3;
  const int nthreads = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(),
                                                 std::min(16, natoms / 32)));
  std::vector<Part> parts(nthreads);
  auto work = [&](int t) {
    Part& P = parts[t];
    P.f.assign(nsp, std::vector<double>());
    for (int is = 0; is < nsp; is++) P.f[is].assign(tau[is].size(), 0.0);
    for (int is1 = 0; is1 < nsp; is1++)
      for (int is2 = is1; is2 < nsp; is2++) {
        const int na1 = (int)tau[is1].size() / 3, na2 = (int)tau[is2].size() / 3;
        for (int ia1 = t; ia1 < na1; ia1 += nthreads) {
          const int ia2min = (is1 == is2) ? ia1 : 0;
          for (int ia2 = ia2min; ia2 < na2; ia2++) {
            const bool same = (is1 == is2 && ia1 == ia2);
            double v12[3];
            for (int j = 0; j < 3; j++) v12[j] = tau[is1][3 * ia1 + j] - tau[is2][3 * ia2 + j];
            fold_in_ws(cell, v12);
            for (int i0 = -nc0; i0 <= nc0; i0++)
              for (int i1 = -nc1; i1 <= nc1; i1++)
                for (int i2 = -nc2; i2 <= nc2; i2++) {
                  if (same && i0 == 0 && i1 == 0 && i2 == 0) continue;
                  const double fac = same ? 0.5 : 1.0;
                  double x[3];
                  for (int j = 0; j < 3; j++)
                    x[j] = v12[j] + i0 * cell[j] + i1 * cell[3 + j] + i2 * cell[6 + j];
                  const double r12 = norm3(x);
                  const double arg = r12 / rc12;
                  const double term = zv[is1] * zv[is2] * std::erfc(arg) / r12;
                  P.esr += fac * term;
                  const double de = 2.0 * zv[is1] * zv[is2] * std::exp(-arg * arg) /
                                    (rc12 * std::sqrt(M_PI));
                  const double dedr = -fac * (term + de) / (r12 * r12);
                  for (int j = 0; j < 3; j++) {
                    P.f[is1][3 * ia1 + j] -= dedr * x[j];
                    P.f[is2][3 * ia2 + j] += dedr * x[j];
                  }
                  for (int k = 0; k < 6; k++) P.sig[k] += dedr * x[vi[k]] * x[vj[k]];
                }
          }
        }
      }
  };
  if (nthreads == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  double esr = 0.0;
  for (const Part& P : parts) {
    esr += P.esr;
    for (int k = 0; k < 6; k++) sig[k] += P.sig[k];
    for (int is = 0; is < nsp; is++)
      for (size_t i = 0; i < f[is].size(); i++) f[is][i] += P.f[is][i];
  }
  if (sigma) {
    const double* a = cell;
    const double omega = std::fabs(a[0] * (a[4] * a[8] - a[5] * a[7]) -
                                   a[1] * (a[3] * a[8] - a[5] * a[6]) +
                                   a[2] * (a[3] * a[7] - a[4] * a[6]));
    for (int k = 0; k < 6; k++) sigma[k] = -sig[k] / omega;
  }
  return esr;
}

}  // namespace qbx
