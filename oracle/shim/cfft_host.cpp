// Test infrastructure: the one-dimensional complex FFT that the reference's
// radial transforms (src/sinft.cpp, the FFT_NOLIB branch) call, for the
// oracle build whose src/FourierTransform.cpp (which defines it in that
// build) is replaced by the GPU FourierTransform.  Same calling convention:
// the input is z1 when *inzee == 1 (else z2), the output goes to the other
// array and *inzee names it; X_k = sum_j x_j exp(-i idir 2 pi j k / n).
// Radix-2 decimation in time for powers of two, a direct sum otherwise.
#include <cmath>
#include <complex>
#include <vector>

using std::complex;

void cfft(int idir, complex<double>* z1, complex<double>* z2, int n, int* inzee) {
  complex<double>* in = (*inzee == 1) ? z1 : z2;
  complex<double>* out = (*inzee == 1) ? z2 : z1;
  const double pi = 3.141592653589793238462643383279502884;
  if (n > 0 && (n & (n - 1)) == 0) {
    int bits = 0;
    while ((1 << bits) < n) bits++;
    for (int i = 0; i < n; i++) {
      int r = 0;
      for (int b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
      out[r] = in[i];
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len / 2;
      std::vector<complex<double> > w(half);
      for (int k = 0; k < half; k++) {
        const double a = -idir * 2.0 * pi * k / len;
        w[k] = complex<double>(std::cos(a), std::sin(a));
      }
      for (int s = 0; s < n; s += len)
        for (int k = 0; k < half; k++) {
          const complex<double> u = out[s + k], t = w[k] * out[s + k + half];
          out[s + k] = u + t;
          out[s + k + half] = u - t;
        }
    }
  } else {
    std::vector<complex<double> > tmp(n);
    for (int k = 0; k < n; k++) {
      complex<double> s = 0.0;
      for (int j = 0; j < n; j++) {
        const double a = -idir * 2.0 * pi * (double)((long long)j * k % n) / n;
        s += in[j] * complex<double>(std::cos(a), std::sin(a));
      }
      tmp[k] = s;
    }
    for (int k = 0; k < n; k++) out[k] = tmp[k];
  }
  *inzee = (*inzee == 1) ? 2 : 1;
}
