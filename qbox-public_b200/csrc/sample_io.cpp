// The <wavefunction> element of a Qbox sample file: written as
// Wavefunction::print / SlaterDet::print write it (src/Wavefunction.cpp:919-962,
// src/SlaterDet.cpp:1382-1549, base64 encoding of each band's real values on
// the wavefunction basis's own FFT grid, Base64Transcoder's 72-character
// lines), and read back as the reference's handler does (each grid function
// transformed forward onto the coefficients, the diagonal density matrix as
// the occupations; src/WavefunctionHandler.cpp:150-175, 340-370, 560-605).
// The transforms run on the device; the host only encodes and parses text.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "qbx_internal.h"

namespace qbx {

namespace {

const char kB64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

std::string b64_encode(const unsigned char* p, size_t n) {
  std::string out;
  out.reserve((n + 2) / 3 * 4);
  size_t i = 0;
  for (; i + 3 <= n; i += 3) {
    const unsigned v = (p[i] << 16) | (p[i + 1] << 8) | p[i + 2];
    out += kB64[(v >> 18) & 63];
    out += kB64[(v >> 12) & 63];
    out += kB64[(v >> 6) & 63];
    out += kB64[v & 63];
  }
  if (n - i == 1) {
    const unsigned v = p[i] << 16;
    out += kB64[(v >> 18) & 63];
    out += kB64[(v >> 12) & 63];
    out += "==";
  } else if (n - i == 2) {
    const unsigned v = (p[i] << 16) | (p[i + 1] << 8);
    out += kB64[(v >> 18) & 63];
    out += kB64[(v >> 12) & 63];
    out += kB64[(v >> 6) & 63];
    out += '=';
  }
  return out;
}

// decodes base64 characters of [b, e), skipping everything else
std::vector<unsigned char> b64_decode(const char* b, const char* e) {
  int table[256];
  for (int& t : table) t = -1;
  for (int i = 0; i < 64; i++) table[(unsigned char)kB64[i]] = i;
  std::vector<unsigned char> out;
  out.reserve((size_t)(e - b) * 3 / 4);
  unsigned v = 0;
  int bits = 0;
  for (const char* q = b; q < e; q++) {
    if (*q == '=') break;
    const int t = table[(unsigned char)*q];
    if (t < 0) continue;
    v = (v << 6) | (unsigned)t;
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back((unsigned char)((v >> bits) & 0xFF));
    }
  }
  return out;
}

// value of attribute `name` inside the tag text [b, e)
std::string attr(const std::string& s, size_t b, size_t e, const std::string& name) {
  const std::string key = name + "=\"";
  const size_t p = s.find(key, b);
  QBX_REQUIRE(p != std::string::npos && p < e, 70, "attribute " + name + " missing");
  const size_t q = s.find('"', p + key.size());
  return s.substr(p + key.size(), q - p - key.size());
}

int nel_of(const Context& c) {
  double s = 0.0;
  for (double o : c.occ) s += o;
  return (int)std::lround(s);
}

// the wavefunction basis on its own FFT grid (Basis::resize,
// src/Basis.cpp:509-521), built on first use
void ensure_wf_grid(Context& c) {
  if (c.have_wgrid) return;
  Basis b = c.wb;
  int np[3];
  for (int i = 0; i < 3; i++) np[i] = fft_size(c.wb.cell, c.wb.ecut, i);
  set_grid(b, np[0], np[1], np[2]);
  upload_sticks(c.dwg, b);
  c.have_wgrid = true;
}

void print_vec(std::ostream& os, const double* v) { os << v[0] << " " << v[1] << " " << v[2]; }

}  // namespace

void write_wavefunction(Context& c, std::ostream& os) {
  ensure_wf_grid(c);
  const DeviceSticks& d = c.dwg;
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  const int ngw = c.wb.ng;
  os << "<wavefunction ecut=\"" << c.wb.ecut << "\" nspin=\"1\" nel=\"" << nel_of(c)
     << "\" nempty=\"0\">" << std::endl;
  os << std::setprecision(10);
  const double* a = c.wb.cell;
  for (const char* tag : {"domain", "reference_domain"}) {
    os << "<" << tag << " a=\"";
    print_vec(os, a);
    os << "\"\n        b=\"";
    print_vec(os, a + 3);
    os << "\"\n        c=\"";
    print_vec(os, a + 6);
    os << "\"/>" << std::endl;
  }
  os << "<grid nx=\"" << d.n0 << "\" ny=\"" << d.n1 << "\" nz=\"" << d.n2 << "\"/>" << std::endl;
  const double zero[3] = {0.0, 0.0, 0.0};
  os << "<slater_determinant kpoint=\"";
  print_vec(os, zero);
  os << "\"\n  weight=\"" << std::setprecision(12) << 1.0 << "\" size=\"" << c.nst << "\">"
     << std::endl;
  os << "<density_matrix form=\"diagonal\" size=\"" << c.nst << "\">" << std::endl;
  os.setf(std::ios::fixed, std::ios::floatfield);
  os.setf(std::ios::right, std::ios::adjustfield);
  for (int i = 0; i < c.nst; i++) {
    os << " " << std::setprecision(8) << c.occ[i];
    if (i % 10 == 9) os << std::endl;
  }
  if (c.nst % 10 != 0) os << std::endl;
  os << "</density_matrix>" << std::endl;
  std::vector<double> f(N);
  for (int n = 0; n < c.nst; n++) {
    wfgrid_backward(c, d, ngw, c.d_c + 2 * (size_t)n * ngw, c.d_grad);
    QBX_CUDA(cudaMemcpyAsync(f.data(), c.d_grad, N * sizeof(double), cudaMemcpyDeviceToHost,
                             c.stream));
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    const std::string e = b64_encode(reinterpret_cast<const unsigned char*>(f.data()),
                                     N * sizeof(double));
    os << "<grid_function type=\"double\" nx=\"" << d.n0 << "\" ny=\"" << d.n1 << "\" nz=\""
       << d.n2 << "\" encoding=\"base64\">" << std::endl;
    for (size_t p = 0; p < e.size(); p += 72) os << e.substr(p, 72) << '\n';
    os << "</grid_function>\n";
  }
  os << "</slater_determinant>" << std::endl;
  os << "</wavefunction>" << std::endl;
}

void read_wavefunction(Context& c, const std::string& s) {
  ensure_wf_grid(c);
  const DeviceSticks& d = c.dwg;
  const size_t N = (size_t)d.n0 * d.n1 * d.n2;
  const int ngw = c.wb.ng;
  const size_t g = s.find("<grid ");
  QBX_REQUIRE(g != std::string::npos, 70, "no <grid> element");
  const size_t ge = s.find('>', g);
  const int nx = std::stoi(attr(s, g, ge, "nx")), ny = std::stoi(attr(s, g, ge, "ny")),
            nz = std::stoi(attr(s, g, ge, "nz"));
  QBX_REQUIRE(nx == d.n0 && ny == d.n1 && nz == d.n2, 71,
              "wavefunction grid differs from this basis's grid");
  // occupations from the diagonal density matrix
  const size_t dm = s.find("<density_matrix");
  if (dm != std::string::npos) {
    const size_t db = s.find('>', dm) + 1, de = s.find("</density_matrix>", db);
    std::istringstream is(s.substr(db, de - db));
    std::vector<double> occ;
    double x;
    while (is >> x) occ.push_back(x);
    QBX_REQUIRE((int)occ.size() == c.nst, 72, "density matrix size differs from the bands");
    c.occ = occ;
    h2d_sync(c.d_occ, c.occ.data(), sizeof(double) * c.nst);
    std::vector<double> w(c.nst);
    for (int n = 0; n < c.nst; n++) w[n] = c.occ[n] / c.wb.omega;
    h2d_sync(density_weights(c), w.data(), sizeof(double) * c.nst);
  }
  size_t p = 0;
  int n = 0;
  std::vector<double> f(N);
  while ((p = s.find("<grid_function", p)) != std::string::npos) {
    QBX_REQUIRE(n < c.nst, 72, "more grid functions than bands");
    const size_t he = s.find('>', p);
    QBX_REQUIRE(attr(s, p, he, "type") == "double", 73, "only real (Gamma) grid functions");
    QBX_REQUIRE(attr(s, p, he, "encoding") == "base64", 73, "only base64 grid functions");
    const size_t de = s.find("</grid_function>", he);
    QBX_REQUIRE(de != std::string::npos, 70, "unterminated grid_function");
    const std::vector<unsigned char> bytes = b64_decode(s.data() + he + 1, s.data() + de);
    QBX_REQUIRE(bytes.size() == N * sizeof(double), 74, "grid function of the wrong size");
    std::memcpy(f.data(), bytes.data(), bytes.size());
    QBX_CUDA(cudaMemcpyAsync(c.d_grad, f.data(), N * sizeof(double), cudaMemcpyHostToDevice,
                             c.stream));
    wfgrid_forward(c, d, ngw, c.d_grad, c.d_c + 2 * (size_t)n * ngw);
    QBX_CUDA(cudaStreamSynchronize(c.stream));
    p = de;
    n++;
  }
  QBX_REQUIRE(n == c.nst, 72, "fewer grid functions than bands");
  c.extrapolate = false;
}

}  // namespace qbx
