// Pointwise, G-space and reduction kernels of the electronic step.
//
// Everything here is memory-bound elementwise work in FP64: the exchange-
// correlation functionals on the real-space grid, the Hartree/local-potential
// algebra on the density sphere, kinetic energy and eigenvalue-sum
// reductions, the preconditioned steepest-descent update with Anderson
// extrapolation, and the per-geometry structure factors and projectors.
// Reductions are deterministic: fixed-size partial sums per CTA, then one CTA
// adds the partials in order.
#include <cmath>
#include <vector>

#include "qbx_internal.h"
#include "reduce.cuh"
#include "split.cuh"

namespace qbx {

using namespace red;

static int blocks_for(size_t n) {
  return (int)std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 32));
}

struct SumF {
  const double* x;
  __device__ void operator()(size_t i, double* a) const { a[0] += x[i]; }
};

void launch_sum(Context& ctx, const double* x, size_t n, int slot) {
  reduce<1>(ctx, SumF{x}, n, slot);
}

// ------------------------------------------------------------------- XC
// Perdew-Zunger LDA (src/LDAFunctional.cpp:92-150), unpolarized.
__device__ void lda_pz(double rh, double& ee, double& vv) {
  const double c1 = 0.6203504908994001, c3 = -0.610887057711;
  const double A = 0.0311, B = -0.048, b1 = 1.0529, b2 = 0.3334, G = -0.1423;
  const double D = G / (1.0 + b1 + b2) - B;
  const double C = -A - D - G * ((b1 / 2.0 + b2) / ((1.0 + b1 + b2) * (1.0 + b1 + b2)));
  ee = 0.0; vv = 0.0;
  if (rh > 0.0) {
    const double rs = c1 / cbrt(rh);
    const double vx = c3 / rs, ex = 0.75 * vx;
    double ec, vc;
    if (rs < 1.0) {
      const double lr = log(rs);
      ec = A * lr + B + C * rs * lr + D * rs;
      vc = A * lr + (B - A / 3.0) + (2.0 / 3.0) * C * rs * lr + ((2.0 * D - C) / 3.0) * rs;
    } else {
      const double sq = sqrt(rs), den = 1.0 + b1 * sq + b2 * rs;
      ec = G / den;
      vc = ec * (1.0 + (7.0 / 6.0) * b1 * sq + (4.0 / 3.0) * b2 * rs) / den;
    }
    ee = ex + ec;
    vv = vx + vc;
  }
}

// PBE (src/PBEFunctional.cpp:168-280; PW92 local correlation via gcor2).
__device__ void pbe(double rho, double grad, double& exc, double& v1, double& v2) {
  const double third = 1.0 / 3.0, third4 = 4.0 / 3.0;
  const double ax = -0.7385587663820224058, um = 0.2195149727645171, uk = 0.804;
  const double ul = um / uk, pi32third = 3.09366772628014, alpha = 1.91915829267751;
  const double seven_sixth = 7.0 / 6.0, four_over_pi = 1.27323954473516;
  const double gamma = 0.03109069086965489, bet = 0.06672455060314922;
  const double delt = bet / gamma;
  exc = 0.0; v1 = 0.0; v2 = 0.0;
  if (rho < 1.e-18) return;
  const double rh13 = pow(rho, third);
  const double exunif = ax * rh13;
  const double fk = pi32third * rh13;
  const double s = grad / (2.0 * fk * rho);
  const double s2 = s * s;
  const double p0 = 1.0 + ul * s2;
  const double fxpbe = 1.0 + uk - uk / p0;
  const double ex = exunif * fxpbe;
  const double fs = 2.0 * uk * ul / (p0 * p0);
  const double vx1 = third4 * exunif * (fxpbe - s2 * fs);
  const double vx2 = -exunif * fs / (rho * 4.0 * fk * fk);
  const double rs = alpha / fk;
  const double twoks = 2.0 * sqrt(four_over_pi * fk);
  const double t = grad / (twoks * rho);
  const double rtrs = sqrt(rs);
  const double a = 0.0310907, a1 = 0.2137, bb1 = 7.5957, bb2 = 3.5876, bb3 = 1.6382, bb4 = 0.49294;
  const double q0 = -2.0 * a * (1.0 + a1 * rtrs * rtrs);
  const double q1 = 2.0 * a * rtrs * (bb1 + rtrs * (bb2 + rtrs * (bb3 + rtrs * bb4)));
  const double q2 = log(1.0 + 1.0 / q1);
  const double ec = q0 * q2;
  const double q3 = a * (bb1 / rtrs + 2.0 * bb2 + rtrs * (3.0 * bb3 + 4.0 * bb4 * rtrs));
  const double ecrs = -2.0 * a * a1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
  const double vc = ec - rs * ecrs * third;
  const double pon = -ec / gamma;
  const double b = delt / (exp(pon) - 1.0);
  const double b2 = b * b, t2 = t * t, t4 = t2 * t2;
  const double q4 = 1.0 + b * t2;
  const double q5 = q4 + b2 * t4;
  const double h = gamma * log(1.0 + delt * q4 * t2 / q5);
  const double t6 = t4 * t2, rsthrd = rs * third;
  const double fac = delt / b + 1.0;
  const double bec = b2 * fac / bet;
  const double q8 = q5 * q5 + delt * q4 * q5 * t2;
  const double q9 = 1.0 + 2.0 * b * t2;
  const double hb = -bet * b * t6 * (2.0 + b * t2) / q8;
  const double hrs = -rsthrd * hb * bec * ecrs;
  const double ht = 2.0 * bet * q9 / q8;
  const double vc1 = vc + h + hrs - t2 * ht * seven_sixth;
  const double vc2 = -ht / (rho * twoks * twoks);
  exc = ex + ec + h;
  v1 = vx1 + vc1;
  v2 = vx2 + vc2;
}

__global__ void k_lda(const double* __restrict__ rho, size_t n, double* __restrict__ vxc,
                      double* __restrict__ erho) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double e, v;
    lda_pz(rho[i], e, v);
    vxc[i] = v;
    erho[i] = rho[i] * e;
  }
}

__global__ void k_pbe(const double* __restrict__ rho, const double* __restrict__ grad, size_t n,
                      double* __restrict__ v1, double* __restrict__ v2, double* __restrict__ erho) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double gx = grad[i], gy = grad[n + i], gz = grad[2 * n + i];
    const double g = sqrt(gx * gx + gy * gy + gz * gz);
    double e, a, b;
    pbe(rho[i], g, e, a, b);
    v1[i] = a;
    v2[i] = b;
    erho[i] = rho[i] * e;
  }
}

// out(G) = i gx_j(G) scale in(G)
__global__ void k_mul_igx(const double2* __restrict__ in, const double* __restrict__ gxj, int ng,
                          double scale, double2* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 v = in[i];
    const double g = gxj[i] * scale;
    out[i] = make_double2(-g * v.y, g * v.x);
  }
}

// out(G) = sum_j i gx_j(G) in_j(G)
__global__ void k_sum_igx3(const double2* __restrict__ a, const double2* __restrict__ b,
                           const double2* __restrict__ c, const double* __restrict__ gx, int ng,
                           double2* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double g0 = gx[i], g1 = gx[(size_t)ng + i], g2 = gx[2 * (size_t)ng + i];
    const double2 u = a[i], v = b[i], w = c[i];
    const double re = g0 * u.x + g1 * v.x + g2 * w.x, im = g0 * u.y + g1 * v.y + g2 * w.y;
    out[i] = make_double2(-im, re);
  }
}

__global__ void k_mul(const double* __restrict__ a, const double* __restrict__ b, size_t n,
                      double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = a[i] * b[i];
}

__global__ void k_axpy(double* __restrict__ y, const double* __restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] += x[i];
}

// sum_i x_i y_i
struct DotF {
  const double* x; const double* y;
  __device__ void operator()(size_t i, double* a) const { a[0] += x[i] * y[i]; }
};

// sum of the energy density and of rho * v1
struct SumRhoV1F {
  const double* e; const double* rho; const double* v1;
  __device__ void operator()(size_t i, double* a) const {
    a[0] += e[i];
    a[1] += rho[i] * v1[i];
  }
};

// XCPotential::update (src/XCPotential.cpp:124-465): vxc and E_xc.
void launch_xc(Context& ctx) {
  const size_t N = ctx.N();
  const double om = ctx.vb.omega;
  const int nb = blocks_for(N);
  if (ctx.xc == "LDA") {
    k_lda<<<nb, kThreads, 0, ctx.stream>>>(ctx.d_rhor, N, ctx.d_vxc, ctx.d_exc);
    QBX_LAUNCHED(ctx);
    launch_sum(ctx, ctx.d_exc, N, SLOT_EXC);
    reduce<1>(ctx, DotF{ctx.d_rhor, ctx.d_vxc}, N, SLOT_EXC + 2);   // for dxc
    return;
  }
  // PBE: grad rho as the backward transforms of i G_j rho(G)/Omega, two real
  // components packed into one complex transform
  const int ngv = ctx.vb.ng;
  double* xg[3] = {ctx.d_xc_g, ctx.d_xc_g + 2 * (size_t)ngv, ctx.d_xc_g + 4 * (size_t)ngv};
  for (int j = 0; j < 3; j++) {
    k_mul_igx<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(
        (const double2*)ctx.d_rhog, ctx.d_gx_v + (size_t)j * ngv, ngv, 1.0 / om,
        (double2*)xg[j]);
    QBX_LAUNCHED(ctx);
  }
  vb_backward_pair(ctx, xg[0], xg[1], ctx.d_grad, ctx.d_grad + N);
  vb_backward(ctx, xg[2], ctx.d_grad + 2 * N);
  k_pbe<<<nb, kThreads, 0, ctx.stream>>>(ctx.d_rhor, ctx.d_grad, N, ctx.d_vxc, ctx.d_vx2,
                                         ctx.d_exc);
  QBX_LAUNCHED(ctx);
  // sum e_xc and sum rho v1 (the latter for the XC stress)
  reduce<2>(ctx, SumRhoV1F{ctx.d_exc, ctx.d_rhor, ctx.d_vxc}, N, SLOT_EXC);
  // vxc += backward(sum_j i G_j forward(grad_j vxc2)): the forward transforms
  // two real fields to a complex one, the sum in G space before one backward
  vb_forward_real_pair(ctx, ctx.d_grad, ctx.d_grad + N, ctx.d_vx2, xg[0], xg[1]);
  vb_forward_real_pair(ctx, ctx.d_grad + 2 * N, nullptr, ctx.d_vx2, xg[2], nullptr);
  k_sum_igx3<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(
      (const double2*)xg[0], (const double2*)xg[1], (const double2*)xg[2], ctx.d_gx_v, ngv,
      (double2*)ctx.d_vtmp_g);
  QBX_LAUNCHED(ctx);
  vb_backward(ctx, ctx.d_vtmp_g, ctx.d_exc);
  k_axpy<<<nb, kThreads, 0, ctx.stream>>>(ctx.d_vxc, ctx.d_exc, N);
  QBX_LAUNCHED(ctx);
  reduce<1>(ctx, DotF{ctx.d_rhor, ctx.d_vxc}, N, SLOT_EXC + 2);   // for dxc
}

// ---------------------------------------------------- Hartree and local
struct EpsEhF {
  const double2* rhog; const double2* vion; const double2* rhops; const double* g2i;
  double om_inv;
  __device__ void operator()(size_t i, double* a) const {
    const double2 r = make_double2(rhog[i].x * om_inv, rhog[i].y * om_inv);
    const double2 v = vion[i];
    const double f = (i == 0) ? 1.0 : 2.0;     // G=0 counted once
    a[0] += f * (r.x * v.x + r.y * v.y);
    const double2 p = rhops[i];
    const double2 t = make_double2(r.x + p.x, r.y + p.y);
    const double gi = g2i[i];
    a[1] += (t.x * t.x + t.y * t.y) * gi;
    a[2] += (r.x * r.x + r.y * r.y) * gi;      // electrons alone
    a[3] += (p.x * p.x + p.y * p.y) * gi;      // pseudocharges alone
  }
};

__global__ void k_vlocal_g(const double2* __restrict__ rhog, const double2* __restrict__ vion,
                           const double2* __restrict__ rhops, const double* __restrict__ g2i,
                           int ng, double om_inv, double2* __restrict__ vloc,
                           double2* __restrict__ rhogt) {
  const double fpi = 4.0 * M_PI;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 t = make_double2(rhog[i].x * om_inv + rhops[i].x, rhog[i].y * om_inv + rhops[i].y);
    rhogt[i] = t;
    vloc[i] = make_double2(vion[i].x + fpi * t.x * g2i[i], vion[i].y + fpi * t.y * g2i[i]);
  }
}

// EnergyFunctional::update_vhxc (src/EnergyFunctional.cpp:231-394) minus XC
void launch_vhxc_gspace(Context& ctx) {
  const int ngv = ctx.vb.ng;
  const double om = ctx.vb.omega;
  reduce<4>(ctx, EpsEhF{(const double2*)ctx.d_rhog, (const double2*)ctx.d_vion,
                        (const double2*)ctx.d_rhops, ctx.d_g2i_v, 1.0 / om},
            (size_t)ngv, SLOT_EPS_EH);
  k_vlocal_g<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(
      (const double2*)ctx.d_rhog, (const double2*)ctx.d_vion, (const double2*)ctx.d_rhops,
      ctx.d_g2i_v, ngv, 1.0 / om, (double2*)ctx.d_vtmp_g, (double2*)ctx.d_vtmp_g2);
  QBX_LAUNCHED(ctx);
  vb_backward(ctx, ctx.d_vtmp_g, ctx.d_vr);
  k_axpy<<<blocks_for(ctx.N()), kThreads, 0, ctx.stream>>>(ctx.d_vr, ctx.d_vxc, ctx.N());
  QBX_LAUNCHED(ctx);
}

// ------------------------------------------------- wavefunction sums
struct EkinF {
  const double2* c; const double* g2; const double* occ; int ngw;
  __device__ void operator()(size_t i, double* a) const {
    const int n = (int)(i / ngw), ig = (int)(i - (size_t)n * ngw);
    const double2 v = c[i];
    a[0] += occ[n] * (v.x * v.x + v.y * v.y) * g2[ig];
  }
};

void launch_ekin(Context& ctx) {
  reduce<1>(ctx, EkinF{(const double2*)ctx.d_c, ctx.d_g2_w, ctx.d_occ, ctx.wb.ng},
            (size_t)ctx.wb.ng * ctx.nst, SLOT_EKIN);
}

struct EigF {
  const double2* c; const double2* hc; int ngw;
  __device__ void operator()(size_t i, double* a) const {
    const int n = (int)(i / ngw), ig = (int)(i - (size_t)n * ngw);
    const double2 x = c[i], y = hc[i];
    // 2 Re(conj(c) hc) on the half sphere, G=0 real part counted once
    a[0] += (ig == 0) ? (2.0 * x.y * y.y + x.x * y.x) : 2.0 * (x.x * y.x + x.y * y.y);
    (void)n;
  }
};

void launch_eigsum(Context& ctx) {
  reduce<1>(ctx, EigF{(const double2*)ctx.d_c, (const double2*)ctx.d_hc, ctx.wb.ng},
            (size_t)ctx.wb.ng * ctx.nst, SLOT_EIG);
}

// Preconditioner::update (src/Preconditioner.cpp:88-143): per-band kinetic
// energy ekin_n = (sum |c|^2 G^2) / (sum |c|^2 - |c_0|^2 / 2), one CTA per band.
__global__ void k_prec(const double2* __restrict__ c, const double* __restrict__ g2, int ngw,
                       double* __restrict__ ekin) {
  __shared__ double sh[32];
  const int n = blockIdx.x;
  const double2* p = c + (size_t)n * ngw;
  double sn = 0.0, se = 0.0;
  for (int ig = threadIdx.x; ig < ngw; ig += blockDim.x) {
    const double2 v = p[ig];
    const double psi2 = v.x * v.x + v.y * v.y;
    sn += psi2;
    se += psi2 * g2[ig];
  }
  const double tn = block_sum(sn, sh);
  const double te = block_sum(se, sh);
  if (threadIdx.x == 0) {
    const double c0 = p[0].x * p[0].x + p[0].y * p[0].y;
    const double bn = 2.0 * (tn - 0.5 * c0), be = 2.0 * te;
    double e = (0.5 * bn > 0.0) ? 0.5 * be / bn : 0.0;
    if (e == 0.0) e = 1.0;
    ekin[n] = e;
  }
}

void launch_precond_update(Context& ctx) {
  k_prec<<<ctx.nst, kThreads, 0, ctx.stream>>>((const double2*)ctx.d_c, ctx.d_g2_w, ctx.wb.ng,
                                               ctx.d_prec);
  QBX_LAUNCHED(ctx);
}

// dc = -K(G) r(G), K = 0.5/max(ekin_n, |G|^2/2) (Preconditioner::diag,
// src/Preconditioner.cpp:49-85); dc overwrites the residual in hc.
__global__ void k_precondition(double2* __restrict__ hc, const double* __restrict__ g2,
                               const double* __restrict__ ekin, int ngw, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / ngw), ig = (int)(i - (size_t)b * ngw);
    const double e = 0.5 * g2[ig];
    const double en = ekin[b];
    const double k = (e < en) ? 0.5 / en : 0.5 / e;
    const double2 r = hc[i];
    hc[i] = make_double2(-k * r.x, -k * r.y);
  }
}

// The Anderson sums of the preconditioned residual dc = -K r (formed as
// k_precondition forms it, not stored: the update forms it again from r):
// <dc, dc - dc_last> and |dc - dc_last|^2 (weight 2 off G = 0, the real view
// of the half sphere; src/PSDAWavefunctionStepper.cpp:129-179)
struct PrecondAndersonF {
  const double2* hc; const double2* fl; const double* g2; const double* ekin; int ngw;
  __device__ void operator()(size_t i, double* a) const {
    const int b = (int)(i / ngw), ig = (int)(i - (size_t)b * ngw);
    const double e = 0.5 * g2[ig];
    const double en = ekin[b];
    const double k = (e < en) ? 0.5 / en : 0.5 / e;
    const double2 r = hc[i];
    const double2 x = make_double2(-k * r.x, -k * r.y);
    const double2 y = fl[i];
    const double dx = x.x - y.x, dy = x.y - y.y;
    const double w = (ig == 0) ? 1.0 : 2.0;
    a[0] += w * (x.x * dx + x.y * dy);
    a[1] += w * (dx * dx + dy * dy);
  }
};

// theta = -<dc, dc - dc_last> / |dc - dc_last|^2 from the two sums, reset to
// 0 below -1 and capped at 2 (src/PSDAWavefunctionStepper.cpp:129-179)
__device__ __forceinline__ double anderson_theta(const double* ab) {
  double theta = ab[1] != 0.0 ? -ab[0] / ab[1] : 0.0;
  if (theta < -1.0) theta = 0.0;
  return fmin(2.0, theta);
}

// The step, one band per grid row: dc = -K r from the residual r (hc), then
// c <- c + theta (c - c_last) + dc + theta (dc - dc_last), and the last c and
// dc kept for the next step.
__global__ void k_psda_update(double2* __restrict__ c, double2* __restrict__ c_last,
                              double2* __restrict__ dc_last, const double2* __restrict__ r,
                              const double* __restrict__ g2, const double* __restrict__ ekin,
                              int ngw, const double* __restrict__ ab, int extrapolate,
                              double* __restrict__ theta_out) {
  const double theta = extrapolate ? anderson_theta(ab) : 0.0;
  const int b = blockIdx.y;
  if (b == 0 && blockIdx.x == 0 && threadIdx.x == 0) *theta_out = theta;
  const double en = ekin[b];
  const size_t off = (size_t)b * ngw;
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ngw; ig += gridDim.x * blockDim.x) {
    const size_t i = off + ig;
    const double e = 0.5 * g2[ig];
    const double k = (e < en) ? 0.5 / en : 0.5 / e;
    const double2 rv = r[i];
    const double2 x = c[i], f = make_double2(-k * rv.x, -k * rv.y);
    double2 nc;
    if (extrapolate) {
      const double2 xl = c_last[i], fl = dc_last[i];
      nc.x = x.x + theta * (x.x - xl.x) + f.x + theta * (f.x - fl.x);
      nc.y = x.y + theta * (x.y - xl.y) + f.y + theta * (f.y - fl.y);
    } else {
      nc.x = x.x + f.x;
      nc.y = x.y + f.y;
    }
    c[i] = nc;
    c_last[i] = x;
    dc_last[i] = f;
  }
}

// k_psda_update with the splits of the new C that ortho_align reads written
// in the same pass: SlaterDet::cleanup (Im c(G=0) = 0, src/SlaterDet.cpp:
// 1341-1356) applied to the new C, then its BF16 hi/lo (ld ldb, padding rows
// zero) and TF32 hi/lo (ld ldt) splits, and per band the partial sums of its
// squares for the overlap's diagonal (part[band * gridDim.x + blockIdx.x],
// gridDim.x as the split kernel's grid, which overlap_diag_from_split
// expects).  One coefficient (two rows) a thread, one band per grid row;
// rows = 2 ngw, all four FP64 blocks have ld rows.
__global__ void __launch_bounds__(256)
k_psda_update_split(double* __restrict__ c, double* __restrict__ c_last,
                    double* __restrict__ dc_last, const double* __restrict__ r,
                    const double* __restrict__ g2, const double* __restrict__ ekin, int rows,
                    const double* __restrict__ ab, int extrapolate, double* __restrict__ theta_out,
                    __nv_bfloat16* __restrict__ bhi, __nv_bfloat16* __restrict__ blo, int ldb,
                    float* __restrict__ thi, float* __restrict__ tlo, int ldt,
                    double* __restrict__ part) {
  const double theta = extrapolate ? anderson_theta(ab) : 0.0;
  const int b = blockIdx.y;
  if (b == 0 && blockIdx.x == 0 && threadIdx.x == 0) *theta_out = theta;
  const double en = ekin[b];
  const int ngw = rows >> 1, half = ldb >> 1;
  double acc = 0.0;
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < half;
       ig += gridDim.x * blockDim.x) {
    double2 nc = make_double2(0.0, 0.0);   // the padding rows split to zero
    if (ig < ngw) {
      const size_t i = (size_t)b * ngw + ig;   // in double2 units
      const double e = 0.5 * g2[ig];
      const double k = (e < en) ? 0.5 / en : 0.5 / e;
      const double2 rv = reinterpret_cast<const double2*>(r)[i];
      const double2 x = reinterpret_cast<const double2*>(c)[i];
      const double2 f = make_double2(-k * rv.x, -k * rv.y);
      if (extrapolate) {
        const double2 xl = reinterpret_cast<const double2*>(c_last)[i];
        const double2 fl = reinterpret_cast<const double2*>(dc_last)[i];
        nc.x = x.x + theta * (x.x - xl.x) + f.x + theta * (f.x - fl.x);
        nc.y = x.y + theta * (x.y - xl.y) + f.y + theta * (f.y - fl.y);
      } else {
        nc.x = x.x + f.x;
        nc.y = x.y + f.y;
      }
      if (ig == 0) nc.y = 0.0;
      reinterpret_cast<double2*>(c)[i] = nc;
      reinterpret_cast<double2*>(c_last)[i] = x;
      reinterpret_cast<double2*>(dc_last)[i] = f;
      acc += nc.x * nc.x + nc.y * nc.y;
      float2 th, tl;
      split_tf32(nc.x, th.x, tl.x);
      split_tf32(nc.y, th.y, tl.y);
      *reinterpret_cast<float2*>(thi + (size_t)b * ldt + 2 * ig) = th;
      *reinterpret_cast<float2*>(tlo + (size_t)b * ldt + 2 * ig) = tl;
    }
    __nv_bfloat162 bh, bl;
    split_bf16(nc.x, bh.x, bl.x);
    split_bf16(nc.y, bh.y, bl.y);
    *reinterpret_cast<__nv_bfloat162*>(bhi + (size_t)b * ldb + 2 * ig) = bh;
    *reinterpret_cast<__nv_bfloat162*>(blo + (size_t)b * ldb + 2 * ig) = bl;
  }
  __shared__ double sh[32];
  const double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = t;
}

// PSDAWavefunctionStepper::update after the residual (src/PSDAWavefunction
// Stepper.cpp:82-212): precondition, Anderson theta, step.  With split_c
// (the mixed path where ortho_align reads C's BF16 and TF32 splits) the step
// also cleans up the new C and writes those splits and the column partials
// (cs_hi/lo[1], ct_hi/lo, d_colred), as split_bf16_tf32 would.
void launch_psda_elementwise(Context& ctx, bool split_c) {
  const size_t n = (size_t)ctx.wb.ng * ctx.nst;
  if (ctx.extrapolate)
    reduce<2>(ctx, PrecondAndersonF{(const double2*)ctx.d_hc, (const double2*)ctx.d_dc_last,
                                    ctx.d_g2_w, ctx.d_prec, ctx.wb.ng},
              n, SLOT_ANDERSON);
  // theta is formed on the device from the two sums; the residual stays in hc
  const int ngw = ctx.wb.ng;
  if (split_c) {
    const int ldp = ctx.ldp, nst = ctx.nst;
    const int nb = split_blocks_per_column(ldp);   // the partials overlap_diag_from_split adds
    QBX_REQUIRE(ldp % 4 == 0 && ldp >= 2 * ngw && nst <= 65535 &&
                    (size_t)nb * nst <= ctx.colred_elems && ctx.cs_hi[1] && ctx.ct_hi,
                50, "PSDA step with the splits of C: no split buffers or partials");
    k_psda_update_split<<<dim3((unsigned)nb, (unsigned)nst), 256, 0, ctx.stream>>>(
        ctx.d_c, ctx.d_c_last, ctx.d_dc_last, ctx.d_hc, ctx.d_g2_w, ctx.d_prec, 2 * ngw,
        ctx.d_scalars + SLOT_ANDERSON, ctx.extrapolate ? 1 : 0, ctx.d_scalars + SLOT_THETA,
        (__nv_bfloat16*)ctx.cs_hi[1], (__nv_bfloat16*)ctx.cs_lo[1], ldp, (float*)ctx.ct_hi,
        (float*)ctx.ct_lo, ldp, ctx.d_colred);
    QBX_LAUNCHED(ctx);
    return;
  }
  dim3 grid((unsigned)std::max(1, std::min((ngw + kThreads - 1) / kThreads, 16)),
            (unsigned)ctx.nst);
  k_psda_update<<<grid, kThreads, 0, ctx.stream>>>(
      (double2*)ctx.d_c, (double2*)ctx.d_c_last, (double2*)ctx.d_dc_last,
      (const double2*)ctx.d_hc, ctx.d_g2_w, ctx.d_prec, ngw, ctx.d_scalars + SLOT_ANDERSON,
      ctx.extrapolate ? 1 : 0, ctx.d_scalars + SLOT_THETA);
  QBX_LAUNCHED(ctx);
}

// JD correction: Z = -K R, R the residual held in hc (Preconditioner::diag)
void launch_precondition_into(Context& ctx, const double* r, double* z) {
  const size_t n = (size_t)ctx.wb.ng * ctx.nst;
  QBX_CUDA(cudaMemcpyAsync(z, r, 2 * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
  k_precondition<<<blocks_for(n), kThreads, 0, ctx.stream>>>((double2*)z, ctx.d_g2_w, ctx.d_prec,
                                                              ctx.wb.ng, n);
  QBX_LAUNCHED(ctx);
}

__global__ void k_cleanup(double2* c, int ngw, int nst) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < nst) c[(size_t)n * ngw].y = 0.0;
}

// SlaterDet::cleanup (src/SlaterDet.cpp:1341-1356): Im c(G=0) = 0
void launch_cleanup(Context& ctx, double* c) {
  k_cleanup<<<(ctx.nst + 255) / 256, 256, 0, ctx.stream>>>((double2*)c, ctx.wb.ng, ctx.nst);
  QBX_LAUNCHED(ctx);
}

// m(i,j) += alpha x_i y_j  (column-major, ld ldm)
__global__ void k_rank1(double* m, int ldm, const double* x, int ldx, const double* y, int ldy,
                        int nrow, int ncol, double alpha, int lower_only) {
  const size_t n = (size_t)nrow * ncol;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nrow), j = (int)(t / nrow);
    if (lower_only && i < j) continue;
    m[i + (size_t)j * ldm] += alpha * x[(size_t)i * ldx] * y[(size_t)j * ldy];
  }
}

void launch_rank1_fix(Context& ctx, double* m, int ldm, const double* x, int ldx,
                      const double* y, int ldy, int nrow, int ncol, double alpha,
                      bool lower_only) {
  k_rank1<<<blocks_for((size_t)nrow * ncol), kThreads, 0, ctx.stream>>>(
      m, ldm, x, ldx, y, ldy, nrow, ncol, alpha, lower_only ? 1 : 0);
  QBX_LAUNCHED(ctx);
}

// ------------------------------------------------------------ nonlocal
struct EnlF {
  double* f; const double* dfac; const double* occ; int np; double om_inv;
  __device__ void operator()(size_t i, double* a) const {
    const int p = (int)(i % np), n = (int)(i / np);
    const double F = f[i];
    const double DF = dfac[p] * F;
    a[0] += occ[n] * F * DF * om_inv;
  }
};

__global__ void k_fnl_scale(double* f, const double* dfac, int np, size_t n, double om_inv) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    f[i] *= dfac[i % np] * om_inv;
}

// E_nl and fnl <- D F / Omega (src/NonLocalPotential.cpp:1469-1597)
void launch_enl(Context& ctx) {
  const size_t n = (size_t)ctx.nproj * ctx.nst;
  reduce<1>(ctx, EnlF{ctx.d_fnl, ctx.d_pdfac, ctx.d_occ, ctx.nproj, 1.0 / ctx.wb.omega}, n,
            SLOT_ENL);
  k_fnl_scale<<<blocks_for(n), kThreads, 0, ctx.stream>>>(ctx.d_fnl, ctx.d_pdfac, ctx.nproj, n,
                                                          1.0 / ctx.wb.omega);
  QBX_LAUNCHED(ctx);
}

// c'(G) = G_j (i c(G)) for the force projections dF_j = 2 A^T c'
__global__ void k_igj_c(const double2* __restrict__ c, const double* __restrict__ gxj, int ngw,
                        size_t n, double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double g = gxj[i % ngw];
    const double2 v = c[i];
    out[i] = make_double2(-g * v.y, g * v.x);
  }
}

// fion[atom, j] -= 2 sum_n occ_n fnl(p,n) dF(p,n) over the atom's projectors
__global__ void k_nl_force(const double* __restrict__ fnl, const double* __restrict__ dfnl,
                           const double* __restrict__ occ, const int* __restrict__ patom, int np,
                           int nst, int j, double* __restrict__ fion) {
  __shared__ double sh[32];
  const int p = blockIdx.x;
  double s = 0.0;
  for (int n = threadIdx.x; n < nst; n += blockDim.x)
    s += occ[n] * fnl[p + (size_t)n * np] * dfnl[p + (size_t)n * np];
  const double t = block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(&fion[3 * patom[p] + j], -2.0 * t);
}

void launch_nl_forces(Context& ctx, double* fion) {
  const int ngw = ctx.wb.ng;
  const size_t n = (size_t)ngw * ctx.nst;
  const double two = 2.0, zero = 0.0;
  for (int j = 0; j < 3; j++) {
    k_igj_c<<<blocks_for(n), kThreads, 0, ctx.stream>>>((const double2*)ctx.d_c,
                                                        ctx.d_gx_w + (size_t)j * ngw, ngw, n,
                                                        (double2*)ctx.d_ctmp);
    QBX_LAUNCHED(ctx);
    if (ctx.precision == MIXED) {
      // dF_j = 2 A^T (i G_j C) as three BF16 split products (the split of
      // H*C is free here: the step splits H*C again after the forces)
      const int K = 2 * ngw;
      split_bf16_2d(ctx, ctx.d_ctmp, K, ctx.nst, K, ctx.hs_hi, ctx.hs_lo, ctx.ldp);
      split_gemm(ctx, true, false, ctx.nproj, ctx.nst, K, 2.0, ctx.as_hi, ctx.as_lo, ctx.ldp,
                 ctx.hs_hi, ctx.hs_lo, ctx.ldp, 0.0, ctx.d_dfnl);
    } else {
      QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, ctx.nproj, ctx.nst, 2 * ngw, &two,
                           ctx.d_anl, 2 * ngw, ctx.d_ctmp, 2 * ngw, &zero, ctx.d_dfnl,
                           ctx.nproj));
    }
    k_nl_force<<<ctx.nproj, kThreads, 0, ctx.stream>>>(ctx.d_fnl, ctx.d_dfnl, ctx.d_occ,
                                                       ctx.d_patom, ctx.nproj, ctx.nst, j, fion);
    QBX_LAUNCHED(ctx);
  }
}

// Cell and reciprocal vectors (rows) for the phase tables of the kernels
// below.
struct CellRows {
  double a[9];
  double b[9];
};

// exp(-i G.tau) for the density-basis vector (x, y, z) from three tables of
// exp(-i 2 pi h u_j) (u_j = tau.b_j / 2 pi the fractional coordinates, h the
// Miller index G.a_j / 2 pi), as the reference's StructureFactor builds its
// phases (src/StructureFactor.cpp:95-151): two complex products per vector
// instead of a sine and cosine.  Indices outside the tables fall back to
// sincos.
__device__ __forceinline__ double2 phase_from_tables(const double2* tab, int hmax,
                                                     const CellRows& cr, double x, double y,
                                                     double z, double tx, double ty, double tz) {
  const double inv2pi = 0.15915494309189533577;
  const int W = 2 * hmax + 1;
  const int h0 = __double2int_rn((x * cr.a[0] + y * cr.a[1] + z * cr.a[2]) * inv2pi);
  const int h1 = __double2int_rn((x * cr.a[3] + y * cr.a[4] + z * cr.a[5]) * inv2pi);
  const int h2 = __double2int_rn((x * cr.a[6] + y * cr.a[7] + z * cr.a[8]) * inv2pi);
  if (abs(h0) > hmax || abs(h1) > hmax || abs(h2) > hmax) {
    double sn, cs;
    sincos(x * tx + y * ty + z * tz, &sn, &cs);
    return make_double2(cs, -sn);
  }
  const double2 p = tab[h0 + hmax], q = tab[W + h1 + hmax], r = tab[2 * W + h2 + hmax];
  const double2 pq = make_double2(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x);
  return make_double2(pq.x * r.x - pq.y * r.y, pq.x * r.y + pq.y * r.x);
}

// the three tables of one atom: tab[j W + h + hmax] = exp(-i 2 pi h u_j)
__device__ __forceinline__ void phase_tables(double2* tab, int hmax, const CellRows& cr,
                                             double tx, double ty, double tz) {
  const int W = 2 * hmax + 1;
  for (int t = threadIdx.x; t < 3 * W; t += blockDim.x) {
    const int j = t / W, h = t - j * W - hmax;
    const double u2 = (tx * cr.b[3 * j] + ty * cr.b[3 * j + 1] + tz * cr.b[3 * j + 2]) *
                      0.31830988618379067154;   // 2 u = tau.b_j / pi
    double sn, cs;
    sincospi((double)h * u2, &sn, &cs);
    tab[t] = make_double2(cs, -sn);
  }
}

// Forces of the local pseudopotential and the Hartree term of the Gaussian
// pseudocharges (src/EnergyFunctional.cpp:841-930), one CTA per atom, its
// phases from the atom's tables in shared memory.
__global__ void k_local_force(const double* __restrict__ gx, const double2* __restrict__ rhogt,
                              const double2* __restrict__ rhog, const double* __restrict__ vps,
                              const double* __restrict__ rhops, const double* __restrict__ g2i,
                              int ng, double om_inv, const double* __restrict__ tau, double fac,
                              int atom0, double* __restrict__ fion, CellRows cr, int hmax) {
  __shared__ double sh[32];
  extern __shared__ double2 tab[];   // 3 (2 hmax + 1)
  const int ia = blockIdx.x;
  const double tx = tau[3 * ia], ty = tau[3 * ia + 1], tz = tau[3 * ia + 2];
  phase_tables(tab, hmax, cr, tx, ty, tz);
  __syncthreads();
  const double fpi = 4.0 * M_PI;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < ng; i += blockDim.x) {
    const double x = gx[i], y = gx[ng + i], z = gx[2 * ng + i];
    const double2 rt = rhogt[i];
    const double2 re = make_double2(rhog[i].x * om_inv, rhog[i].y * om_inv);
    const double t = fpi * rhops[i] * g2i[i];
    // vtemp = t conj(rhogt) + vps conj(rhoelg)
    const double vr = t * rt.x + vps[i] * re.x;
    const double vi = -t * rt.y - vps[i] * re.y;
    const double2 ph = phase_from_tables(tab, hmax, cr, x, y, z, tx, ty, tz);
    const double cs = ph.x, sn = -ph.y;
    // exp(-i G.tau) = cs - i sn
    const double tmp = cs * vi + (-sn) * vr;
    s0 += tmp * x; s1 += tmp * y; s2 += tmp * z;
  }
  const double a0 = block_sum(s0, sh);
  const double a1 = block_sum(s1, sh);
  const double a2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    fion[3 * (atom0 + ia)] += fac * a0;
    fion[3 * (atom0 + ia) + 1] += fac * a1;
    fion[3 * (atom0 + ia) + 2] += fac * a2;
  }
}

// The same forces for kLfAtoms atoms per CTA and one slice of the G vectors
// per grid row: the per-G factors are formed once for the CTA's atoms, and
// the slices' partial sums go to part[(atom 3 + j) nslice + slice], added in
// order by k_local_force_finish.
constexpr int kLfAtoms = 8;
__global__ void __launch_bounds__(256)
k_local_force_multi(const double* __restrict__ gx, const double2* __restrict__ rhogt,
                    const double2* __restrict__ rhog, const double* __restrict__ vps,
                    const double* __restrict__ rhops, const double* __restrict__ g2i, int ng,
                    double om_inv, const double* __restrict__ tau, int na, CellRows cr, int hmax,
                    double* __restrict__ part) {
  __shared__ double sh[32];
  extern __shared__ double2 tabs[];   // kLfAtoms x 3 (2 hmax + 1)
  const int W3 = 3 * (2 * hmax + 1);
  const int a0 = blockIdx.x * kLfAtoms, nat = min(kLfAtoms, na - a0);
  for (int a = 0; a < nat; a++)
    phase_tables(tabs + (size_t)a * W3, hmax, cr, tau[3 * (a0 + a)], tau[3 * (a0 + a) + 1],
                 tau[3 * (a0 + a) + 2]);
  __syncthreads();
  const int nslice = gridDim.y;
  const int per = (ng + nslice - 1) / nslice;
  const int g0 = blockIdx.y * per, g1 = min(ng, g0 + per);
  const double fpi = 4.0 * M_PI;
  double s[kLfAtoms][3];
#pragma unroll
  for (int a = 0; a < kLfAtoms; a++) s[a][0] = s[a][1] = s[a][2] = 0.0;
  for (int i = g0 + threadIdx.x; i < g1; i += blockDim.x) {
    const double x = gx[i], y = gx[ng + i], z = gx[2 * ng + i];
    const double2 rt = rhogt[i];
    const double2 re = make_double2(rhog[i].x * om_inv, rhog[i].y * om_inv);
    const double t = fpi * rhops[i] * g2i[i];
    const double vr = t * rt.x + vps[i] * re.x;
    const double vi = -t * rt.y - vps[i] * re.y;
#pragma unroll
    for (int a = 0; a < kLfAtoms; a++) {
      if (a < nat) {
        const int ia = a0 + a;
        const double2 ph = phase_from_tables(tabs + (size_t)a * W3, hmax, cr, x, y, z, tau[3 * ia],
                                             tau[3 * ia + 1], tau[3 * ia + 2]);
        // exp(-i G.tau) = ph.x + i ph.y = cs - i sn
        const double tmp = ph.x * vi + ph.y * vr;
        s[a][0] += tmp * x;
        s[a][1] += tmp * y;
        s[a][2] += tmp * z;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < kLfAtoms; a++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double v = block_sum(s[a][j], sh);
      if (threadIdx.x == 0 && a < nat) part[((size_t)(a0 + a) * 3 + j) * nslice + blockIdx.y] = v;
    }
}

__global__ void k_local_force_finish(const double* __restrict__ part, int na, int nslice,
                                     double fac, int atom0, double* __restrict__ fion) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * na) return;
  double t = 0.0;
  for (int sl = 0; sl < nslice; sl++) t += part[(size_t)k * nslice + sl];
  fion[3 * (size_t)atom0 + k] += fac * t;
}

static CellRows cell_rows(const Context& ctx) {
  CellRows cr;
  for (int i = 0; i < 9; i++) {
    cr.a[i] = ctx.vb.cell[i];
    cr.b[i] = ctx.vb.recip[i];
  }
  return cr;
}
// largest Miller index of the density grid
static int phase_hmax(const Context& ctx) {
  return std::max(ctx.vb.n0, std::max(ctx.vb.n1, ctx.vb.n2)) / 2 + 1;
}
static size_t phase_table_bytes(const Context& ctx) {
  return sizeof(double2) * 3 * (2 * (size_t)phase_hmax(ctx) + 1);
}

void launch_local_forces(Context& ctx, double* fion) {
  const int ngv = ctx.vb.ng;
  int atom0 = 0;
  for (size_t is = 0; is < ctx.species.size(); is++) {
    const int na = (int)ctx.tau[is].size() / 3;
    if (na == 0) continue;
    // positions of this species: a slice of the species-major d_tau_all
    constexpr int kSlices = 16;
    if ((size_t)na * 3 * kSlices <= ctx.fpart_elems) {
      const size_t sm = kLfAtoms * phase_table_bytes(ctx);
      allow_smem(k_local_force_multi, sm);
      dim3 grid((na + kLfAtoms - 1) / kLfAtoms, kSlices);
      k_local_force_multi<<<grid, kThreads, sm, ctx.stream>>>(
          ctx.d_gx_v, (const double2*)ctx.d_vtmp_g2, (const double2*)ctx.d_rhog,
          ctx.d_vps + is * (size_t)ngv, ctx.d_rhops_sp + is * (size_t)ngv, ctx.d_g2i_v, ngv,
          1.0 / ctx.vb.omega, ctx.d_tau_all + 3 * (size_t)atom0, na, cell_rows(ctx),
          phase_hmax(ctx), ctx.d_fpart);
      QBX_LAUNCHED(ctx);
      k_local_force_finish<<<(3 * na + 127) / 128, 128, 0, ctx.stream>>>(
          ctx.d_fpart, na, kSlices, -2.0 * ctx.vb.omega, atom0, fion);
    } else {
      k_local_force<<<na, kThreads, phase_table_bytes(ctx), ctx.stream>>>(
          ctx.d_gx_v, (const double2*)ctx.d_vtmp_g2, (const double2*)ctx.d_rhog,
          ctx.d_vps + is * (size_t)ngv, ctx.d_rhops_sp + is * (size_t)ngv, ctx.d_g2i_v, ngv,
          1.0 / ctx.vb.omega, ctx.d_tau_all + 3 * (size_t)atom0, -2.0 * ctx.vb.omega, atom0,
          fion, cell_rows(ctx), phase_hmax(ctx));
    }
    QBX_LAUNCHED(ctx);
    atom0 += na;
  }
}

// ---------------------------------------------------- small n x n helpers
__global__ void k_identity_axpy(double* t, const double* q, int n, double alpha) {
  const size_t nn = (size_t)n * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % n), c = (int)(i / n);
    t[i] = (r == c ? 1.0 : 0.0) + (alpha != 0.0 ? alpha * q[i] : 0.0);
  }
}
void launch_identity_axpy(Context& ctx, double* t, const double* q, int n, double alpha) {
  k_identity_axpy<<<blocks_for((size_t)n * n), kThreads, 0, ctx.stream>>>(t, q, n, alpha);
  QBX_LAUNCHED(ctx);
}

__global__ void k_symmetrize_lower(double* q, int n) {
  const size_t nn = (size_t)n * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % n), c = (int)(i / n);
    if (r < c) q[i] = q[c + (size_t)r * n];
  }
}
void launch_symmetrize_lower(Context& ctx, double* q, int n) {
  k_symmetrize_lower<<<blocks_for((size_t)n * n), kThreads, 0, ctx.stream>>>(q, n);
  QBX_LAUNCHED(ctx);
}

__global__ void k_avg(double* x, const double* t, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = 0.5 * (x[i] + t[i]);
}
void launch_avg_transpose(Context& ctx, double* x, const double* t, int n) {
  k_avg<<<blocks_for((size_t)n * n), kThreads, 0, ctx.stream>>>(x, t, (size_t)n * n);
  QBX_LAUNCHED(ctx);
}

struct Sq {
  const double* q;
  __device__ void operator()(size_t i, double* a) const { a[0] += q[i] * q[i]; }
};
void launch_frob2(Context& ctx, const double* q, int n) {
  reduce<1>(ctx, Sq{q}, (size_t)n * n, SLOT_FROB);
}

void launch_sumsq(Context& ctx, const double* x, size_t len, int slot) {
  reduce<1>(ctx, Sq{x}, len, slot);
}

// ------------------------------------------------------ per-geometry setup
// S(G) = sum_a exp(-i G.tau_a) on the density sphere
__global__ void k_sfac(const double* __restrict__ gx, int ng, const double* __restrict__ tau,
                       int na, double2* __restrict__ s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double x = gx[i], y = gx[ng + i], z = gx[2 * ng + i];
    double re = 0.0, im = 0.0;
    for (int a = 0; a < na; a++) {
      double sn, cs;
      sincos(x * tau[3 * a] + y * tau[3 * a + 1] + z * tau[3 * a + 2], &sn, &cs);
      re += cs;
      im -= sn;
    }
    s[i] = make_double2(re, im);
  }
}

// the phase tables of every atom of a species, tab[a 3W + j W + h + hmax]
__global__ void k_phase_tables(const double* __restrict__ tau, CellRows cr, int hmax,
                               double2* __restrict__ tab) {
  const int a = blockIdx.x;
  phase_tables(tab + (size_t)a * 3 * (2 * hmax + 1), hmax, cr, tau[3 * a], tau[3 * a + 1],
               tau[3 * a + 2]);
}

// S(G) = sum_a exp(-i G.tau_a) from the atoms' phase tables
__global__ void k_sfac_tab(const double* __restrict__ gx, int ng, const double* __restrict__ tau,
                           int na, const double2* __restrict__ tab, CellRows cr, int hmax,
                           double2* __restrict__ s) {
  const int W3 = 3 * (2 * hmax + 1);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double x = gx[i], y = gx[ng + i], z = gx[2 * ng + i];
    double re = 0.0, im = 0.0;
    for (int a = 0; a < na; a++) {
      const double2 ph = phase_from_tables(tab + (size_t)a * W3, hmax, cr, x, y, z, tau[3 * a],
                                           tau[3 * a + 1], tau[3 * a + 2]);
      re += ph.x;
      im += ph.y;
    }
    s[i] = make_double2(re, im);
  }
}

__global__ void k_vion(const double2* __restrict__ s, const double* __restrict__ vps,
                       const double* __restrict__ rhops, int ng, double2* __restrict__ vion,
                       double2* __restrict__ rhopst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    const double2 v = s[i];
    vion[i].x += v.x * vps[i];
    vion[i].y += v.y * vps[i];
    rhopst[i].x += v.x * rhops[i];
    rhopst[i].y += v.y * rhops[i];
  }
}

// anl(G) = twnl(G) (-i)^l exp(-i G.tau) for one projector column per atom
__global__ void k_anl(const double* __restrict__ gx, int ngw, const double* __restrict__ twnl,
                      const double* __restrict__ tau, int na, int l, double2* __restrict__ anl) {
  const int ia = blockIdx.y;
  const double tx = tau[3 * ia], ty = tau[3 * ia + 1], tz = tau[3 * ia + 2];
  double2* out = anl + (size_t)ia * ngw;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngw; i += gridDim.x * blockDim.x) {
    double sn, cs;
    sincos(gx[i] * tx + gx[ngw + i] * ty + gx[2 * ngw + i] * tz, &sn, &cs);
    const double t = twnl[i];
    // exp(-i G.tau) = (cs, -sn); times -i for l = 1: (-sn, -cs)
    out[i] = (l == 0) ? make_double2(t * cs, -t * sn) : make_double2(-t * sn, -t * cs);
  }
}

// Projector forms twnl = Y_lm(q) V_nl(|q|) (spline of the radial form) on
// the vectors q of basis b (G, or k+G for a complex basis), one row of ngw
// per (species, projector, m) (NonLocalPotential::update_twnl,
// src/NonLocalPotential.cpp:235-560, with the basis's kpg, kpgi, kpgx).
std::vector<double> twnl_rows(const Context& ctx, const Basis& b) {
  const double s14pi = std::sqrt(1.0 / (4.0 * M_PI));
  const double s34pi = std::sqrt(3.0 / (4.0 * M_PI));
  const int ngw = b.ng;
  std::vector<double> tw;
  for (const SpeciesTables& sp : ctx.species) {
    for (size_t iop = 0; iop < sp.proj_l.size(); iop++) {
      const int l = sp.proj_l[iop];
      std::vector<double> v(ngw);
      for (int ig = 0; ig < ngw; ig++) {
        double val, dv;
        sp.dvnlg((int)iop, b.g[ig], val, dv);
        v[ig] = val;
      }
      for (int m = 0; m < 2 * l + 1; m++)
        for (int ig = 0; ig < ngw; ig++)
          tw.push_back(l == 0 ? s14pi * v[ig]
                              : s34pi * b.gx[(size_t)m * ngw + ig] * b.gi[ig] * v[ig]);
    }
  }
  return tw;
}

// The projector columns anl = twnl (-i)^l exp(-i q.tau) of every atom on the
// ngw vectors q (device, x, y and z blocks), column order (species,
// projector, m, atom) as ctx.nproj counts them.
void build_anl(Context& ctx, const double* d_q, int ngw, const double* d_twnl, double* d_anl) {
  int col = 0, row = 0, atom0 = 0;
  for (size_t is = 0; is < ctx.species.size(); is++) {
    const SpeciesTables& sp = ctx.species[is];
    const int na = (int)ctx.tau[is].size() / 3;
    const double* d_tau = ctx.d_tau_all + 3 * (size_t)atom0;
    for (size_t iop = 0; iop < sp.proj_l.size(); iop++) {
      const int l = sp.proj_l[iop];
      for (int m = 0; m < 2 * l + 1; m++, row++) {
        dim3 grid((ngw + kThreads - 1) / kThreads, na);
        k_anl<<<grid, kThreads, 0, ctx.stream>>>(d_q, ngw, d_twnl + (size_t)row * ngw, d_tau,
                                                  na, l, (double2*)d_anl + (size_t)col * ngw);
        QBX_LAUNCHED(ctx);
        col += na;
      }
    }
    atom0 += na;
  }
  QBX_REQUIRE(col == ctx.nproj, 30, "projector count mismatch");
}

void launch_setup_atoms(Context& ctx) {
  const Basis& vb = ctx.vb;
  const int ngv = vb.ng, ngw = ctx.wb.ng;
  const int nsp = (int)ctx.species.size();
  // the projector forms do not depend on the positions: built once per set
  // of atoms
  if (!ctx.d_twnl) {
    const std::vector<double> tw = twnl_rows(ctx, ctx.wb);
    ctx.d_twnl = tw.empty() ? nullptr : dupload(tw);
  }
  QBX_CUDA(cudaMemsetAsync(ctx.d_vion, 0, 2 * sizeof(double) * ngv, ctx.stream));
  QBX_CUDA(cudaMemsetAsync(ctx.d_rhops, 0, 2 * sizeof(double) * ngv, ctx.stream));
  int atom0 = 0;
  for (int is = 0; is < nsp; is++) {
    const int na = (int)ctx.tau[is].size() / 3;
    // positions of this species: a slice of the species-major d_tau_all
    const double* d_tau = ctx.d_tau_all + 3 * (size_t)atom0;
    double2* sf = (double2*)ctx.d_sfac + (size_t)is * ngv;
    if ((size_t)na * phase_table_bytes(ctx) <= ctx.phase_tab_bytes) {
      k_phase_tables<<<na, 128, 0, ctx.stream>>>(d_tau, cell_rows(ctx), phase_hmax(ctx),
                                                (double2*)ctx.d_phase_tab);
      QBX_LAUNCHED(ctx);
      k_sfac_tab<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(
          ctx.d_gx_v, ngv, d_tau, na, (const double2*)ctx.d_phase_tab, cell_rows(ctx),
          phase_hmax(ctx), sf);
    } else {
      k_sfac<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(ctx.d_gx_v, ngv, d_tau, na, sf);
    }
    QBX_LAUNCHED(ctx);
    k_vion<<<blocks_for(ngv), kThreads, 0, ctx.stream>>>(sf, ctx.d_vps + (size_t)is * ngv,
                                                         ctx.d_rhops_sp + (size_t)is * ngv, ngv,
                                                         (double2*)ctx.d_vion,
                                                         (double2*)ctx.d_rhops);
    QBX_LAUNCHED(ctx);
    atom0 += na;
  }
  // projector columns: twnl times the phases
  if (ctx.nproj) build_anl(ctx, ctx.d_gx_w, ngw, ctx.d_twnl, ctx.d_anl);
}

// ------------------------------------------------------------ stress
// The stress tensor of EnergyFunctional::energy with compute_stress
// (src/EnergyFunctional.cpp:440-1044), components in the reference's Voigt
// order xx yy zz xy yz xz.  Every part is a reduction over the state left
// by update_density, update_vhxc and energy; the nonlocal part recomputes
// the projections with the strain derivatives of the projector forms (one
// K x nproj block and one GEMM per component) instead of storing them.
__device__ __forceinline__ void voigt6(double x, double y, double z, double w, double* a) {
  a[0] += w * x * x;
  a[1] += w * y * y;
  a[2] += w * z * z;
  a[3] += w * x * y;
  a[4] += w * y * z;
  a[5] += w * x * z;
}

// kinetic: sum_n occ_n |c_n(G)|^2 G_i G_j (src/EnergyFunctional.cpp:440-570)
struct EkinStressF {
  const double2* c; const double* gx; const double* occ; int ngw;
  __device__ void operator()(size_t i, double* a) const {
    const int n = (int)(i / ngw), ig = (int)(i - (size_t)n * ngw);
    const double2 v = c[i];
    voigt6(gx[ig], gx[ngw + ig], gx[2 * ngw + ig], occ[n] * (v.x * v.x + v.y * v.y), a);
  }
};

// local pseudopotential: 2/|G| Re(conj(rho_el) dV_ion) G_i G_j, dV_ion =
// sum_s S_s(G) dV_s(G)/Omega (src/EnergyFunctional.cpp:574-608)
struct EpsStressF {
  const double2* rhog; const double2* sfac; const double* dvps; const double* g2i;
  const double* gx; int ng, nsp; double om_inv;
  __device__ void operator()(size_t i, double* a) const {
    double dx = 0.0, dy = 0.0;
    for (int s = 0; s < nsp; s++) {
      const double2 sg = sfac[(size_t)s * ng + i];
      const double d = dvps[(size_t)s * ng + i];
      dx += sg.x * d;
      dy += sg.y * d;
    }
    const double2 r = rhog[i];
    const double w = 2.0 * sqrt(g2i[i]) * om_inv * (r.x * dx + r.y * dy);
    voigt6(gx[i], gx[ng + i], gx[2 * ng + i], w, a);
  }
};

// Hartree with the Gaussian pseudocharges: |rho_t|^2/G^4 + sum_s
// rcps^2/2 Re(rho_t conj S_s) rhops_s/G^2 (src/EnergyFunctional.cpp:611-683)
struct EhartStressF {
  const double2* rhog; const double2* rhops_t; const double2* sfac; const double* rhops;
  const double* g2i; const double* gx; int ng, nsp; double om_inv, rc2;
  __device__ void operator()(size_t i, double* a) const {
    const double2 r = rhog[i], p = rhops_t[i];
    const double tx = r.x * om_inv + p.x, ty = r.y * om_inv + p.y;
    const double gi2 = g2i[i];
    double w = (tx * tx + ty * ty) * gi2 * gi2;
    for (int s = 0; s < nsp; s++) {
      const double2 sg = sfac[(size_t)s * ng + i];
      w += 0.5 * rc2 * (tx * sg.x + ty * sg.y) * rhops[(size_t)s * ng + i] * gi2;
    }
    voigt6(gx[i], gx[ng + i], gx[2 * ng + i], w, a);
  }
};

// XC, LDA: sum_r rho (e - v) with e the energy per particle
struct LdaStressF {
  const double* rhoe; const double* rho; const double* v;
  __device__ void operator()(size_t i, double* a) const { a[0] += rhoe[i] - rho[i] * v[i]; }
};

// XC, GGA gradient part: v2 (|grad rho|^2 delta_ij + d_i rho d_j rho)
// (src/XCPotential.cpp:520-640)
struct GgaStressF {
  const double* grad; const double* v2; size_t N;
  __device__ void operator()(size_t i, double* a) const {
    const double x = grad[i], y = grad[N + i], z = grad[2 * N + i];
    const double w = v2[i], g2 = x * x + y * y + z * z;
    a[0] += w * (g2 + x * x);
    a[1] += w * (g2 + y * y);
    a[2] += w * (g2 + z * z);
    a[3] += w * x * y;
    a[4] += w * y * z;
    a[5] += w * x * z;
  }
};

// Strain derivative of the projector forms times the structure phase,
// component ij, for every projector column (src/NonLocalPotential.cpp:
// 266-440 for l = 0, 1, phases as in anl):
//   l = 0: dt = s14pi dV/dG G_i G_j / |G|
//   l = 1: dt_m = -y_m (V - |G| dV/dG) G_i G_j / G^2 + [j == m] V y_i,
//          y_m = s34pi G_m / |G|
__global__ void k_danl(const double* __restrict__ gx, const double* __restrict__ g2, int ngw,
                       const double* __restrict__ vnl, const double* __restrict__ dvnl,
                       const int* __restrict__ pcol, const double* __restrict__ tau, int i,
                       int j, double2* __restrict__ out) {
  const int p = blockIdx.y;
  const int l = pcol[4 * p], m = pcol[4 * p + 1], rad = pcol[4 * p + 2], at = pcol[4 * p + 3];
  const double tx = tau[3 * at], ty = tau[3 * at + 1], tz = tau[3 * at + 2];
  const double s14pi = sqrt(1.0 / (4.0 * M_PI)), s34pi = sqrt(3.0 / (4.0 * M_PI));
  const double* v = vnl + (size_t)rad * ngw;
  const double* dv = dvnl + (size_t)rad * ngw;
  double2* o = out + (size_t)p * ngw;
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ngw; ig += gridDim.x * blockDim.x) {
    const double G[3] = {gx[ig], gx[ngw + ig], gx[2 * ngw + ig]};
    const double gg = g2[ig];
    const double gi = gg > 0.0 ? 1.0 / sqrt(gg) : 0.0;
    double t;
    if (l == 0) {
      t = gi * s14pi * dv[ig] * G[i] * G[j];
    } else {
      const double ym = s34pi * G[m] * gi;
      const double g = gg * gi;
      t = -ym * (v[ig] - g * dv[ig]) * gi * gi * G[i] * G[j];
      if (j == m) t += v[ig] * s34pi * G[i] * gi;
    }
    double sn, cs;
    sincos(G[0] * tx + G[1] * ty + G[2] * tz, &sn, &cs);
    // exp(-i G.tau) = (cs, -sn); times -i for l = 1: (-sn, -cs)
    o[ig] = (l == 0) ? make_double2(t * cs, -t * sn) : make_double2(-t * sn, -t * cs);
  }
}

// sum_{p,n} 2 occ_n fnl(p,n) dF(p,n), fnl = D F / Omega
struct EnlStressF {
  const double* fnl; const double* dfnl; const double* occ; int np;
  __device__ void operator()(size_t i, double* a) const {
    const int n = (int)(i / np);
    a[0] += 2.0 * occ[n] * fnl[i] * dfnl[i];
  }
};

// stress slots: kinetic, local, Hartree, XC, nonlocal sums (6 each)
enum : int { SS_EKIN = SLOT_STRESS, SS_EPS = SLOT_STRESS + 6, SS_EHART = SLOT_STRESS + 12,
             SS_EXC = SLOT_STRESS + 18, SS_ENL = SLOT_STRESS + 24 };
static_assert(SS_ENL + 6 <= SLOT_SCRATCH, "stress slots overlap the scratch slots");

void compute_stress(Context& ctx) {
  const double om_inv = 1.0 / ctx.wb.omega;
  const int ngw = ctx.wb.ng, ngv = ctx.vb.ng, nst = ctx.nst;
  const int nsp = (int)ctx.species.size();
  const size_t N = ctx.N();
  reduce<6>(ctx, EkinStressF{(const double2*)ctx.d_c, ctx.d_gx_w, ctx.d_occ, ngw},
            (size_t)ngw * nst, SS_EKIN);
  reduce<6>(ctx, EpsStressF{(const double2*)ctx.d_rhog, (const double2*)ctx.d_sfac, ctx.d_dvps,
                            ctx.d_g2i_v, ctx.d_gx_v, ngv, nsp, om_inv},
            (size_t)ngv, SS_EPS);
  reduce<6>(ctx, EhartStressF{(const double2*)ctx.d_rhog, (const double2*)ctx.d_rhops,
                              (const double2*)ctx.d_sfac, ctx.d_rhops_sp, ctx.d_g2i_v,
                              ctx.d_gx_v, ngv, nsp, om_inv, 1.5 * 1.5},
            (size_t)ngv, SS_EHART);
  if (ctx.xc == "LDA")
    reduce<1>(ctx, LdaStressF{ctx.d_exc, ctx.d_rhor, ctx.d_vxc}, N, SS_EXC);
  else
    reduce<6>(ctx, GgaStressF{ctx.d_grad, ctx.d_vx2, N}, N, SS_EXC);
  compute_stress_nl(ctx);
}

// The nonlocal part alone (src/NonLocalPotential.cpp:1790-2069): per Voigt
// component the strain derivative of the projector forms times the phases,
// dF = 2 A_ij^T C, contracted with D F / Omega into the SS_ENL slots.
void compute_stress_nl(Context& ctx) {
  static const int vi[6] = {0, 1, 2, 0, 1, 0}, vj[6] = {0, 1, 2, 1, 2, 2};
  const int ngw = ctx.wb.ng, nst = ctx.nst, np = ctx.nproj;
  QBX_CUDA(cudaMemsetAsync(ctx.d_scalars + SS_ENL, 0, 6 * sizeof(double), ctx.stream));
  if (np) {
    const int K = 2 * ngw;
    if (!ctx.d_astress) ctx.d_astress = dalloc<double>((size_t)K * np);
    const bool mx = ctx.precision == MIXED && ctx.gemm_backend == 1 &&
                    tc_gemm_supported(ctx, true, false, np, nst, K);
    if (mx && !ctx.sa_hi) {
      QBX_CUDA(cudaMalloc(&ctx.sa_hi, (size_t)ctx.ldp * np * 2));
      QBX_CUDA(cudaMalloc(&ctx.sa_lo, (size_t)ctx.ldp * np * 2));
    }
    const double two = 2.0, zero = 0.0;
    for (int k = 0; k < 6; k++) {
      dim3 grid((ngw + kThreads - 1) / kThreads, np);
      k_danl<<<grid, kThreads, 0, ctx.stream>>>(ctx.d_gx_w, ctx.d_g2_w, ngw, ctx.d_vnl,
                                                ctx.d_dvnl, ctx.d_pcol, ctx.d_tau_all, vi[k],
                                                vj[k], (double2*)ctx.d_astress);
      QBX_LAUNCHED(ctx);
      // dF = 2 A_ij^T C; the G=0 row of A_ij is zero, so no correction
      if (mx) {
        split_bf16_2d(ctx, ctx.d_astress, K, np, K, ctx.sa_hi, ctx.sa_lo, ctx.ldp);
        split_gemm(ctx, true, false, np, nst, K, 2.0, ctx.sa_hi, ctx.sa_lo, ctx.ldp,
                   ctx.cs_hi[0], ctx.cs_lo[0], ctx.ldp, 0.0, ctx.d_dfnl);
      } else {
        QBX_BLAS(cublasDgemm(ctx.blas, CUBLAS_OP_T, CUBLAS_OP_N, np, nst, K, &two,
                             ctx.d_astress, K, ctx.d_c, K, &zero, ctx.d_dfnl, np));
      }
      reduce<1>(ctx, EnlStressF{ctx.d_fnl, ctx.d_dfnl, ctx.d_occ, np}, (size_t)np * nst,
                SS_ENL + k);
    }
  }
}

// sigma_enl of NonLocalPotential::energy (src/NonLocalPotential.cpp:2057-2066)
// from E_nl and the SS_ENL slots read back after compute_stress_nl
void nl_stress_part(const Context& ctx, double enl, double* sigma_enl) {
  const double om_inv = 1.0 / ctx.wb.omega;
  for (int k = 0; k < 6; k++)
    sigma_enl[k] = ((k < 3 ? enl : 0.0) + ctx.h_scalars[SS_ENL + k]) * om_inv;
}

// The stress parts from the slots of compute_stress and the energies of the
// same state (src/EnergyFunctional.cpp:397-1044 with compute_stress).
void finish_stress(Context& ctx) {
  const double om = ctx.wb.omega, om_inv = 1.0 / om;
  const double N = (double)ctx.N();
  const double* h = ctx.h_scalars;
  double* P = ctx.sigma_parts;        // ekin, eps, enl, ehart, exc, esr
  const double eye[6] = {1, 1, 1, 0, 0, 0};
  for (int k = 0; k < 6; k++) {
    P[k] = 2.0 * h[SS_EKIN + k] * om_inv;
    P[6 + k] = eye[k] * ctx.eps * om_inv + h[SS_EPS + k];
    P[12 + k] = (eye[k] * ctx.enl + h[SS_ENL + k]) * om_inv;
    P[18 + k] = eye[k] * ctx.ehart * om_inv - 8.0 * M_PI * h[SS_EHART + k];
    if (ctx.xc == "LDA") {
      P[24 + k] = -eye[k] * h[SS_EXC] / N;
    } else {
      const double dsum = ctx.exc * N / om - ctx.xc_rhov1;   // sum rho (e - v1)
      P[24 + k] = -(eye[k] * dsum + h[SS_EXC + k]) / N;
    }
    P[30 + k] = ctx.sigma_esr[k];
  }
  for (int k = 0; k < 6; k++) {
    double s = 0.0;
    for (int q = 0; q < 6; q++) s += P[6 * q + k];
    ctx.sigma[k] = s;
  }
  ctx.have_stress = true;
}

}  // namespace qbx
