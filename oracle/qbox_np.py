"""CPU restatement (numpy, FP64) of the reference's Kohn-Sham electronic step.

TEST INFRASTRUCTURE - this is the oracle, not the product.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg may use it,
and only as the checker.  Its results are pinned against the reference itself
built single-task (oracle/_ref, see oracle/Makefile) by tests/test_oracle.py
and the committed fixtures in tests/golden/.

Each function cites the reference file:line it restates.  The reference keeps
Gamma-point wavefunctions on the half sphere of G vectors and represents them
as real matrices of twice the number of rows ("DoubleMatrix proxy"); every
inner product therefore carries the factor 2 for +G/-G and a correction that
removes the double-counted G=0 row.  Here coefficients are kept as complex
arrays c[n, ig] in sorted Miller order, and the same conventions are written
out explicitly.

Grids are numpy arrays of shape (np2, np1, np0) indexed [z, y, x], which is
the reference's memory order x + np0*(y + np1*z) (src/BasisMapping.cpp:206-216).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

FPI = 4.0 * math.pi
RCPS = 1.5           # Gaussian pseudocharge radius, src/AtomSet.cpp:43-44


# --------------------------------------------------------------------------
# basis and FFT sizes
# --------------------------------------------------------------------------
def factorizable(n: int) -> bool:
    """src/Basis.cpp:105-133: n = 2^a 3^{0,1,2} 5^{0,1} 7^{0,1} 11^{0,1}."""
    for p in (11, 7, 5, 3, 3):
        if n % p == 0:
            n //= p
    while n % 2 == 0:
        n //= 2
    return n == 1


def reciprocal(cell: np.ndarray) -> np.ndarray:
    return 2.0 * math.pi * np.linalg.inv(cell).T


def fft_size_for(cell: np.ndarray, ecut: float) -> List[int]:
    """src/Basis.cpp:332-341,513-521: np_i = smallest factorizable even
    number >= 2*hmax_i with hmax_i = int(1.5 + sqrt(2 ecut)/(2 pi) |a_i|)."""
    fac = math.sqrt(2.0 * ecut) / (2.0 * math.pi)
    out = []
    for i in range(3):
        hmax = int(1.5 + fac * np.linalg.norm(cell[i]))
        n = 2 * hmax
        while not factorizable(n):
            n += 2
        out.append(n)
    return out


def dense_grid(cell: np.ndarray, ecut: float) -> List[int]:
    """src/ChargeDensity.cpp:36-49: vbasis at 4*ecut, grid np+2 rounded up to
    a factorizable size; the wavefunction FFTs use the same grid (:98)."""
    out = []
    for n in fft_size_for(cell, 4.0 * ecut):
        n += 2
        while not factorizable(n):
            n += 2
        out.append(n)
    return out


def half_sphere(cell: np.ndarray, ecut: float) -> np.ndarray:
    """Sorted (h,k,l) of {G: |G|^2 < 2 ecut} on the Gamma half sphere
    (rods of src/Basis.cpp:357-447)."""
    b = reciprocal(cell)
    fac = math.sqrt(2.0 * ecut) / (2.0 * math.pi)
    m = [int(1.5 + fac * np.linalg.norm(cell[i])) for i in range(3)]
    h, k, l = np.meshgrid(np.arange(0, m[0] + 1), np.arange(-m[1], m[1] + 1),
                          np.arange(-m[2], m[2] + 1), indexing="ij")
    h, k, l = h.ravel(), k.ravel(), l.ravel()
    keep = (h > 0) | ((h == 0) & (k > 0)) | ((h == 0) & (k == 0) & (l >= 0))
    h, k, l = h[keep], k[keep], l[keep]
    gx = h * b[0, 0] + k * b[1, 0] + l * b[2, 0]
    gy = h * b[0, 1] + k * b[1, 1] + l * b[2, 1]
    gz = h * b[0, 2] + k * b[1, 2] + l * b[2, 2]
    inside = gx * gx + gy * gy + gz * gz < 2.0 * ecut
    hkl = np.stack([h[inside], k[inside], l[inside]], 1).astype(np.int64)
    order = np.lexsort((hkl[:, 2], hkl[:, 1], hkl[:, 0]))
    return hkl[order]


@dataclass
class Basis:
    """G vectors of a Gamma half-sphere basis (src/Basis.cpp:646-690).
    With fixed_hkl the Miller set is given instead of cut from the sphere
    (used to differentiate at a fixed set of plane waves under strain)."""
    cell: np.ndarray
    ecut: float
    fixed_hkl: Optional[np.ndarray] = None
    hkl: np.ndarray = field(init=False)
    gx: np.ndarray = field(init=False)   # (ng, 3)
    g2: np.ndarray = field(init=False)
    g: np.ndarray = field(init=False)
    g2i: np.ndarray = field(init=False)
    gi: np.ndarray = field(init=False)

    def __post_init__(self):
        self.hkl = half_sphere(self.cell, self.ecut) if self.fixed_hkl is None else self.fixed_hkl
        b = reciprocal(self.cell)
        self.gx = self.hkl @ b
        self.g2 = (self.gx ** 2).sum(1)
        self.g = np.sqrt(self.g2)
        with np.errstate(divide="ignore"):
            self.gi = np.where(self.g > 0, 1.0 / np.where(self.g > 0, self.g, 1), 0.0)
        self.g2i = self.gi * self.gi

    @property
    def size(self) -> int:
        return self.hkl.shape[0]

    def g0(self) -> int:
        return int(np.flatnonzero((self.hkl == 0).all(1))[0])


class Grid:
    """Complex 3-D FFT on the dense grid for a half-sphere basis
    (src/FourierTransform.cpp:147-239; forward scales by 1/N, src:733-744)."""

    def __init__(self, basis: Basis, shape: List[int]):
        self.n0, self.n1, self.n2 = shape
        self.N = self.n0 * self.n1 * self.n2
        h, k, l = basis.hkl[:, 0], basis.hkl[:, 1], basis.hkl[:, 2]
        self.ip = ((l % self.n2) * self.n1 + (k % self.n1)) * self.n0 + (h % self.n0)
        self.im = (((-l) % self.n2) * self.n1 + ((-k) % self.n1)) * self.n0 + ((-h) % self.n0)
        self.shape = (self.n2, self.n1, self.n0)

    def backward(self, c: np.ndarray, c2: Optional[np.ndarray] = None) -> np.ndarray:
        """src/BasisMapping.cpp:628-700 + fz_inv/fxy_inv: one or two real
        functions packed as c1 + i c2; returns the complex grid."""
        z = np.zeros(self.N, complex)
        if c2 is None:
            z[self.ip] = c
            z[self.im] = np.conj(c)
        else:
            z[self.ip] = c + 1j * c2
            z[self.im] = np.conj(c) + 1j * np.conj(c2)
        return np.fft.ifftn(z.reshape(self.shape)) * self.N

    def forward(self, f: np.ndarray, two: bool = False):
        """src/BasisMapping.cpp:703-750 + fxy/fz: grid -> coefficients."""
        z = (np.fft.fftn(f.reshape(self.shape)) / self.N).ravel()
        if not two:
            return z[self.ip]
        zp, zm = z[self.ip], np.conj(z[self.im])
        return 0.5 * (zp + zm), -0.5j * (zp - zm)


# --------------------------------------------------------------------------
# species: radial tables -> G-space splines (src/Species.cpp:510-1055)
# --------------------------------------------------------------------------
def simpsn(t: np.ndarray) -> float:
    """src/Species.cpp:34-48 (end-corrected trapezoid weights)."""
    n = t.size
    c = (17.0 / 48.0, 59.0 / 48.0, 43.0 / 48.0, 49.0 / 48.0)
    s = sum(c[i] * (t[i] + t[n - 1 - i]) for i in range(4))
    return s + t[4:n - 4].sum()


def sinft(y: np.ndarray) -> np.ndarray:
    """src/sinft.cpp: y_k = sum_{j=1}^{n-1} y_j sin(pi j k / n), computed as
    the reference does through a length-2n complex FFT of the odd extension."""
    n = y.size
    z = np.zeros(2 * n, complex)
    z[1:n] = y[1:]
    z[2 * n - np.arange(1, n)] = -y[1:]
    return -0.5 * np.fft.fft(z)[:n].imag


def cosft1(y: np.ndarray) -> np.ndarray:
    """src/sinft.cpp cosft1: y has n+1 entries; returns n values
    0.5*Re(FFT of the even extension)."""
    n = y.size - 1
    z = np.zeros(2 * n, complex)
    z[0] = y[0]
    z[1:n + 1] = y[1:n + 1]
    z[2 * n - np.arange(1, n + 1)] = y[1:n + 1]
    return 0.5 * np.fft.fft(z)[:n].real


def spline(x, y, yp_left, yp_right, nat_left, nat_right):
    """src/spline.cpp spline(): second derivatives of a cubic spline."""
    n = x.size
    d = np.empty(n); e = np.empty(n); f = np.empty(n); y2 = np.empty(n)
    third, sixth = 1.0 / 3.0, 1.0 / 6.0
    if nat_left == 0:
        h = x[1] - x[0]
        d[0], e[0], f[0] = third * h, sixth * h, 0.0
        y2[0] = (y[1] - y[0]) / h - yp_left
    else:
        d[0], e[0], f[0], y2[0] = 1.0, 0.0, 0.0, 0.0
    if nat_right == 0:
        h = x[n - 1] - x[n - 2]
        d[n - 1], e[n - 1], f[n - 1] = third * h, 0.0, sixth * h
        y2[n - 1] = yp_right - (y[n - 1] - y[n - 2]) / h
    else:
        d[n - 1], e[n - 1], f[n - 1], y2[n - 1] = 1.0, 0.0, 0.0, 0.0
    hp = x[2:] - x[1:-1]
    hm = x[1:-1] - x[:-2]
    d[1:-1] = third * (hp + hm)
    e[1:-1] = sixth * hp
    f[1:-1] = sixth * hm
    y2[1:-1] = (y[2:] - y[1:-1]) / hp - (y[1:-1] - y[:-2]) / hm
    # tridiagonal solve, src/spline.cpp tridsolve()
    for i in range(1, n):
        f[i] /= d[i - 1]
        d[i] -= f[i] * e[i - 1]
    for i in range(1, n):
        y2[i] -= f[i] * y2[i - 1]
    y2[n - 1] /= d[n - 1]
    for i in range(n - 2, -1, -1):
        y2[i] = (y2[i] - e[i] * y2[i + 1]) / d[i]
    return y2


def splintd(xa, ya, y2a, x):
    """src/spline.cpp splint/splintd, vectorised: value and derivative."""
    n = xa.size
    kl = np.clip(np.searchsorted(xa, x, side="right") - 1, 0, n - 2)
    kh = kl + 1
    h = xa[kh] - xa[kl]
    a = (xa[kh] - x) / h
    b = (x - xa[kl]) / h
    y = a * ya[kl] + b * ya[kh] + h * h * (1.0 / 6.0) * (
        (a ** 3 - a) * y2a[kl] + (b ** 3 - b) * y2a[kh])
    dy = (ya[kh] - ya[kl]) / h + h * (((1.0 / 6.0) - 0.5 * a * a) * y2a[kl]
                                      + (0.5 * b * b - (1.0 / 6.0)) * y2a[kh])
    return y, dy


class Species:
    """G-space tables of one SLPP species (src/Species.cpp:510-1055,
    evaluation :1133-1192)."""

    def __init__(self, sp):
        self.zval = float(sp.zval)
        dr = sp.mesh_spacing
        ndft = 1
        while ndft * dr < 40.0:
            ndft *= 2
        self.ndft = ndft
        r = np.arange(ndft) * dr
        vloc_in = sp.local_potential()
        npts = vloc_in.size
        vlocr = np.empty(ndft)
        vlocr[:npts] = vloc_in
        vlocr[npts:] = -self.zval / r[npts:]
        z = self.zval
        vlocr[0] += (z / RCPS) * (2.0 / math.sqrt(math.pi))
        from math import erf
        vlocr[1:] += (z / r[1:]) * np.array([erf(x / RCPS) for x in r[1:]])
        vlocr *= FPI * r * dr
        v0 = simpsn(vlocr * r)
        vg = sinft(vlocr)
        fac = math.pi / (ndft * dr)
        self.gspl = np.arange(ndft) * fac
        vg[0] = v0
        vg[1:] /= self.gspl[1:]
        self.vlocg = vg
        self.vlocg2 = spline(self.gspl, vg, 0.0, 0.0, 0, 1)
        self.proj = []     # (l, table, second derivatives)
        self.dmat = dict(sp.dmatrix())
        for l, phi_in in sp.projectors():
            phi = np.zeros(ndft)
            phi[:npts] = phi_in
            vnlr = FPI * dr * phi
            if l == 0:
                v0 = simpsn(vnlr * r * r)
                t = sinft(vnlr * r)
                t[0] = v0
                t[1:] /= self.gspl[1:]
                t2 = spline(self.gspl, t, 0.0, 0.0, 0, 1)
            elif l == 1:
                s = sinft(vnlr)
                fint = np.zeros(ndft)
                fint[1:] = s[1:] / self.gspl[1:] ** 2
                yy = np.zeros(ndft + 1)
                yy[:ndft] = vnlr * r
                c = cosft1(yy)
                t = np.zeros(ndft)
                t[1:] = fint[1:] - c[1:] / self.gspl[1:]
                t2 = spline(self.gspl, t, 0.0, 0.0, 1, 1)
            else:
                raise NotImplementedError("l > 1 projectors")
            self.proj.append((l, t, t2))
        self.nlm = sum(2 * l + 1 for l, _, _ in self.proj)
        self.eself = z * z / (math.sqrt(2.0 * math.pi) * RCPS)

    def dvlocg(self, g):
        v, dv = splintd(self.gspl, self.vlocg, self.vlocg2, g)
        out = g > self.gspl[-1]
        return np.where(out, 0.0, v), np.where(out, 0.0, dv)

    def vnlg(self, iop, g):
        l, t, t2 = self.proj[iop]
        v, dv = splintd(self.gspl, t, t2, g)
        out = g > self.gspl[-1]
        return np.where(out, 0.0, v), np.where(out, 0.0, dv)

    def rhopsg(self, g):
        return -self.zval * np.exp(-0.25 * RCPS * RCPS * g * g)


# --------------------------------------------------------------------------
# XC functionals (src/LDAFunctional.cpp:92-160, src/PBEFunctional.cpp:168-280)
# --------------------------------------------------------------------------
def lda_pz(rho):
    """Perdew-Zunger LDA, unpolarized (src/LDAFunctional.cpp:92-150)."""
    c1 = 0.6203504908994001
    c3 = -0.610887057711
    A, B, b1, b2, G = 0.0311, -0.048, 1.0529, 0.3334, -0.1423
    D = G / (1.0 + b1 + b2) - B
    C = -A - D - G * ((b1 / 2.0 + b2) / ((1.0 + b1 + b2) * (1.0 + b1 + b2)))
    ee = np.zeros_like(rho)
    vv = np.zeros_like(rho)
    pos = rho > 0.0
    r = rho[pos]
    rs = c1 / np.cbrt(r)
    vx = c3 / rs
    ex = 0.75 * vx
    lo = rs < 1.0
    ec = np.empty_like(rs); vc = np.empty_like(rs)
    lr = np.log(rs[lo]); rl = rs[lo]
    ec[lo] = A * lr + B + C * rl * lr + D * rl
    vc[lo] = A * lr + (B - A / 3.0) + (2.0 / 3.0) * C * rl * lr + ((2.0 * D - C) / 3.0) * rl
    rh = rs[~lo]
    sq = np.sqrt(rh)
    den = 1.0 + b1 * sq + b2 * rh
    ec[~lo] = G / den
    vc[~lo] = ec[~lo] * (1.0 + (7.0 / 6.0) * b1 * sq + (4.0 / 3.0) * b2 * rh) / den
    ee[pos] = ex + ec
    vv[pos] = vx + vc
    return ee, vv


def pbe(rho, grad):
    """PBE exchange-correlation (src/PBEFunctional.cpp:168-280, gcor2 :488)."""
    third, third4 = 1.0 / 3.0, 4.0 / 3.0
    ax = -0.7385587663820224058
    um, uk = 0.2195149727645171, 0.804
    ul = um / uk
    pi32third = 3.09366772628014
    alpha = 1.91915829267751
    seven_sixth = 7.0 / 6.0
    four_over_pi = 1.27323954473516
    gamma = 0.03109069086965489
    bet = 0.06672455060314922
    delt = bet / gamma
    exc = np.zeros_like(rho); v1 = np.zeros_like(rho); v2 = np.zeros_like(rho)
    m = rho >= 1.e-18
    r = rho[m]; gr = grad[m]
    rh13 = r ** third
    exunif = ax * rh13
    fk = pi32third * rh13
    s = gr / (2.0 * fk * r)
    s2 = s * s
    p0 = 1.0 + ul * s2
    fxpbe = 1.0 + uk - uk / p0
    ex = exunif * fxpbe
    fs = 2.0 * uk * ul / (p0 * p0)
    vx1 = third4 * exunif * (fxpbe - s2 * fs)
    vx2 = -exunif * fs / (r * 4.0 * fk * fk)
    rs = alpha / fk
    twoks = 2.0 * np.sqrt(four_over_pi * fk)
    t = gr / (twoks * r)
    rtrs = np.sqrt(rs)
    a_, a1, b1, b2, b3, b4 = 0.0310907, 0.2137, 7.5957, 3.5876, 1.6382, 0.49294
    q0 = -2.0 * a_ * (1.0 + a1 * rtrs * rtrs)
    q1 = 2.0 * a_ * rtrs * (b1 + rtrs * (b2 + rtrs * (b3 + rtrs * b4)))
    q2 = np.log(1.0 + 1.0 / q1)
    ec = q0 * q2
    q3 = a_ * (b1 / rtrs + 2.0 * b2 + rtrs * (3.0 * b3 + 4.0 * b4 * rtrs))
    ecrs = -2.0 * a_ * a1 * q2 - q0 * q3 / (q1 * (1.0 + q1))
    vc = ec - rs * ecrs * third
    pon = -ec / gamma
    b = delt / (np.exp(pon) - 1.0)
    b2_ = b * b
    t2 = t * t
    t4 = t2 * t2
    q4 = 1.0 + b * t2
    q5 = q4 + b2_ * t4
    h = gamma * np.log(1.0 + delt * q4 * t2 / q5)
    t6 = t4 * t2
    rsthrd = rs * third
    fac = delt / b + 1.0
    bec = b2_ * fac / bet
    q8 = q5 * q5 + delt * q4 * q5 * t2
    q9 = 1.0 + 2.0 * b * t2
    hb = -bet * b * t6 * (2.0 + b * t2) / q8
    hrs = -rsthrd * hb * bec * ecrs
    ht = 2.0 * bet * q9 / q8
    vc1 = vc + h + hrs - t2 * ht * seven_sixth
    vc2 = -ht / (r * twoks * twoks)
    exc[m] = ex + ec + h
    v1[m] = vx1 + vc1
    v2[m] = vx2 + vc2
    return exc, v1, v2


# --------------------------------------------------------------------------
# the electronic step
# --------------------------------------------------------------------------
def fold_in_ws(v: np.ndarray, cell: np.ndarray) -> np.ndarray:
    """src/UnitCell.cpp:157-187 (13 neighbour vectors, 1e-10 tolerance)."""
    a = cell
    an = [a[0], a[1], a[2], a[0] + a[1], a[0] - a[1], a[1] + a[2], a[1] - a[2],
          a[2] + a[0], a[2] - a[0], a[0] + a[1] + a[2], a[0] - a[1] - a[2],
          a[0] + a[1] - a[2], a[0] - a[1] + a[2]]
    v = v.copy()
    eps = 1.e-10
    for _ in range(10):
        done = True
        for ai in an:
            h = 0.5 * ai @ ai
            sp = v @ ai
            if sp > h + eps:
                done = False
                while v @ ai > h + eps:
                    v -= ai
            elif sp < -h - eps:
                done = False
                while v @ ai < -h - eps:
                    v += ai
        if done:
            break
    return v


# Voigt order of the reference's stress components: xx yy zz xy yz xz
VOIGT = ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2))


def esr_forces(system, zv, positions, with_stress=False):
    """Pseudocharge repulsion E_sr, its forces and (with_stress) its stress
    sigma_esr (src/EnergyFunctional.cpp:1112-1194)."""
    cell = system.cell
    b = reciprocal(cell)
    d = [2.0 * math.pi / np.linalg.norm(b[i]) for i in range(3)]
    nsp = len(positions)
    esr = 0.0
    sig = np.zeros(6)
    f = [np.zeros_like(p) for p in positions]
    from math import erfc
    for is1 in range(nsp):
        for is2 in range(is1, nsp):
            rc12 = math.sqrt(2.0 * RCPS * RCPS)
            nc = [int(8.0 * rc12 / d[i]) for i in range(3)]
            for ia1 in range(len(positions[is1])):
                ia2min = ia1 if is1 == is2 else 0
                for ia2 in range(ia2min, len(positions[is2])):
                    same = is1 == is2 and ia1 == ia2
                    v12 = fold_in_ws(positions[is1][ia1] - positions[is2][ia2], cell)
                    for i0 in range(-nc[0], nc[0] + 1):
                        for i1 in range(-nc[1], nc[1] + 1):
                            for i2 in range(-nc[2], nc[2] + 1):
                                if same and i0 == 0 and i1 == 0 and i2 == 0:
                                    continue
                                fac = 0.5 if same else 1.0
                                x = v12 + i0 * cell[0] + i1 * cell[1] + i2 * cell[2]
                                r12 = math.sqrt(x @ x)
                                arg = r12 / rc12
                                term = zv[is1] * zv[is2] * erfc(arg) / r12
                                esr += fac * term
                                de = 2.0 * zv[is1] * zv[is2] * math.exp(-arg * arg) / (
                                    rc12 * math.sqrt(math.pi))
                                dedr = -fac * (term + de) / (r12 * r12)
                                f[is1][ia1] -= dedr * x
                                f[is2][ia2] += dedr * x
                                if with_stress:
                                    for k, (i, j) in enumerate(VOIGT):
                                        sig[k] += dedr * x[i] * x[j]
    if with_stress:
        omega = abs(np.linalg.det(np.asarray(cell, float)))
        return esr, f, -sig / omega
    return esr, f


class ElectronicStep:
    """State and operators of the reference's SCF iteration with nite=0
    (src/BOSampleStepper.cpp:795-977) on one Gamma-point SlaterDet."""

    def __init__(self, system, c: Optional[np.ndarray] = None, like=None):
        """like: another ElectronicStep whose plane-wave sets and grid are
        kept (a strained copy of a system for finite differences)."""
        self.system = system
        cell = np.array(system.cell, float)
        self.cell = cell
        self.omega = abs(np.linalg.det(cell))
        self.wb = Basis(cell, system.ecut, None if like is None else like.wb.hkl)
        self.vb = Basis(cell, 4.0 * system.ecut, None if like is None else like.vb.hkl)
        shape = dense_grid(cell, system.ecut) if like is None else list(like.grid_shape)
        self.grid_shape = shape
        self.wgrid = Grid(self.wb, shape)
        self.vgrid = Grid(self.vb, shape)
        self.N = self.wgrid.N
        self.nst = system.nbands
        self.occ = np.full(self.nst, 2.0)
        self.xc = system.xc
        self.species = [Species(sp) for sp in system.species]
        self.positions = [system.positions(i) for i in range(len(system.species))]
        if c is None:
            c = system.coefficients(self.wb.hkl)
        self.c = np.array(c, complex)
        self.g0 = self.wb.g0()
        self._setup_tables()
        self.gram()
        self.c_last = None
        self.dc_last = None
        self.extrapolate = False

    # ---- setup (src/EnergyFunctional.cpp:1047-1245, NonLocal update_twnl)
    def _setup_tables(self):
        vb, wb = self.vb, self.wb
        om = self.omega
        self.vion_g = np.zeros(vb.size, complex)
        self.rhops_t = np.zeros(vb.size, complex)
        self.sfac = []
        self.vps = []
        self.rhops = []
        for isp, sp in enumerate(self.species):
            tau = self.positions[isp]
            phase = -(vb.gx @ tau.T)             # (ng, na)
            s = np.exp(1j * phase).sum(1)        # S(G) = sum_a exp(-i G.tau)
            self.sfac.append(s)
            v, dv = sp.dvlocg(vb.g)
            vps = v / om
            rhops = sp.rhopsg(vb.g) / om
            self.vps.append(vps); self.rhops.append(rhops)
            self.vion_g += s * vps
            self.rhops_t += s * rhops
        zv = [sp.zval for sp in self.species]
        self.esr, self.fion_esr = esr_forces(self.system, zv, self.positions)
        self.eself = sum(sp.eself * len(self.positions[i])
                         for i, sp in enumerate(self.species))
        # nonlocal projectors twnl (src/NonLocalPotential.cpp:235-560)
        s14pi = math.sqrt(1.0 / FPI)
        s34pi = math.sqrt(3.0 / FPI)
        self.nl = []
        for isp, sp in enumerate(self.species):
            if not sp.proj:
                continue
            tw = []
            lp = []
            dfac = []
            for iop, (l, _, _) in enumerate(sp.proj):
                v, dv = sp.vnlg(iop, wb.g)
                if l == 0:
                    tw.append(s14pi * v); lp.append(0); dfac.append(sp.dmat[0])
                else:
                    for j in range(3):
                        tw.append(s34pi * wb.gx[:, j] * wb.gi * v)
                        lp.append(1); dfac.append(sp.dmat[1])
            self.nl.append((isp, np.array(tw), np.array(lp), np.array(dfac)))

    def anl(self, isp, tw, lp):
        """Projector x phase, A[ipr, ia, G] (src/NonLocalPotential.cpp:1316-1394)."""
        tau = self.positions[isp]
        e = np.exp(-1j * (self.wb.gx @ tau.T)).T    # (na, ng) exp(-i G.tau)
        a = tw[:, None, :] * e[None, :, :]
        a[lp == 1] *= -1j
        return a

    # ---- SlaterDet operations
    def real_dot(self, x, y):
        """2 Re sum_G conj(x) y - Re x(0) Re y(0): the DoubleMatrix proxy
        gemm('t','n',2.0) + ger(-1.0) pattern (src/SlaterDet.cpp:809-813)."""
        m = 2.0 * (x.conj() @ y.T).real
        m -= np.outer(x[:, self.g0].real, y[:, self.g0].real)
        return m

    def cleanup(self):
        """src/SlaterDet.cpp:1341-1356: Im c(G=0) = 0."""
        self.c[:, self.g0] = self.c[:, self.g0].real

    def gram(self):
        """src/SlaterDet.cpp:480-534: S = 2C^T C - c0 c0^T, S = L L^T,
        C <- C L^-T."""
        self.cleanup()
        s = self.real_dot(self.c, self.c)
        L = np.linalg.cholesky(s)
        self.c = np.linalg.solve(L, self.c)

    def ortho_align(self, c_last):
        """src/SlaterDet.cpp:768-876."""
        self.cleanup()
        ctmp = self.c.copy()
        L = np.linalg.cholesky(self.real_dot(self.c, self.c))
        x = self.real_dot(self.c, c_last)           # B = C^T C_last (x2, fix)
        x = np.linalg.solve(L, x)                   # L^-1 B
        x = polar(x, 1.e-6, 20)
        x = np.linalg.solve(L.T, x)                 # L^-T Q
        self.c = x.T @ ctmp                         # C <- C_tmp X

    def lowdin(self):
        """src/SlaterDet.cpp:674-721: S = L L^T, U the orthogonal polar
        factor of L^T, C <- C L^-T U."""
        self.cleanup()
        L = np.linalg.cholesky(self.real_dot(self.c, self.c))
        u = polar(L.T.copy(), 1.e-6, 20)
        t = np.linalg.solve(L.T, u)                 # L^-T U
        self.c = t.T @ self.c

    def align(self, cv):
        """src/SlaterDet.cpp:979-1044, cv.align(self): cv <- cv X with X the
        orthogonal polar factor of B = cv^T C (x2, G=0 fix).  Returns the
        aligned cv."""
        x = polar(self.real_dot(cv, self.c), 1.e-6, 20)
        return x.T @ cv

    def set_positions(self, positions):
        """AtomSet::set_positions followed by EnergyFunctional::atoms_moved
        (src/EnergyFunctional.cpp:1047-1197): structure factors, local
        potential and pseudocharge sums, E_sr and the projector phases."""
        self.positions = [np.array(p, float) for p in positions]
        self._setup_tables()

    # ---- density (src/SlaterDet.cpp:225-298, src/ChargeDensity.cpp:136-198)
    def update_density(self):
        rho = np.zeros(self.N)
        om_inv = 1.0 / self.omega
        n = 0
        while n + 1 < self.nst:
            f = self.wgrid.backward(self.c[n], self.c[n + 1]).ravel()
            rho += om_inv * self.occ[n] * f.real ** 2 + om_inv * self.occ[n + 1] * f.imag ** 2
            n += 2
        if self.nst % 2:
            f = self.wgrid.backward(self.c[-1]).ravel()
            rho += om_inv * self.occ[-1] * f.real ** 2
        self.rhor = rho
        self.total_charge = rho.sum() * self.omega / self.N
        self.rhog = self.vgrid.forward(self.omega * rho)

    def update_rhor(self):
        """ChargeDensity::update_rhor (src/ChargeDensity.cpp:201-240):
        rho(r) = Re FFT_bwd(rho(G)) / Omega from the (mixed) rho(G)."""
        self.rhor = self.vgrid.backward(self.rhog).real.ravel() / self.omega
        self.total_charge = self.rhor.sum() * self.omega / self.N

    # ---- potentials (src/EnergyFunctional.cpp:231-394, XCPotential:124-465)
    def update_vhxc(self):
        vb, om = self.vb, self.omega
        rhoelg = self.rhog / om
        self.rhoelg = rhoelg
        rho = self.rhor
        if self.xc == "LDA":
            e, v = lda_pz(rho)
            vxc = v
            self.exc = (rho * e).sum() * om / self.N
            self.xc_parts = (e, v, None, None)
        else:
            grads = []
            for j in range(3):
                t = 1j * vb.gx[:, j] / om * self.rhog
                grads.append(self.vgrid.backward(t).real.ravel())
            grad = np.sqrt(grads[0] ** 2 + grads[1] ** 2 + grads[2] ** 2)
            e, v1, v2 = pbe(rho, grad)
            vxt = np.zeros(self.N)
            for j in range(3):
                t = self.vgrid.forward(grads[j] * v2)
                t = t * (1j * vb.gx[:, j])
                vxt += self.vgrid.backward(t).real.ravel()
            vxc = v1 + vxt
            self.exc = (rho * e).sum() * om / self.N
            self.xc_parts = (e, v1, v2, grads)
        # dxc = sum rho (e_xc - v_xc) Omega / N (src/XCPotential.cpp:199-229, 376-423)
        self.dxc = (rho * (e - vxc)).sum() * om / self.N
        g0 = vb.g0()
        eps = 2.0 * (np.conj(rhoelg) * self.vion_g).real.sum()
        eps -= (np.conj(rhoelg[g0]) * self.vion_g[g0]).real
        self.eps = eps * om
        rt = rhoelg + self.rhops_t
        self.rhogt = rt
        self.ehart = om * FPI * (np.abs(rt) ** 2 * vb.g2i).sum()
        # electronic and pseudocharge parts (src/EnergyFunctional.cpp:320-351)
        self.ehart_e = om * FPI * (np.abs(rhoelg) ** 2 * vb.g2i).sum()
        self.ehart_p = om * FPI * (np.abs(self.rhops_t) ** 2 * vb.g2i).sum()
        vloc_g = self.vion_g + FPI * rt * vb.g2i
        self.v_r = vxc + self.vgrid.backward(vloc_g).real.ravel()

    # ---- nonlocal (src/NonLocalPotential.cpp:1258-1640)
    def nonlocal_energy(self, hc: Optional[np.ndarray], forces=False):
        enl = 0.0
        om_inv = 1.0 / self.omega
        fion = [np.zeros_like(p) for p in self.positions]
        for isp, tw, lp, dfac in self.nl:
            a = self.anl(isp, tw, lp)                   # (npr, na, ng)
            npr, na, ng = a.shape
            af = a.reshape(npr * na, ng)
            F = self.real_dot(af, self.c)               # (npr*na, nst)
            DF = F * np.repeat(dfac, na)[:, None]
            enl += om_inv * (F * DF * self.occ[None, :]).sum()
            if hc is not None:
                hc += (om_inv * DF).T @ af
            if forces:
                for j in range(3):
                    daf = af * (-1j * self.wb.gx[:, j])[None, :]
                    dF = self.real_dot(daf, self.c)
                    t = (self.occ[None, :] * DF * dF).sum(1).reshape(npr, na)
                    fion[isp][:, j] -= 2.0 * om_inv * t.sum(0)
        return enl, fion

    # ---- energy and H*psi (src/EnergyFunctional.cpp:397-1044)
    def energy(self, compute_hpsi=True, forces=False):
        wb = self.wb
        psi2 = (self.occ[:, None] * np.abs(self.c) ** 2).sum(0)
        self.ekin = (psi2 * wb.g2).sum()
        hc = np.zeros_like(self.c) if compute_hpsi else None
        self.enl, fnl = self.nonlocal_energy(hc, forces)
        self.ecoul = self.ehart + self.esr - self.eself
        self.etotal = self.ekin + self.eps + self.enl + self.ecoul + self.exc
        if compute_hpsi:
            hc += 0.5 * wb.g2[None, :] * self.c
            self.rs_mul_add(self.v_r, hc)
            self.hc = hc
        if forces:
            self.fion = self._local_forces(fnl)
        return self.etotal

    def rs_mul_add(self, v, hc):
        """src/SlaterDet.cpp:410-477: hc += FFT_fwd(v FFT_bwd(c))."""
        n = 0
        while n + 1 < self.nst:
            f = self.wgrid.backward(self.c[n], self.c[n + 1]).ravel() * v
            c1, c2 = self.wgrid.forward(f, two=True)
            hc[n] += c1
            hc[n + 1] += c2
            n += 2
        if self.nst % 2:
            f = self.wgrid.backward(self.c[-1]).ravel() * v
            hc[-1] += self.wgrid.forward(f)

    def _local_forces(self, fnl):
        """src/EnergyFunctional.cpp:841-930."""
        vb = self.vb
        out = []
        for isp, sp in enumerate(self.species):
            vtemp = FPI * self.rhops[isp] * vb.g2i * np.conj(self.rhogt) \
                + self.vps[isp] * np.conj(self.rhoelg)
            tau = self.positions[isp]
            e = np.exp(-1j * (vb.gx @ tau.T))        # (ng, na)
            tmp = e.real * vtemp.imag[:, None] + e.imag * vtemp.real[:, None]
            f_loc = -2.0 * self.omega * (tmp.T @ vb.gx)
            out.append(fnl[isp] + self.fion_esr[isp] + f_loc)
        return out

    # ---- stress tensor (src/EnergyFunctional.cpp:397-1044 with
    # compute_stress, src/XCPotential.cpp:467-640,
    # src/NonLocalPotential.cpp:235-560 dtwnl and :1790-2069)
    def dtwnl(self, isp):
        """Strain derivatives of the projector forms, dt[ipr, ij, G]
        (src/NonLocalPotential.cpp:266-440, Kleinman-Bylander l = 0, 1)."""
        sp = self.species[isp]
        wb = self.wb
        g, gi, gx = wb.g, wb.gi, wb.gx
        s14pi = math.sqrt(1.0 / FPI)
        s34pi = math.sqrt(3.0 / FPI)
        out = []
        for iop, (l, _, _) in enumerate(sp.proj):
            v, dv = sp.vnlg(iop, g)
            if l == 0:
                tmp = gi * s14pi * dv
                out.append(np.array([tmp * gx[:, i] * gx[:, j] for i, j in VOIGT]))
            else:
                y = [s34pi * gx[:, m] * gi for m in range(3)]
                for m in range(3):
                    fac = -y[m] * (v - g * dv) * gi * gi
                    dt = []
                    for i, j in VOIGT:
                        t = fac * gx[:, i] * gx[:, j]
                        if j == m:
                            t = t + v * y[i]
                        dt.append(t)
                    out.append(np.array(dt))
        return np.array(out)                       # (npr, 6, ng)

    def stress(self):
        """sigma (6, Voigt order) and its parts at the current C, after
        update_density, update_vhxc and energy."""
        wb, vb, om = self.wb, self.vb, self.omega
        parts = {}
        # kinetic: (2/Omega) sum_G psi2(G) G_i G_j
        psi2 = (self.occ[:, None] * np.abs(self.c) ** 2).sum(0)
        parts["ekin"] = np.array([2.0 * (psi2 * wb.gx[:, i] * wb.gx[:, j]).sum()
                                  for i, j in VOIGT]) / om
        eye = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
        # local pseudopotential
        dvion = np.zeros(vb.size, complex)
        for isp, sp in enumerate(self.species):
            v, dv = sp.dvlocg(vb.g)
            dvion += self.sfac[isp] * dv / om
        fac = 2.0 * vb.gi * (np.conj(self.rhoelg) * dvion).real
        parts["eps"] = eye * self.eps / om + np.array(
            [(fac * vb.gx[:, i] * vb.gx[:, j]).sum() for i, j in VOIGT])
        # Hartree (with the Gaussian pseudocharges)
        temp = np.abs(self.rhogt) ** 2 * vb.g2i ** 2
        for isp, sp in enumerate(self.species):
            sg = self.sfac[isp]
            temp = temp + 2.0 * 0.25 * RCPS * RCPS * (
                self.rhogt.real * sg.real + self.rhogt.imag * sg.imag) * self.rhops[isp] * vb.g2i
        tsum = np.array([(temp * vb.gx[:, i] * vb.gx[:, j]).sum() for i, j in VOIGT])
        parts["ehart"] = eye * self.ehart / om - 2.0 * FPI * tsum
        # exchange-correlation
        e, v1, v2, grads = self.xc_parts
        rho = self.rhor
        dsum = (rho * (e - v1)).sum()
        if v2 is None:
            parts["exc"] = -eye * dsum / self.N
        else:
            g2 = grads[0] ** 2 + grads[1] ** 2 + grads[2] ** 2
            sx = []
            for i, j in VOIGT:
                t = grads[i] * grads[j] * v2
                if i == j:
                    t = t + g2 * v2
                sx.append(t.sum())
            parts["exc"] = -(eye * dsum + np.array(sx)) / self.N
        # nonlocal
        tsum = np.zeros(6)
        for isp, tw, lp, dfac in self.nl:
            a = self.anl(isp, tw, lp)                 # (npr, na, ng)
            npr, na, ng = a.shape
            F = self.real_dot(a.reshape(npr * na, ng), self.c)
            fnl = F * np.repeat(dfac, na)[:, None] / om
            dt = self.dtwnl(isp)                      # (npr, 6, ng)
            for k in range(6):
                ak = self.anl(isp, dt[:, k, :], lp).reshape(npr * na, ng)
                dF = self.real_dot(ak, self.c)
                tsum[k] += (2.0 * self.occ[None, :] * fnl * dF).sum()
        parts["enl"] = (eye * self.enl + tsum) / om
        # pseudocharge repulsion
        zv = [sp.zval for sp in self.species]
        _, _, parts["esr"] = esr_forces(self.system, zv, self.positions, with_stress=True)
        self.sigma_parts = parts
        self.sigma = sum(parts.values())
        return self.sigma

    def diag(self, eigvec=True):
        """src/Wavefunction.cpp:834-917 (real basis): h = 2 C^T HC - c0 hc0^T,
        eigenvalues by syev; with eigvec C <- C Z and dwf (hc) <- the old
        C.  Returns the eigenvalues."""
        h = self.real_dot(self.c, self.hc)
        w, z = np.linalg.eigh(h)
        if eigvec:
            old = self.c.copy()
            self.c = z.T @ old
            self.hc = old
        return w

    def eigenvalue_sum(self):
        """Wavefunction::dot (src/SlaterDet.cpp:1122-1153)."""
        d = 2.0 * (np.conj(self.c) * self.hc).real.sum()
        d -= (self.c[:, self.g0].real * self.hc[:, self.g0].real).sum()
        return d

    # ---- preconditioner (src/Preconditioner.cpp:88-143, diag :49-85)
    def kdiag(self):
        p2 = np.abs(self.c) ** 2
        snorm = p2.sum(1) - 0.5 * p2[:, self.g0]
        sek = (p2 * self.wb.g2[None, :]).sum(1)
        bn, be = 2.0 * snorm, 2.0 * sek
        ekin = np.where(0.5 * bn > 0.0, 0.5 * be / np.where(bn != 0, bn, 1), 0.0)
        ekin = np.where(ekin == 0.0, 1.0, ekin)
        e = 0.5 * self.wb.g2[None, :]
        with np.errstate(divide="ignore"):
            return np.where(e < ekin[:, None], 0.5 / ekin[:, None], 0.5 / e)

    # ---- JD (src/JDWavefunctionStepper.cpp:47-376, real basis)
    def jd_update(self):
        """Rayleigh-Ritz on span(Y, Z): Y = C, Z = the preconditioned
        residual made orthogonal to Y and orthonormal; a second H*psi on Z;
        C <- the lowest nst eigenvectors of the 2 nst x 2 nst projected H."""
        y, hy = self.c.copy(), self.hc.copy()
        a = self.real_dot(y, hy)
        r = hy - a.T @ y
        z = -self.kdiag() * r
        a = self.real_dot(y, z)
        self.c = z - a.T @ y
        self.gram()
        z = self.c
        self.energy(True)                      # H Z with the current potential
        hz = self.hc
        n = self.nst
        h = np.zeros((2 * n, 2 * n))
        h[:n, :n] = self.real_dot(y, hy)
        h[n:, :n] = self.real_dot(z, hy)
        h[n:, n:] = self.real_dot(z, hz)
        h = np.tril(h) + np.tril(h, -1).T      # syevd('l') reads the lower part
        w, q = np.linalg.eigh(h)
        self.c = q[:n, :n].T @ y + q[n:, :n].T @ z

    # ---- PSDA (src/PSDAWavefunctionStepper.cpp:46-249, Preconditioner)
    def psda_update(self):
        hc = self.hc
        a = self.real_dot(self.c, hc)              # A = C^T HC (x2, fix)
        hc = hc - a.T @ self.c                     # HC - C A
        kdiag = self.kdiag()
        dc = -kdiag * hc
        x = self.c
        if self.extrapolate:
            df = dc - self.dc_last
            av = 2.0 * (dc.real * df.real + dc.imag * df.imag).sum()
            bv = 2.0 * (df.real ** 2 + df.imag ** 2).sum()
            f0, d0 = dc[:, self.g0], df[:, self.g0]
            av -= (f0.real * d0.real + f0.imag * d0.imag).sum()
            bv -= (d0.real ** 2 + d0.imag ** 2).sum()
            theta = -av / bv if bv != 0.0 else 0.0
            if theta < -1.0:
                theta = 0.0
            theta = min(2.0, theta)
            self.theta = theta
            xbar = x + theta * (x - self.c_last)
            fbar = dc + theta * (dc - self.dc_last)
            newc = xbar + fbar
        else:
            self.theta = 0.0
            newc = x + dc
        self.c_last = x.copy()
        self.dc_last = dc
        self.c = newc
        self.ortho_align(self.c_last)
        self.extrapolate = True

    def step(self, forces=False, wf_dyn="PSDA") -> Dict[str, float]:
        self.update_density()
        self.update_vhxc()
        self.energy(True, forces)
        eig = self.eigenvalue_sum()
        out = dict(ekin=self.ekin, eps=self.eps, enl=self.enl,
                   ehart=self.ehart, ecoul=self.ecoul, exc=self.exc,
                   esr=self.esr, eself=self.eself, etotal=self.etotal,
                   eigenvalue_sum=eig)
        if wf_dyn == "JD":
            self.jd_update()
        else:
            self.psda_update()
        return out


class KPoint:
    """One k point off Gamma: the complex basis {G: |k+G|^2 < 2 ecut} over the
    whole sphere (src/Basis.cpp:449-486, update_g :646-690 with kpg), its
    coefficients c[n, ig] in sorted Miller order, the projector forms at k+G
    (src/NonLocalPotential.cpp:235-560 with the basis's kpg, kpgi, kpgx) and
    the PSDA history."""

    def __init__(self, es: "ElectronicStep", k, weight: float, hkl: np.ndarray,
                 c: np.ndarray):
        self.k = np.array(k, float)
        self.weight = float(weight)
        self.hkl = np.asarray(hkl, np.int64)
        b = reciprocal(es.cell)
        self.kpgx = (self.hkl + self.k[None, :]) @ b
        self.kpg2 = (self.kpgx ** 2).sum(1)
        self.kpg = np.sqrt(self.kpg2)
        with np.errstate(divide="ignore"):
            self.kpgi = np.where(self.kpg > 0, 1.0 / np.where(self.kpg > 0, self.kpg, 1), 0.0)
        n0, n1, n2 = es.grid_shape
        h, kk, l = self.hkl[:, 0], self.hkl[:, 1], self.hkl[:, 2]
        self.ip = ((l % n2) * n1 + (kk % n1)) * n0 + (h % n0)
        # the first coefficient of the reference's local basis: rod (0,0)
        # is moved to the front (src/Basis.cpp:587-597), its lowest l first
        on = np.flatnonzero((h == 0) & (kk == 0))
        self.first = int(on[np.argmin(l[on])])
        self.c = np.array(c, complex)
        self.c_last = None
        self.dc_last = None
        s14pi, s34pi = math.sqrt(1.0 / FPI), math.sqrt(3.0 / FPI)
        self.nl = []
        for isp, sp in enumerate(es.species):
            if not sp.proj:
                continue
            tw, lp, dfac = [], [], []
            for iop, (lq, _, _) in enumerate(sp.proj):
                v, dv = sp.vnlg(iop, self.kpg)
                if lq == 0:
                    tw.append(s14pi * v); lp.append(0); dfac.append(sp.dmat[0])
                else:
                    for j in range(3):
                        tw.append(s34pi * self.kpgx[:, j] * self.kpgi * v)
                        lp.append(1); dfac.append(sp.dmat[1])
            self.nl.append((isp, np.array(tw), np.array(lp), np.array(dfac)))


class KPointStep:
    """The electronic step of ElectronicStep on a set of k points off Gamma,
    each a complex SlaterDet (src/SlaterDet.cpp complex branches): one band
    per FFT, C^H C products, k-weighted sums (src/ChargeDensity.cpp:136-198,
    src/EnergyFunctional.cpp:440-560, :700-716, src/Wavefunction.cpp:814-830).
    The density, potentials and the Coulomb and XC energies are the Gamma
    machinery of an ElectronicStep on the same cell and atoms."""

    def __init__(self, system, cs: Optional[List[np.ndarray]] = None):
        self.base = ElectronicStep(system)
        es = self.base
        self.nst = es.nst
        self.occ = es.occ
        self.kpts = []
        for ik, (k, w) in enumerate(system.kpoints):
            hkl = system.kmiller(ik)
            c = system.kcoefficients(ik, hkl) if cs is None else cs[ik]
            self.kpts.append(KPoint(es, k, w, hkl, c))
        self.extrapolate = False
        self.gram()

    # ---- complex SlaterDet operations
    def gram(self):
        """src/SlaterDet.cpp:524-533: S = C^H C = L L^H, C <- C L^-H."""
        for kp in self.kpts:
            L = np.linalg.cholesky(np.conj(kp.c) @ kp.c.T)
            kp.c = np.linalg.solve(np.conj(L), kp.c)

    def ortho_align(self, kp):
        """src/SlaterDet.cpp:877-975: L = chol(C^H C), X = L^-1 C^H C_last,
        X <- unitary polar factor, C <- C L^-H X."""
        L = np.linalg.cholesky(np.conj(kp.c) @ kp.c.T)
        x = np.conj(kp.c) @ kp.c_last.T
        x = np.linalg.solve(L, x)
        x = polar_complex(x, 1.e-6, 20)
        x = np.linalg.solve(np.conj(L).T, x)
        kp.c = x.T @ kp.c

    def _backward(self, kp, c):
        z = np.zeros(self.base.N, complex)
        z[kp.ip] = c
        return np.fft.ifftn(z.reshape(self.base.wgrid.shape)) * self.base.N

    def _forward(self, kp, f):
        return (np.fft.fftn(f.reshape(self.base.wgrid.shape)) / self.base.N).ravel()[kp.ip]

    # ---- density (src/SlaterDet.cpp:280-298 complex branch)
    def update_density(self):
        es = self.base
        rho = np.zeros(es.N)
        for kp in self.kpts:
            for n in range(self.nst):
                f = self._backward(kp, kp.c[n]).ravel()
                rho += kp.weight * self.occ[n] / es.omega * (f.real ** 2 + f.imag ** 2)
        es.rhor = rho
        es.total_charge = rho.sum() * es.omega / es.N
        es.rhog = es.vgrid.forward(es.omega * rho)

    def update_vhxc(self):
        self.base.update_vhxc()

    def anl(self, kp, isp, tw, lp):
        """src/NonLocalPotential.cpp:1316-1394 at k: twnl(k+G) (-i)^l
        exp(-i (k+G).tau)."""
        tau = self.base.positions[isp]
        e = np.exp(-1j * (kp.kpgx @ tau.T)).T
        a = tw[:, None, :] * e[None, :, :]
        a[lp == 1] *= -1j
        return a

    def nonlocal_energy(self, kp, hc):
        """src/NonLocalPotential.cpp:1420-1610, complex branch: F = A^H C,
        E_nl = sum occ D |F|^2 / Omega, HC += A D F / Omega."""
        enl = 0.0
        om_inv = 1.0 / self.base.omega
        for isp, tw, lp, dfac in kp.nl:
            a = self.anl(kp, isp, tw, lp)
            npr, na, ng = a.shape
            af = a.reshape(npr * na, ng)
            F = np.conj(af) @ kp.c.T                    # (npr*na, nst)
            DF = F * np.repeat(dfac, na)[:, None]
            enl += om_inv * (self.occ[None, :] * (F.real * DF.real + F.imag * DF.imag)).sum()
            if hc is not None:
                hc += (om_inv * DF).T @ af
        return enl

    def energy(self, compute_hpsi=True):
        es = self.base
        self.ekin = 0.0
        self.enl = 0.0
        for kp in self.kpts:
            psi2 = (0.5 * self.occ[:, None] * np.abs(kp.c) ** 2).sum(0)
            self.ekin += kp.weight * (psi2 * kp.kpg2).sum()
            hc = np.zeros_like(kp.c) if compute_hpsi else None
            self.enl += kp.weight * self.nonlocal_energy(kp, hc)
            if compute_hpsi:
                hc += 0.5 * kp.kpg2[None, :] * kp.c
                for n in range(self.nst):
                    f = self._backward(kp, kp.c[n]).ravel() * es.v_r
                    hc[n] += self._forward(kp, f)
                kp.hc = hc
        self.eps, self.exc, self.ehart = es.eps, es.exc, es.ehart
        self.esr, self.eself = es.esr, es.eself
        self.ecoul = es.ehart + es.esr - es.eself
        self.etotal = self.ekin + es.eps + self.enl + self.ecoul + es.exc
        return self.etotal

    def eigenvalue_sum(self):
        """Wavefunction::dot (src/Wavefunction.cpp:814-830, complex
        SlaterDet::dot src/SlaterDet.cpp:1149-1152): sum_k w_k Re tr(C^H HC)."""
        return sum(kp.weight * (np.conj(kp.c) * kp.hc).real.sum() for kp in self.kpts)

    def kdiag(self, kp):
        """src/Preconditioner.cpp:88-143 on a complex basis: fac = 1, and the
        reference still removes half of |c|^2 of the first local coefficient
        from the norm (its G = 0 correction, here rod (0,0)'s first)."""
        p2 = np.abs(kp.c) ** 2
        snorm = p2.sum(1) - 0.5 * p2[:, kp.first]
        sek = (p2 * kp.kpg2[None, :]).sum(1)
        ekin = np.where(0.5 * snorm > 0.0, 0.5 * sek / np.where(snorm != 0, snorm, 1), 0.0)
        ekin = np.where(ekin == 0.0, 1.0, ekin)
        e = 0.5 * kp.kpg2[None, :]
        with np.errstate(divide="ignore"):
            return np.where(e < ekin[:, None], 0.5 / ekin[:, None], 0.5 / e)

    def psda_update(self):
        """src/PSDAWavefunctionStepper.cpp:46-249, complex branch, per k point
        (theta of each k point from its own sums)."""
        for kp in self.kpts:
            a = np.conj(kp.c) @ kp.hc.T                # A = C^H HC
            hc = kp.hc - a.T @ kp.c                    # HC - C A
            dc = -self.kdiag(kp) * hc
            x = kp.c
            if self.extrapolate:
                df = dc - kp.dc_last
                av = (dc.real * df.real + dc.imag * df.imag).sum()
                bv = (df.real ** 2 + df.imag ** 2).sum()
                theta = -av / bv if bv != 0.0 else 0.0
                if theta < -1.0:
                    theta = 0.0
                theta = min(2.0, theta)
                kp.theta = theta
                newc = x + theta * (x - kp.c_last) + dc + theta * (dc - kp.dc_last)
            else:
                kp.theta = 0.0
                newc = x + dc
            kp.c_last = x.copy()
            kp.dc_last = dc
            kp.c = newc
            self.ortho_align(kp)
        self.extrapolate = True

    def step(self) -> Dict[str, float]:
        self.update_density()
        self.update_vhxc()
        self.energy(True)
        eig = self.eigenvalue_sum()
        out = dict(ekin=self.ekin, eps=self.eps, enl=self.enl, ehart=self.ehart,
                   ecoul=self.ecoul, exc=self.exc, esr=self.esr, eself=self.eself,
                   etotal=self.etotal, eigenvalue_sum=eig)
        self.psda_update()
        return out


AMU = 1822.89      # atomic mass unit in electron masses, src/IonicStepper.cpp:40


class AndersonMixer:
    """src/AndersonMixer.cpp:28-256 with diag = true, eig_ratio = 0: history
    of nmax+1 (x, f) pairs; theta solves the least-squares system on the
    differences to the newest f through the positive eigenvalues of its
    normal matrix."""

    def __init__(self, m: int, nmax: int):
        self.m, self.nmax = m, nmax
        self.x = [None] * (nmax + 1)
        self.f = [None] * (nmax + 1)
        self.restart()

    def restart(self):
        self.n, self.k = -1, -1

    def update(self, x, f):
        nmax = self.nmax
        self.k = (self.k + 1) % (nmax + 1)
        if self.n < nmax:
            self.n += 1
        k, n = self.k, self.n
        self.x[k] = x.copy()
        self.f[k] = f.copy()
        theta = np.zeros(n)
        if n > 0:
            km = [(k - i + nmax) % (nmax + 1) for i in range(n)]
            d = [self.f[k] - self.f[j] for j in km]
            a = np.array([[d[i] @ d[j] for j in range(n)] for i in range(n)])
            b = np.array([d[i] @ self.f[k] for i in range(n)])
            w, u = np.linalg.eigh(a)
            for kk in range(n):
                if w[kk] > 0.0 * w[n - 1]:
                    theta += (u[:, kk] @ b / w[kk]) * u[:, kk]
        xbar = self.x[k].copy()
        fbar = self.f[k].copy()
        for i in range(n):
            j = (k - i + nmax) % (nmax + 1)
            fbar -= theta[i] * (self.f[k] - self.f[j])
            xbar -= theta[i] * (self.x[k] - self.x[j])
        return xbar, fbar


def scf_run(es: "ElectronicStep", nitscf: int, nite: int, mix_coeff: float = 0.5,
            mix_rcut: float = 10.0, mix_ndim: int = 3, scf_tol: float = 0.0):
    """The SCF loop of BOSampleStepper::step(0) (ground state, atoms fixed,
    src/BOSampleStepper.cpp:781-1114) with wf_dyn = PSDA: nitscf iterations,
    each an update of the density (mixed with the Anderson mixer and the
    Kerker weights when nite > 0, :805-881), of the potentials, and up to
    nite electronic steps (stopping early when the eigenvalue sum moves less
    than 0.01 of the Hartree energy change, :903-980); the Harris-Foulkes
    estimate etotal_int per iteration (:1075-1101).

    Returns {"etotal_int": [...], "eigenvalue_sum": [...], "nite_done": [...]}."""
    vb = es.vb
    g2 = vb.g2
    q1 = 2.0 * math.pi / 3.0                                        # rc1 = 3 (:344-386)
    wls = np.where(g2 != 0.0, np.sqrt(g2 / np.where(g2 != 0.0, g2 + q1 * q1, 1.0)), 1.0)
    if mix_rcut > 0.0:
        q0 = 2.0 * math.pi / mix_rcut
        wk = np.where(g2 != 0.0, g2 / (g2 + q0 * q0), 1.0)         # (:391-407)
    else:
        wk = np.ones_like(g2)
    mixer = AndersonMixer(2 * vb.size, mix_ndim) if mix_ndim > 0 else None
    es.extrapolate = False                                           # preprocess (:785)
    out = {"etotal_int": [], "eigenvalue_sum": [], "nite_done": []}
    rhog_in = None
    ehart = ehart_m = delta_ehart = 0.0
    etotal = etotal_m = etotal_mm = 0.0
    for itscf in range(nitscf):
        es.update_density()
        if nite > 0:
            if itscf == 0:
                rhog_in = es.rhog.copy()
            else:
                drhog = es.rhog - rhog_in
                if mixer is not None:
                    dr = (drhog / wls).view(np.float64)
                    xbar, fbar = mixer.update(rhog_in.view(np.float64).copy(), dr.copy())
                    rhobar = xbar.view(np.complex128)
                    drhobar = fbar.view(np.complex128) * wls
                    rhog_in = rhobar + mix_coeff * drhobar * wk
                else:
                    rhog_in = rhog_in + mix_coeff * drhog * wk
                es.rhog = rhog_in.copy()
                es.update_rhor()
        es.update_vhxc()
        if nite > 0:
            es.extrapolate = False                                   # (:897)
        if itscf == 0:
            ehart = es.ehart
            delta_ehart = 0.0
        elif itscf == 1:
            ehart_m, ehart = ehart, es.ehart
            delta_ehart = abs(ehart - ehart_m)
        else:
            ehart_m, ehart = ehart, es.ehart
            delta_ehart = min(delta_ehart, abs(ehart - ehart_m))
        ite = 0
        conv = False
        eig = eig_m = 0.0
        while not conv and ite < max(nite, 1):
            es.energy(True)
            if ite > 0:
                eig_m = eig
            eig = es.eigenvalue_sum()
            out["eigenvalue_sum"].append(eig)
            es.psda_update()
            if ite > 0:
                conv = abs(eig - eig_m) < 0.01 * delta_ehart
            ite += 1
        out["nite_done"].append(ite)
        eint = 2.0 * eig - es.ehart_e + es.ehart_p + es.esr - es.eself + es.dxc
        out["etotal_int"].append(eint)
        etotal_mm, etotal_m, etotal = etotal_m, etotal, eint
        d = max(abs(etotal - etotal_m), abs(etotal - etotal_mm), abs(etotal_m - etotal_mm))
        if d < scf_tol:
            break
    return out


def md_run(es: "ElectronicStep", niter: int, nitscf: int, dt: float, masses):
    """BOSampleStepper::step(niter) with atoms_dyn = MD, wf_dyn = PSDA,
    nite = 0, no thermostat and the default (linear) wavefunction
    extrapolation (src/BOSampleStepper.cpp:412-1420), with
    MDIonicStepper::compute_r / compute_v (src/MDIonicStepper.cpp:8-30,
    37-253).  masses: per species, in atomic mass units.

    Returns {"ionic": [per ionic step: etotal, ekin_ion, econst, fion],
    "scf": [per electronic step: the step() energies], "positions",
    "velocities", "c", "cv"}."""
    pm = [m * AMU for m in masses]
    nsp = len(es.positions)
    r0 = [p.copy() for p in es.positions]
    v0 = [np.zeros_like(p) for p in r0]
    rm = None
    cv = np.zeros_like(es.c)
    ionic, scf = [], []

    def compute_v(f):
        return [(r0[i] - rm[i]) / dt + dt / (2.0 * pm[i]) * f[i] for i in range(nsp)]

    def ekin_of(v):
        return sum(0.5 * pm[i] * (v[i] ** 2).sum() for i in range(nsp))

    for it in range(niter):
        # energy and forces at r0 with the current wavefunctions (:427-440)
        es.update_density()
        es.update_vhxc()
        es.energy(False, forces=True)
        f = [x.copy() for x in es.fion]
        if it > 0:
            v0 = compute_v(f)                        # (:466-469)
        ek = ekin_of(v0)
        ionic.append(dict(etotal=es.etotal, ekin_ion=ek, econst=es.etotal + ek,
                          fion=np.concatenate(f)))
        # r0 <- r0 + v0 dt + dt^2/(2m) f (:572), then atoms_moved
        rp = [r0[i] + v0[i] * dt + dt * dt / (2.0 * pm[i]) * f[i] for i in range(nsp)]
        rm, r0 = r0, rp
        es.set_positions(r0)
        # wavefunction extrapolation (:593-780, normal extrapolation)
        x = es.c.copy()
        if it == 0:
            es.c = x + dt * cv
            cv = x
            es.gram()
        else:
            cv = es.align(cv)
            es.c = 2.0 * x - cv
            cv = x
            es.lowdin()
        es.extrapolate = False                       # wf_stepper->preprocess()
        for _ in range(nitscf):
            scf.append(es.step())
    # wavefunction velocity and the forces at the last positions (:1351-1420)
    cv = es.align(cv)
    cv = (es.c - cv) / dt
    es.gram()
    es.update_density()
    es.update_vhxc()
    es.energy(False, forces=True)
    v0 = compute_v([x.copy() for x in es.fion])
    return dict(ionic=ionic, scf=scf, positions=r0, velocities=v0, c=es.c.copy(), cv=cv)


def polar(x, tol, maxiter):
    """src/Matrix.cpp:2446-2540: Bjorck-Bowie iteration while
    ||I - X^T X||_F < 1, else the Higham step X <- (X + X^-T)/2."""
    n = x.shape[0]
    eye = np.eye(n)
    for _ in range(maxiter):
        q = eye - x.T @ x
        qn = math.sqrt((q * q).sum())
        if qn < 1.0:
            t = eye + 0.75 * q
            qt = q @ t
            t = eye + 0.5 * qt
            x = x @ t
        else:
            x = 0.5 * (x + np.linalg.inv(x.T))
        if qn <= tol:      # the update above still runs on the last pass
            break
    return x


def polar_complex(x, tol, maxiter):
    """ComplexMatrix::polar (src/Matrix.cpp:2524-2595): Bjorck-Bowie while
    ||I - X^H X||_F < 1, else the Higham step X <- (X + X^-H)/2.  (The
    reference's serial ComplexMatrix::transpose leaves the diagonal
    unconjugated, src/Matrix.cpp:1182-1190; the ScaLAPACK build's pztranc
    conjugates it; this follows the latter.)"""
    n = x.shape[0]
    eye = np.eye(n)
    for _ in range(maxiter):
        q = eye - np.conj(x).T @ x
        qn = math.sqrt((np.abs(q) ** 2).sum())
        if qn < 1.0:
            t = eye + 0.75 * q
            qt = q @ t
            t = eye + 0.5 * qt
            x = x @ t
        else:
            x = 0.5 * (x + np.linalg.inv(np.conj(x).T))
        if qn <= tol:
            break
    return x
