"""Seeded synthetic Kohn-Sham systems (cells, species, atoms, coefficients).

These are the workloads the electronic step is measured and checked on:

* ``si8``     - 8-atom diamond cubic cell a=10.26 bohr, 20 Ry, 16 bands, LDA,
                coefficient seed 1.
* ``si64``    - 2x2x2 supercell (a=20.52), atoms displaced by U(-0.05,0.05)
                bohr (seed 2), 30 Ry, 128 bands, PBE.
* ``h2o32``   - 32 water-like molecules in an 18.6 bohr cell (seed 4), 70 Ry,
                128 bands, PBE.
* ``si512``   - 4x4x4 supercell (a=41.04), displaced (seed 5), 25 Ry,
                1024 bands, PBE.
* ``batch``   - random cubic cells L in [10,20] bohr with 8-64 Si-like atoms at
                >= 3.5 bohr separation (seed 3), ecut in [20,30] Ry, bands =
                2 x atoms, LDA.

Species are norm-conserving semilocal pseudopotentials (the SLPP form read by
the reference's src/SpeciesHandler.cpp:120-248 and initialised by
src/Species.cpp:510-1055) tabulated on a 0.01-bohr radial mesh to 10 bohr:
local potential -Z erf(r/rc)/r (+ optional Gaussian), projectors
r^l exp(-(r/w)^2), one per l, with a diagonal D matrix.

Coefficients are complex N(0,1) drawn from ``numpy.random.default_rng(seed)``
over the Gamma-point half sphere of Miller indices in sorted (h,k,l) order, so
that any implementation can map them onto its own basis order by Miller index.
Units are Hartree atomic units; ``ecut_ry`` is in Rydberg as in the reference's
``set ecut`` command (src/Ecut.h:40-50).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class SpeciesDef:
    name: str
    zval: int
    mass: float
    rc_loc: float                 # local potential -Z erf(r/rc_loc)/r
    gauss_amp: float = 0.0        # + gauss_amp * exp(-(r/gauss_w)^2)
    gauss_w: float = 1.0
    proj_w: Optional[float] = None  # projector width (None: local only)
    d_s: float = 0.0
    d_p: float = 0.0
    atomic_number: int = 14
    mesh_spacing: float = 0.01
    mesh_size: int = 1001

    def radial_mesh(self) -> np.ndarray:
        return np.arange(self.mesh_size) * self.mesh_spacing

    def local_potential(self) -> np.ndarray:
        r = self.radial_mesh()
        v = np.empty_like(r)
        z = float(self.zval)
        v[0] = -2.0 * z / (self.rc_loc * math.sqrt(math.pi))
        v[1:] = -z * np.array([math.erf(x / self.rc_loc) for x in r[1:]]) / r[1:]
        if self.gauss_amp != 0.0:
            v += self.gauss_amp * np.exp(-(r / self.gauss_w) ** 2)
        return v

    def projectors(self):
        """List of (l, radial array) pairs, one projector per l."""
        if self.proj_w is None:
            return []
        r = self.radial_mesh()
        g = np.exp(-(r / self.proj_w) ** 2)
        return [(0, g.copy()), (1, r * g)]

    def dmatrix(self):
        if self.proj_w is None:
            return []
        return [(0, self.d_s), (1, self.d_p)]


SI = SpeciesDef("Si", 4, 28.0855, rc_loc=0.5, gauss_amp=1.2, gauss_w=0.9,
                proj_w=1.0, d_s=2.0, d_p=-1.0, atomic_number=14)
O = SpeciesDef("O", 6, 15.9994, rc_loc=0.4, proj_w=0.7, d_s=3.0, d_p=-1.5,
               atomic_number=8)
H = SpeciesDef("H", 1, 1.00794, rc_loc=0.3, atomic_number=1)


@dataclasses.dataclass
class System:
    name: str
    cell: np.ndarray              # 3x3, rows are a0, a1, a2 (bohr)
    species: List[SpeciesDef]
    atoms: List[tuple]            # (species index, np.array([x,y,z]))
    ecut_ry: float
    nbands: int
    xc: str
    seed: int
    nel_override: Optional[int] = None   # electrons when not the ions' total
    # k points (units of the reciprocal vectors) and weights; None = Gamma
    kpoints: Optional[List[tuple]] = None

    @property
    def ecut(self) -> float:      # Hartree
        return 0.5 * self.ecut_ry

    @property
    def nel(self) -> int:
        if self.nel_override is not None:
            return self.nel_override
        return sum(self.species[i].zval for i, _ in self.atoms)

    def band_sample(self, nbands: int) -> "System":
        """Same cell, atoms and cutoff with only nbands doubly occupied
        bands (a bounded timing sample of the full system)."""
        return dataclasses.replace(self, nbands=nbands, nel_override=2 * nbands,
                                   name=f"{self.name}_b{nbands}")

    def positions(self, isp: int) -> np.ndarray:
        return np.array([p for i, p in self.atoms if i == isp]).reshape(-1, 3)

    def miller(self) -> np.ndarray:
        return gamma_miller(self.cell, self.ecut)

    def kmiller(self, ik: int) -> np.ndarray:
        return kpoint_miller(self.cell, self.ecut, self.kpoints[ik][0])

    def kcoefficients(self, ik: int, hkl: Optional[np.ndarray] = None) -> np.ndarray:
        """(nbands, ngw_k) complex128 for k point ik, keyed by its sorted
        Miller list (no constraint at G = 0: the basis is complex)."""
        if hkl is None:
            hkl = self.kmiller(ik)
        rng = np.random.default_rng(1000 * self.seed + 7 + ik)
        ngw = hkl.shape[0]
        return rng.standard_normal((self.nbands, ngw)) \
            + 1j * rng.standard_normal((self.nbands, ngw))

    def with_kpoints(self, kpoints, name: Optional[str] = None) -> "System":
        return dataclasses.replace(self, kpoints=[(tuple(map(float, k)), float(w))
                                                  for k, w in kpoints],
                                   name=name or f"{self.name}_k{len(kpoints)}")

    def coefficients(self, hkl: Optional[np.ndarray] = None) -> np.ndarray:
        """(nbands, ngw) complex128, keyed by the sorted Miller list."""
        if hkl is None:
            hkl = self.miller()
        rng = np.random.default_rng(self.seed)
        ngw = hkl.shape[0]
        c = rng.standard_normal((self.nbands, ngw)) \
            + 1j * rng.standard_normal((self.nbands, ngw))
        g0 = np.flatnonzero((hkl == 0).all(axis=1))
        c[:, g0] = c[:, g0].real
        return c


def reciprocal(cell: np.ndarray) -> np.ndarray:
    """Rows b0,b1,b2 with a_i . b_j = 2 pi delta_ij."""
    return 2.0 * math.pi * np.linalg.inv(cell).T


def gamma_miller(cell: np.ndarray, ecut: float) -> np.ndarray:
    """Sorted (h,k,l) of the Gamma half sphere {G: |G|^2 < 2 ecut}.

    The half sphere is (0,0,l>=0), (0,k>0,l), (h>0,k,l), the set of rods that
    the reference's src/Basis.cpp:357-447 builds for a real basis.
    """
    b = reciprocal(cell)
    fac = math.sqrt(2.0 * ecut) / (2.0 * math.pi)
    hmax = int(1.5 + fac * np.linalg.norm(cell[0]))
    kmax = int(1.5 + fac * np.linalg.norm(cell[1]))
    lmax = int(1.5 + fac * np.linalg.norm(cell[2]))
    h, k, l = np.meshgrid(np.arange(0, hmax + 1), np.arange(-kmax, kmax + 1),
                          np.arange(-lmax, lmax + 1), indexing="ij")
    h, k, l = h.ravel(), k.ravel(), l.ravel()
    half = (h > 0) | ((h == 0) & (k > 0)) | ((h == 0) & (k == 0) & (l >= 0))
    h, k, l = h[half], k[half], l[half]
    gx = h * b[0, 0] + k * b[1, 0] + l * b[2, 0]
    gy = h * b[0, 1] + k * b[1, 1] + l * b[2, 1]
    gz = h * b[0, 2] + k * b[1, 2] + l * b[2, 2]
    inside = gx * gx + gy * gy + gz * gz < 2.0 * ecut
    hkl = np.stack([h[inside], k[inside], l[inside]], axis=1).astype(np.int32)
    order = np.lexsort((hkl[:, 2], hkl[:, 1], hkl[:, 0]))
    return np.ascontiguousarray(hkl[order])


def kpoint_miller(cell: np.ndarray, ecut: float, kpoint) -> np.ndarray:
    """Sorted (h,k,l) of the complex basis at k: {G: |k+G|^2 < 2 ecut} over
    the whole sphere (the rod set of src/Basis.cpp:449-486)."""
    b = reciprocal(cell)
    fac = math.sqrt(2.0 * ecut) / (2.0 * math.pi)
    m = [int(1.5 + fac * np.linalg.norm(cell[i])) for i in range(3)]
    h, k, l = np.meshgrid(np.arange(-m[0], m[0] + 1), np.arange(-m[1], m[1] + 1),
                          np.arange(-m[2], m[2] + 1), indexing="ij")
    q = np.stack([h.ravel() + kpoint[0], k.ravel() + kpoint[1], l.ravel() + kpoint[2]], 1) @ b
    inside = (q * q).sum(1) < 2.0 * ecut
    hkl = np.stack([h.ravel()[inside], k.ravel()[inside], l.ravel()[inside]], 1).astype(np.int32)
    order = np.lexsort((hkl[:, 2], hkl[:, 1], hkl[:, 0]))
    return np.ascontiguousarray(hkl[order])


DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                    [.25, .25, .25], [.25, .75, .75], [.75, .25, .75],
                    [.75, .75, .25]])


def diamond_supercell(a0: float, n: int, displace: float, seed: int):
    pos = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                for f in DIAMOND:
                    pos.append((np.array([i, j, k]) + f) * a0)
    pos = np.array(pos)
    if displace > 0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-displace, displace, size=pos.shape)
    return pos


def si8() -> System:
    a = 10.26
    pos = diamond_supercell(a, 1, 0.0, 1)
    return System("si8", np.eye(3) * a, [SI], [(0, p) for p in pos],
                  20.0, 16, "LDA", 1)


def si64() -> System:
    a = 10.26
    pos = diamond_supercell(a, 2, 0.05, 2)
    return System("si64", np.eye(3) * 2 * a, [SI], [(0, p) for p in pos],
                  30.0, 128, "PBE", 2)


def si512() -> System:
    a = 10.26
    pos = diamond_supercell(a, 4, 0.05, 5)
    return System("si512", np.eye(3) * 4 * a, [SI], [(0, p) for p in pos],
                  25.0, 1024, "PBE", 5)


def _random_rotation(rng) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _min_image_dist(d: np.ndarray, L: float) -> np.ndarray:
    d = d - L * np.round(d / L)
    return np.sqrt((d * d).sum(axis=-1))


def h2o32(nmol: int = 32, L: float = 18.6, seed: int = 4,
          ecut_ry: float = 70.0, nbands: int = 128) -> System:
    rng = np.random.default_rng(seed)
    roh, ang = 1.81, math.radians(104.5)
    local = np.array([[roh * math.sin(ang / 2), 0, roh * math.cos(ang / 2)],
                      [-roh * math.sin(ang / 2), 0, roh * math.cos(ang / 2)]])
    oxy: List[np.ndarray] = []
    atoms = []
    tries = 0
    while len(oxy) < nmol:
        tries += 1
        if tries > 200000:
            raise RuntimeError("cannot place molecules")
        p = rng.uniform(0, L, 3)
        if oxy and _min_image_dist(np.array(oxy) - p, L).min() < 4.5:
            continue
        oxy.append(p)
        R = _random_rotation(rng)
        atoms.append((0, p))
        for h in local:
            atoms.append((1, p + R @ h))
    atoms.sort(key=lambda t: t[0])
    return System("h2o32", np.eye(3) * L, [O, H], atoms, ecut_ry, nbands,
                  "PBE", seed)


def batch(nsys: int = 32, seed: int = 3) -> List[System]:
    rng = np.random.default_rng(seed)
    out = []
    for isys in range(nsys):
        L = rng.uniform(10.0, 20.0)
        nat_target = int(rng.integers(8, 65))
        pos: List[np.ndarray] = []
        tries = 0
        while len(pos) < nat_target and tries < 20000:
            tries += 1
            p = rng.uniform(0, L, 3)
            if pos and _min_image_dist(np.array(pos) - p, L).min() < 3.5:
                continue
            pos.append(p)
        ecut_ry = float(rng.uniform(20.0, 30.0))
        out.append(System(f"batch{isys}", np.eye(3) * L, [SI],
                          [(0, p) for p in pos], ecut_ry, 2 * len(pos), "LDA",
                          1000 + isys))
    return out


def si8k2() -> System:
    """si8 at two k points off Gamma (complex bases), LDA."""
    return si8().with_kpoints([((0.25, 0.25, 0.25), 0.5), ((-0.25, 0.25, 0.25), 0.5)],
                              "si8k2")


def h2o4k2() -> System:
    """Four water molecules at two k points, PBE, two species."""
    return h2o32(nmol=4, L=9.0, seed=9, ecut_ry=40.0, nbands=16).with_kpoints(
        [((0.0, 0.5, 0.0), 0.5), ((0.25, 0.0, 0.5), 0.5)], "h2o4k2")


def si64k2() -> System:
    """si64 (PBE, 30 Ry, 128 bands) at two k points off Gamma."""
    return si64().with_kpoints([((0.25, 0.25, 0.25), 0.5), ((-0.25, 0.25, 0.25), 0.5)],
                               "si64k2")


REGISTRY = {"si8": si8, "si64": si64, "si512": si512, "h2o32": h2o32,
            "si8k2": si8k2, "h2o4k2": h2o4k2, "si64k2": si64k2}


def get(name: str) -> System:
    return REGISTRY[name]()
