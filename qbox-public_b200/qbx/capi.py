"""ctypes binding of libqbx.so (the C ABI declared in include/qbx.h).

Loading fails loudly when the CUDA library has not been built: there is no
CPU path behind this module.  ``Context`` mirrors the reference's objects on
the electronic-step path (Wavefunction/SlaterDet coefficients,
ChargeDensity::update_density, EnergyFunctional::update_vhxc/energy,
PSDAWavefunctionStepper::update) on one GPU.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqbx.so")

FP64 = 0
MIXED = 1
NENERGY = 12
ENERGY_NAMES = ("ekin", "eps", "enl", "ehart", "ecoul", "exc", "esr", "eself",
                "etotal", "eigenvalue_sum", "total_charge", "theta")

# every entry point of include/qbx.h
SYMBOLS = (
    "qbx_stream_in", "qbx_scf_step_async", "qbx_stream_out", "qbx_stream_wait",
    "qbx_set_kpoints", "qbx_kpoint_basis", "qbx_set_kpoint_coeffs",
    "qbx_get_kpoint_coeffs", "qbx_get_kpoint_hpsi", "qbx_host_kbasis",
    "qbx_version", "qbx_create", "qbx_destroy", "qbx_last_error",
    "qbx_set_precision", "qbx_set_cell", "qbx_basis_sizes", "qbx_basis_miller",
    "qbx_set_coeff_order", "qbx_add_species", "qbx_set_atoms",
    "qbx_set_coeffs", "qbx_get_coeffs", "qbx_set_coeffs_async",
    "qbx_get_coeffs_async", "qbx_gram", "qbx_update_density",
    "qbx_get_density", "qbx_update_vhxc", "qbx_get_vr", "qbx_energy",
    "qbx_get_hpsi", "qbx_eigenvalue_sum", "qbx_psda_update", "qbx_psda_reset",
    "qbx_scf_step", "qbx_ft_backward_pair", "qbx_synchronize",
    "qbx_host_basis", "qbx_host_species_eval", "qbx_host_esr",
    "qbx_profile", "qbx_profile_get", "qbx_launch_count", "qbx_stream",
    "qbx_set_gemm_backend", "qbx_split_gemm_tn", "qbx_density_static",
    "qbx_stress", "qbx_get_stress", "qbx_autotune", "qbx_set_wf_dyn", "qbx_jd_update",
    "qbx_scf_step_batch", "qbx_set_step_graph", "qbx_step_graph_info", "qbx_polar",
    "qbx_move_atoms", "qbx_md_run", "qbx_scf_run", "qbx_write_wavefunction",
    "qbx_read_wavefunction",
    "qbx_ft_create", "qbx_ft_destroy", "qbx_ft_last_error", "qbx_ft_backward",
    "qbx_ft_backward2", "qbx_ft_forward", "qbx_ft_forward2", "qbx_compute_density",
    "qbx_rs_mul_add", "qbx_nonlocal_energy", "qbx_ortho_align", "qbx_dot",
    "qbx_nccl_unique_id", "qbx_set_band_shard", "qbx_shard_pairs", "qbx_diag",
    "qbx_lower_inverse",
)

NCCL_ID_BYTES = 128

_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


class QbxError(RuntimeError):
    pass


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libqbx.so; raises if it is missing (build it with qbx.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise QbxError(f"{path} is not built; run qbox-public_b200/qbx/build.py")
    lib = ctypes.CDLL(path)
    sig = {
        "qbx_version": (_I, []),
        "qbx_create": (_I, [ctypes.POINTER(_P), _I, _I]),
        "qbx_destroy": (None, [_P]),
        "qbx_last_error": (ctypes.c_char_p, [_P]),
        "qbx_set_precision": (_I, [_P, _I]),
        "qbx_set_cell": (_I, [_P, _DP, _D, _I, ctypes.c_char_p]),
        "qbx_basis_sizes": (_I, [_P, _IP, _IP, _IP]),
        "qbx_basis_miller": (_I, [_P, _IP]),
        "qbx_set_coeff_order": (_I, [_P, _IP]),
        "qbx_add_species": (_I, [_P, _I, _D, _I, _DP, _I, _IP, _DP, _DP, _IP]),
        "qbx_set_atoms": (_I, [_P, _IP, _DP]),
        "qbx_set_coeffs": (_I, [_P, _DP]),
        "qbx_get_coeffs": (_I, [_P, _DP]),
        "qbx_set_coeffs_async": (_I, [_P, _DP]),
        "qbx_get_coeffs_async": (_I, [_P, _DP]),
        "qbx_gram": (_I, [_P]),
        "qbx_update_density": (_I, [_P, _DP]),
        "qbx_get_density": (_I, [_P, _DP]),
        "qbx_update_vhxc": (_I, [_P]),
        "qbx_get_vr": (_I, [_P, _DP]),
        "qbx_energy": (_I, [_P, _I, _I, _DP, _DP]),
        "qbx_get_hpsi": (_I, [_P, _DP]),
        "qbx_eigenvalue_sum": (_I, [_P, _DP]),
        "qbx_psda_update": (_I, [_P]),
        "qbx_psda_reset": (_I, [_P]),
        "qbx_scf_step": (_I, [_P, _I, _DP, _DP]),
        "qbx_ft_backward_pair": (_I, [_P, _I, _I, _DP]),
        "qbx_synchronize": (_I, [_P]),
        "qbx_host_basis": (_I, [_DP, _D, _IP, _IP, _IP, _IP]),
        "qbx_host_species_eval": (_I, [_I, _D, _I, _DP, _I, _IP, _DP, _I, _DP,
                                       _DP, _DP, _DP]),
        "qbx_host_esr": (_I, [_DP, _I, _IP, _DP, _DP, _DP, _DP]),
        "qbx_host_kbasis": (_I, [_DP, _D, _DP, _IP, _IP, _IP]),
        "qbx_profile": (_I, [_P, _I]),
        "qbx_profile_get": (_I, [_P, ctypes.c_char_p, _DP, ctypes.POINTER(ctypes.c_long)]),
        "qbx_launch_count": (_I, [_P, ctypes.POINTER(ctypes.c_long)]),
        "qbx_stream": (_P, [_P]),
        "qbx_set_gemm_backend": (_I, [_P, _I]),
        "qbx_split_gemm_tn": (_I, [_P, _I, _I, _I, _DP, _DP, _DP, _I]),
        "qbx_lower_inverse": (_I, [_P, _I, _DP, _DP, _IP]),
        "qbx_density_static": (_I, [_P, ctypes.c_void_p, _I, _DP, ctypes.c_void_p]),
        "qbx_stress": (_I, [_P, _DP, _DP]),
        "qbx_autotune": (_I, [_P, ctypes.c_char_p, _I]),
        "qbx_set_wf_dyn": (_I, [_P, ctypes.c_char_p]),
        "qbx_scf_step_batch": (_I, [ctypes.POINTER(_P), _I, _I, _DP]),
        "qbx_jd_update": (_I, [_P]),
        "qbx_get_stress": (_I, [_P, _DP, _DP]),
        "qbx_set_step_graph": (_I, [_P, _I]),
        "qbx_move_atoms": (_I, [_P, _DP]),
        "qbx_write_wavefunction": (_I, [_P, ctypes.c_char_p]),
        "qbx_read_wavefunction": (_I, [_P, ctypes.c_char_p]),
        "qbx_scf_run": (_I, [_P, _I, _I, _D, _D, _I, _D, _DP, _DP, _IP, _IP]),
        "qbx_md_run": (_I, [_P, _I, _I, _D, _DP, _DP, _DP, _DP, _DP]),
        "qbx_polar": (_I, [_P, _DP, _D, _I, _I, ctypes.POINTER(_I)]),
        "qbx_stream_in": (_I, [_P, _DP]),
        "qbx_scf_step_async": (_I, [_P]),
        "qbx_stream_out": (_I, [_P, _DP]),
        "qbx_stream_wait": (_I, [_P, _DP]),
        "qbx_set_kpoints": (_I, [_P, _I, _DP, _DP]),
        "qbx_kpoint_basis": (_I, [_P, _I, _IP, _IP]),
        "qbx_set_kpoint_coeffs": (_I, [_P, _I, _DP]),
        "qbx_get_kpoint_coeffs": (_I, [_P, _I, _DP]),
        "qbx_get_kpoint_hpsi": (_I, [_P, _I, _DP]),
        "qbx_step_graph_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_long),
                                     ctypes.POINTER(ctypes.c_long), ctypes.c_char_p, _I]),
        "qbx_ft_create": (_I, [ctypes.POINTER(_P), _I, _I, _IP, _I, _I, _I, _I]),
        "qbx_ft_destroy": (None, [_P]),
        "qbx_ft_last_error": (ctypes.c_char_p, [_P]),
        "qbx_ft_backward": (_I, [_P, _DP, _DP]),
        "qbx_ft_backward2": (_I, [_P, _DP, _DP, _DP]),
        "qbx_ft_forward": (_I, [_P, _DP, _DP]),
        "qbx_ft_forward2": (_I, [_P, _DP, _DP, _DP]),
        "qbx_compute_density": (_I, [_P, _D, _DP]),
        "qbx_rs_mul_add": (_I, [_P, _DP, _DP]),
        "qbx_nonlocal_energy": (_I, [_P, _I, _DP, _I, _DP, _I, _DP, _DP]),
        "qbx_ortho_align": (_I, [_P, _DP]),
        "qbx_dot": (_I, [_P, _DP, _DP]),
        "qbx_nccl_unique_id": (_I, [ctypes.c_char_p]),
        "qbx_set_band_shard": (_I, [_P, _I, _I, ctypes.c_char_p]),
        "qbx_shard_pairs": (_I, [_I, _I, _I, _IP, _IP]),
        "qbx_diag": (_I, [_P, _I, _DP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def _ip(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_IP)


class Context:
    """One Gamma-point Slater determinant and its Hamiltonian on one GPU."""

    def __init__(self, device: int = 0, precision: int = FP64):
        self.lib = load()
        h = _P()
        rc = self.lib.qbx_create(ctypes.byref(h), device, precision)
        if rc:
            raise QbxError(f"qbx_create failed with code {rc}")
        self.h = h
        self.precision = precision
        self.natoms = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.qbx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc: int, what: str):
        if rc:
            msg = self.lib.qbx_last_error(self.h)
            raise QbxError(f"{what}: code {rc}: {msg.decode() if msg else ''}")

    # ---- setup
    def set_cell(self, cell, ecut: float, nst: int, xc: str = "LDA"):
        a = np.ascontiguousarray(np.asarray(cell, float).ravel())
        self._ok(self.lib.qbx_set_cell(self.h, _dp(a), float(ecut), int(nst),
                                       xc.encode()), "set_cell")
        self.nst = nst
        ngw, ngv = _I(), _I()
        npg = (ctypes.c_int * 3)()
        self._ok(self.lib.qbx_basis_sizes(self.h, ctypes.byref(ngw),
                                          ctypes.byref(ngv), npg), "basis_sizes")
        self.ngw, self.ngv = ngw.value, ngv.value
        self.grid = (npg[0], npg[1], npg[2])

    def set_precision(self, precision: int):
        self._ok(self.lib.qbx_set_precision(self.h, precision), "set_precision")
        self.precision = precision

    def miller(self) -> np.ndarray:
        out = np.empty((self.ngw, 3), np.int32)
        self._ok(self.lib.qbx_basis_miller(self.h, _ip(out)), "basis_miller")
        return out

    def set_coeff_order(self, hkl: Optional[np.ndarray]):
        a = None if hkl is None else np.ascontiguousarray(hkl, np.int32)
        self._ok(self.lib.qbx_set_coeff_order(self.h, _ip(a)), "set_coeff_order")

    def add_species(self, zval, mesh_spacing, vlocal, projectors: Sequence, dmat):
        v = np.ascontiguousarray(vlocal, float)
        nproj = len(projectors)
        pl = np.array([l for l, _ in projectors], np.int32)
        pr = (np.ascontiguousarray(np.stack([p for _, p in projectors]), float)
              if nproj else np.zeros(1))
        dm = np.ascontiguousarray(np.array(dmat, float) if nproj else np.zeros(1))
        isp = _I()
        self._ok(self.lib.qbx_add_species(self.h, int(zval), float(mesh_spacing),
                                          v.size, _dp(v), nproj,
                                          _ip(pl) if nproj else None, _dp(pr),
                                          _dp(dm), ctypes.byref(isp)), "add_species")
        return isp.value

    def set_atoms(self, counts: Sequence[int], tau: np.ndarray):
        na = np.ascontiguousarray(np.array(counts, np.int32))
        t = np.ascontiguousarray(np.asarray(tau, float).reshape(-1))
        self._ok(self.lib.qbx_set_atoms(self.h, _ip(na), _dp(t)), "set_atoms")
        self.natoms = int(na.sum())

    # ---- coefficients
    def set_coeffs(self, c: np.ndarray):
        a = np.ascontiguousarray(c, np.complex128).view(np.float64)
        self._ok(self.lib.qbx_set_coeffs(self.h, _dp(a)), "set_coeffs")

    def get_coeffs(self) -> np.ndarray:
        out = np.empty((self.nst, self.ngw), np.complex128)
        self._ok(self.lib.qbx_get_coeffs(self.h, _dp(out.view(np.float64))), "get_coeffs")
        return out

    def get_hpsi(self) -> np.ndarray:
        out = np.empty((self.nst, self.ngw), np.complex128)
        self._ok(self.lib.qbx_get_hpsi(self.h, _dp(out.view(np.float64))), "get_hpsi")
        return out

    # ---- streamed SlaterDet: pinned host buffers, copies overlapping compute
    def stream_in(self, c_pinned: np.ndarray):
        """Enqueue the upload of a step's input (complex coefficients as a
        pinned float64 buffer); returns at once."""
        self._ok(self.lib.qbx_stream_in(self.h, _dp(c_pinned)), "stream_in")

    def scf_step_async(self):
        self._ok(self.lib.qbx_scf_step_async(self.h), "scf_step_async")

    def stream_out(self, c_pinned: np.ndarray):
        self._ok(self.lib.qbx_stream_out(self.h, _dp(c_pinned)), "stream_out")

    def stream_wait(self):
        e = np.zeros(NENERGY)
        self._ok(self.lib.qbx_stream_wait(self.h, _dp(e)), "stream_wait")
        return dict(zip(ENERGY_NAMES, e))

    # ---- k points off Gamma (complex bases)
    def set_kpoints(self, kpoints, weights):
        """Wavefunction::add_kpoint for each k point (units of the
        reciprocal vectors), the Gamma point removed; [] returns to Gamma."""
        k = np.ascontiguousarray(np.asarray(kpoints, float).reshape(-1))
        w = np.ascontiguousarray(np.asarray(weights, float).reshape(-1))
        nk = w.size
        self._ok(self.lib.qbx_set_kpoints(self.h, nk, _dp(k) if nk else None,
                                          _dp(w) if nk else None), "set_kpoints")
        self.kngw = []
        for ik in range(nk):
            n = _I()
            self._ok(self.lib.qbx_kpoint_basis(self.h, ik, ctypes.byref(n), None), "kpoint_basis")
            self.kngw.append(n.value)

    def kpoint_miller(self, ik: int) -> np.ndarray:
        out = np.empty((self.kngw[ik], 3), np.int32)
        self._ok(self.lib.qbx_kpoint_basis(self.h, ik, None, _ip(out)), "kpoint_basis")
        return out

    def set_kpoint_coeffs(self, ik: int, c: np.ndarray):
        a = np.ascontiguousarray(c, np.complex128).view(np.float64)
        self._ok(self.lib.qbx_set_kpoint_coeffs(self.h, ik, _dp(a)), "set_kpoint_coeffs")

    def get_kpoint_coeffs(self, ik: int) -> np.ndarray:
        out = np.empty((self.nst, self.kngw[ik]), np.complex128)
        self._ok(self.lib.qbx_get_kpoint_coeffs(self.h, ik, _dp(out.view(np.float64))),
                 "get_kpoint_coeffs")
        return out

    def get_kpoint_hpsi(self, ik: int) -> np.ndarray:
        out = np.empty((self.nst, self.kngw[ik]), np.complex128)
        self._ok(self.lib.qbx_get_kpoint_hpsi(self.h, ik, _dp(out.view(np.float64))),
                 "get_kpoint_hpsi")
        return out

    # ---- operations
    def gram(self):
        self._ok(self.lib.qbx_gram(self.h), "gram")

    def update_density(self) -> float:
        q = _D()
        self._ok(self.lib.qbx_update_density(self.h, ctypes.byref(q)), "update_density")
        return q.value

    def density(self) -> np.ndarray:
        out = np.empty(self.grid[0] * self.grid[1] * self.grid[2])
        self._ok(self.lib.qbx_get_density(self.h, _dp(out)), "get_density")
        return out

    def update_vhxc(self):
        self._ok(self.lib.qbx_update_vhxc(self.h), "update_vhxc")

    def vr(self) -> np.ndarray:
        out = np.empty(self.grid[0] * self.grid[1] * self.grid[2])
        self._ok(self.lib.qbx_get_vr(self.h, _dp(out)), "get_vr")
        return out

    def energy(self, hpsi=True, forces=False):
        e = np.zeros(NENERGY)
        f = np.zeros(3 * max(1, self.natoms)) if forces else None
        self._ok(self.lib.qbx_energy(self.h, int(hpsi), int(forces), _dp(e), _dp(f)),
                 "energy")
        out = dict(zip(ENERGY_NAMES, e))
        if forces:
            out["fion"] = f[:3 * self.natoms].reshape(-1, 3)
        return out

    def eigenvalue_sum(self) -> float:
        v = _D()
        self._ok(self.lib.qbx_eigenvalue_sum(self.h, ctypes.byref(v)), "eigenvalue_sum")
        return v.value

    def psda_update(self):
        self._ok(self.lib.qbx_psda_update(self.h), "psda_update")

    def psda_reset(self):
        self._ok(self.lib.qbx_psda_reset(self.h), "psda_reset")

    def scf_step(self, forces=False, stress=False):
        e = np.zeros(NENERGY)
        f = np.zeros(3 * max(1, self.natoms)) if forces else None
        flags = (1 if forces else 0) | (2 if stress else 0)
        self._ok(self.lib.qbx_scf_step(self.h, flags, _dp(e), _dp(f)), "scf_step")
        out = dict(zip(ENERGY_NAMES, e))
        if forces:
            out["fion"] = f[:3 * self.natoms].reshape(-1, 3)
        if stress:
            out["sigma"], out["sigma_parts"] = self.last_stress()
        return out

    def ft_backward_pair(self, n1: int, n2: int) -> np.ndarray:
        n = self.grid[0] * self.grid[1] * self.grid[2]
        out = np.empty(n, np.complex128)
        self._ok(self.lib.qbx_ft_backward_pair(self.h, n1, n2, _dp(out.view(np.float64))),
                 "ft_backward_pair")
        return out.reshape(self.grid[2], self.grid[1], self.grid[0])

    def synchronize(self):
        self._ok(self.lib.qbx_synchronize(self.h), "synchronize")

    # ---- timing
    def profile(self, on: bool = True):
        self._ok(self.lib.qbx_profile(self.h, int(on)), "profile")

    def profile_get(self, name: str):
        ms = _D()
        n = ctypes.c_long()
        self._ok(self.lib.qbx_profile_get(self.h, name.encode(), ctypes.byref(ms),
                                          ctypes.byref(n)), "profile_get")
        return ms.value, n.value

    def launch_count(self) -> int:
        n = ctypes.c_long()
        self._ok(self.lib.qbx_launch_count(self.h, ctypes.byref(n)), "launch_count")
        return n.value

    def set_gemm_backend(self, backend: int):
        self._ok(self.lib.qbx_set_gemm_backend(self.h, backend), "set_gemm_backend")

    def split_gemm_tn(self, a: np.ndarray, b: np.ndarray, backend: int) -> np.ndarray:
        """A^T B through the split-precision product (a: k x m, b: k x n)."""
        k, m = a.shape
        _, n = b.shape
        # column-major k x m is the C-ordered m x k array a.T
        at = np.ascontiguousarray(np.asarray(a, float).T)
        bt = np.ascontiguousarray(np.asarray(b, float).T)
        out = np.empty((n, m))          # column-major m x n
        self._ok(self.lib.qbx_split_gemm_tn(self.h, m, n, k, _dp(at), _dp(bt), _dp(out),
                                            backend), "split_gemm_tn")
        return out.T

    def lower_inverse(self, l: np.ndarray):
        """qbx_lower_inverse: (l^-1, blocked) for a lower-triangular n x n l."""
        n = l.shape[0]
        lt = np.ascontiguousarray(np.asarray(l, float).T)   # column-major
        out = np.empty((n, n))
        blocked = ctypes.c_int(0)
        self._ok(self.lib.qbx_lower_inverse(self.h, n, _dp(lt), _dp(out), ctypes.byref(blocked)),
                 "lower_inverse")
        return out.T, bool(blocked.value)

    def set_wf_dyn(self, name: str):
        """qbx_set_wf_dyn: "PSDA" or "JD" for the update of scf_step."""
        self._ok(self.lib.qbx_set_wf_dyn(self.h, name.encode()), "set_wf_dyn")

    def jd_update(self):
        self._ok(self.lib.qbx_jd_update(self.h), "jd_update")

    def polar(self, x: np.ndarray, tol: float = 1e-6, maxiter: int = 20,
              graph: bool = False):
        """qbx_polar: the polar factor of an nst x nst matrix; returns
        (factor, iterations)."""
        a = np.asfortranarray(np.array(x, dtype=float))
        it = _I()
        self._ok(self.lib.qbx_polar(self.h, _dp(a.reshape(-1, order="F")), tol, maxiter,
                                    int(graph), ctypes.byref(it)), "polar")
        return a, it.value

    def scf_run(self, nitscf: int, nite: int, mix_coeff: float = 0.5, mix_rcut: float = 10.0,
                mix_ndim: int = 3, scf_tol: float = 0.0):
        """qbx_scf_run: the ground-state SCF loop with charge mixing.
        Returns {"etotal_int": (iterations,), "eigenvalue_sum": list per
        electronic step run, "nite_done": (iterations,)}."""
        ns = max(nite, 1)
        eint = np.zeros(nitscf)
        eig = np.zeros(nitscf * ns)
        nd = np.zeros(nitscf, np.int32)
        done = ctypes.c_int()
        self._ok(self.lib.qbx_scf_run(self.h, nitscf, nite, mix_coeff, mix_rcut, mix_ndim,
                                      scf_tol, _dp(eint), _dp(eig), _ip(nd),
                                      ctypes.byref(done)), "scf_run")
        n = done.value
        sums = [eig[i * ns + j] for i in range(n) for j in range(int(nd[i]))]
        return {"etotal_int": eint[:n], "eigenvalue_sum": np.array(sums), "nite_done": nd[:n]}

    def write_wavefunction(self, path: str):
        """qbx_write_wavefunction: the sample file's <wavefunction> element."""
        self._ok(self.lib.qbx_write_wavefunction(self.h, path.encode()), "write_wavefunction")

    def read_wavefunction(self, path: str):
        """qbx_read_wavefunction: coefficients and occupations from a
        sample file's <wavefunction> element."""
        self._ok(self.lib.qbx_read_wavefunction(self.h, path.encode()), "read_wavefunction")

    def move_atoms(self, tau: np.ndarray):
        """qbx_move_atoms: the same atoms at new positions (species-major)."""
        t = np.ascontiguousarray(np.asarray(tau, float).reshape(-1))
        self._ok(self.lib.qbx_move_atoms(self.h, _dp(t)), "move_atoms")

    def md_run(self, niter: int, nitscf: int, dt: float, masses, vel=None):
        """qbx_md_run: niter ionic steps of velocity Verlet MD with nitscf
        electronic steps each.  Returns {"ionic": (niter, 3) etotal,
        ekin_ion, econst; "scf": list of energy dicts; "positions",
        "velocities": (natoms, 3)}."""
        m = np.ascontiguousarray(np.asarray(masses, float))
        v = np.zeros(3 * self.natoms) if vel is None else \
            np.ascontiguousarray(np.asarray(vel, float).reshape(-1)).copy()
        tau = np.zeros(3 * self.natoms)
        ionic = np.zeros(3 * niter)
        scf = np.zeros(max(1, niter * nitscf) * NENERGY)
        self._ok(self.lib.qbx_md_run(self.h, niter, nitscf, dt, _dp(m), _dp(v), _dp(tau),
                                     _dp(ionic), _dp(scf)), "md_run")
        return {"ionic": ionic.reshape(niter, 3),
                "scf": [dict(zip(ENERGY_NAMES, scf[i * NENERGY:(i + 1) * NENERGY]))
                        for i in range(niter * nitscf)],
                "positions": tau.reshape(-1, 3), "velocities": v.reshape(-1, 3)}

    def set_step_graph(self, on: bool = True):
        """qbx_set_step_graph: run scf_step as a captured CUDA graph (from
        the second step of each configuration on)."""
        self._ok(self.lib.qbx_set_step_graph(self.h, int(on)), "set_step_graph")

    def step_graph_info(self):
        """qbx_step_graph_info: (graphs captured, graph launches, note)."""
        n, launches, _, note = self.step_graph_info_full()
        return n, launches, note

    def step_graph_info_full(self):
        """(graphs captured, graph launches, batch graph launches, note)."""
        n = _I()
        launches = ctypes.c_long()
        batch = ctypes.c_long()
        buf = ctypes.create_string_buffer(512)
        self._ok(self.lib.qbx_step_graph_info(self.h, ctypes.byref(n), ctypes.byref(launches),
                                              ctypes.byref(batch), buf, 512), "step_graph_info")
        return n.value, launches.value, batch.value, buf.value.decode()

    def autotune(self) -> str:
        """qbx_autotune: time the staged-FFT configurations on this context
        and keep the fastest; returns the report."""
        buf = ctypes.create_string_buffer(4096)
        self._ok(self.lib.qbx_autotune(self.h, buf, 4096), "autotune")
        return buf.value.decode()

    STRESS_PARTS = ("ekin", "eps", "enl", "ehart", "exc", "esr")

    def _stress_out(self, fn, what):
        sig = np.zeros(6)
        parts = np.zeros(36)
        self._ok(fn(self.h, _dp(sig), _dp(parts)), what)
        return sig, dict(zip(self.STRESS_PARTS, parts.reshape(6, 6)))

    def stress(self):
        """qbx_stress: sigma (xx yy zz xy yz xz) of the last energy() and its
        parts {ekin, eps, enl, ehart, exc, esr}."""
        return self._stress_out(self.lib.qbx_stress, "stress")

    def last_stress(self):
        """qbx_get_stress: the stress of the last scf_step(stress=True)."""
        return self._stress_out(self.lib.qbx_get_stress, "get_stress")

    def density_static(self, c_dev_ptr: int, nst: int, rho_dev_ptr: int,
                       occ: Optional[np.ndarray] = None):
        """qbx_density_static: density of nst bands held in device memory
        (default coefficient order) into a device grid, using the library's
        static scratch array; pointers are raw device addresses."""
        o = None if occ is None else np.ascontiguousarray(occ, dtype=float)
        if o is not None and o.size != nst:
            raise ValueError(f"density_static: {o.size} occupations for {nst} bands")
        self._ok(self.lib.qbx_density_static(self.h, ctypes.c_void_p(c_dev_ptr), nst,
                                             _dp(o), ctypes.c_void_p(rho_dev_ptr)),
                 "density_static")

    # ---- the reference's class methods on host arrays
    def compute_density(self, weight: float, rho: np.ndarray):
        """SlaterDet::compute_density: rho += weight * sum_n occ_n/Omega
        |psi_n|^2 (rho: float64 array of the grid size, x fastest)."""
        assert rho.dtype == np.float64 and rho.flags["C_CONTIGUOUS"]
        assert rho.size == self.grid[0] * self.grid[1] * self.grid[2]
        self._ok(self.lib.qbx_compute_density(self.h, float(weight), _dp(rho)),
                 "compute_density")

    def rs_mul_add(self, v: np.ndarray, dc: np.ndarray):
        """SlaterDet::rs_mul_add: dc += FFT_fwd(v FFT_bwd(c)) (dc: complex
        (nst, ngw), modified in place)."""
        vv = np.ascontiguousarray(v, float)
        assert vv.size == self.grid[0] * self.grid[1] * self.grid[2]
        assert dc.dtype == np.complex128 and dc.flags["C_CONTIGUOUS"]
        assert dc.shape == (self.nst, self.ngw)
        self._ok(self.lib.qbx_rs_mul_add(self.h, _dp(vv), _dp(dc.view(np.float64))),
                 "rs_mul_add")

    def nonlocal_energy(self, dc: Optional[np.ndarray] = None, forces: bool = False,
                        stress: bool = False):
        """NonLocalPotential::energy: returns {"enl", "fion" (natoms x 3),
        "sigma_enl" (6)}; with dc the nonlocal H*C is added into it."""
        if dc is not None:
            assert dc.dtype == np.complex128 and dc.flags["C_CONTIGUOUS"]
            assert dc.shape == (self.nst, self.ngw)
        f = np.zeros(3 * max(1, self.natoms))
        sig = np.zeros(6)
        e = _D()
        self._ok(self.lib.qbx_nonlocal_energy(
            self.h, int(dc is not None), _dp(dc.view(np.float64)) if dc is not None else None,
            int(forces), _dp(f), int(stress), _dp(sig), ctypes.byref(e)), "nonlocal_energy")
        out = {"enl": e.value}
        if forces:
            out["fion"] = f[:3 * self.natoms].reshape(-1, 3)
        if stress:
            out["sigma_enl"] = sig
        return out

    def ortho_align(self, c_ref: np.ndarray):
        """SlaterDet::ortho_align(sd) with sd's coefficients c_ref."""
        a = np.ascontiguousarray(c_ref, np.complex128)
        assert a.shape == (self.nst, self.ngw)
        self._ok(self.lib.qbx_ortho_align(self.h, _dp(a.view(np.float64))), "ortho_align")

    def diag(self, eigvec: bool = True) -> np.ndarray:
        """Wavefunction::diag after energy(hpsi=True): the eigenvalues of
        C^T H C; with eigvec C becomes its eigenvectors."""
        w = np.zeros(self.nst)
        self._ok(self.lib.qbx_diag(self.h, int(eigvec), _dp(w)), "diag")
        return w

    def dot(self, c_other: np.ndarray) -> float:
        """SlaterDet::dot(sd) at Gamma."""
        a = np.ascontiguousarray(c_other, np.complex128)
        assert a.shape == (self.nst, self.ngw)
        d = _D()
        self._ok(self.lib.qbx_dot(self.h, _dp(a.view(np.float64)), ctypes.byref(d)), "dot")
        return d.value

    def set_band_shard(self, rank: int, nranks: int, nccl_id: Optional[bytes]):
        """qbx_set_band_shard: this GPU transforms its share of the band
        pairs; densities and H*psi blocks are exchanged over NCCL."""
        if nccl_id is not None:
            assert len(nccl_id) == NCCL_ID_BYTES
        self._ok(self.lib.qbx_set_band_shard(self.h, rank, nranks, nccl_id), "set_band_shard")

    def stream(self) -> int:
        return self.lib.qbx_stream(self.h)

    def set_coeffs_async(self, c_pinned: np.ndarray):
        self._ok(self.lib.qbx_set_coeffs_async(self.h, _dp(c_pinned)), "set_coeffs_async")

    def get_coeffs_async(self, out_pinned: np.ndarray):
        self._ok(self.lib.qbx_get_coeffs_async(self.h, _dp(out_pinned)), "get_coeffs_async")


def nccl_unique_id() -> bytes:
    """qbx_nccl_unique_id: a new NCCL group id (made on one rank, passed to
    the others by the caller)."""
    lib = load()
    buf = ctypes.create_string_buffer(NCCL_ID_BYTES)
    rc = lib.qbx_nccl_unique_id(buf)
    if rc:
        raise QbxError(f"qbx_nccl_unique_id failed with code {rc}")
    return buf.raw


def shard_pairs(nst: int, rank: int, nranks: int):
    """qbx_shard_pairs: the band pairs [first, end) of rank among nranks."""
    lib = load()
    a, b = _I(), _I()
    rc = lib.qbx_shard_pairs(nst, rank, nranks, ctypes.byref(a), ctypes.byref(b))
    if rc:
        raise QbxError(f"qbx_shard_pairs: code {rc}")
    return a.value, b.value


class FourierTransform:
    """qbx_ft: the reference's FourierTransform(basis, np0, np1, np2) on a
    caller's basis (Miller indices in the caller's order) and grid."""

    def __init__(self, hkl: np.ndarray, grid, real_basis: bool = True, device: int = 0):
        self.lib = load()
        idx = np.ascontiguousarray(np.asarray(hkl, np.int32).reshape(-1, 3))
        self.ngw = idx.shape[0]
        self.grid = tuple(int(x) for x in grid)
        h = _P()
        rc = self.lib.qbx_ft_create(ctypes.byref(h), device, self.ngw, _ip(idx),
                                    int(real_basis), *self.grid)
        if rc:
            raise QbxError(f"qbx_ft_create failed with code {rc}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.qbx_ft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc, what):
        if rc:
            msg = self.lib.qbx_ft_last_error(self.h)
            raise QbxError(f"{what}: code {rc}: {msg.decode() if msg else ''}")

    @property
    def N(self):
        return self.grid[0] * self.grid[1] * self.grid[2]

    def _c(self, c):
        a = np.ascontiguousarray(c, np.complex128)
        assert a.size == self.ngw
        return a

    def backward(self, c: np.ndarray, c2: Optional[np.ndarray] = None) -> np.ndarray:
        """Complex grid (np2, np1, np0) of one band, or of c + i c2."""
        f = np.empty(self.N, np.complex128)
        a = self._c(c)
        if c2 is None:
            self._ok(self.lib.qbx_ft_backward(self.h, _dp(a.view(np.float64)),
                                              _dp(f.view(np.float64))), "ft_backward")
        else:
            b = self._c(c2)
            self._ok(self.lib.qbx_ft_backward2(self.h, _dp(a.view(np.float64)),
                                               _dp(b.view(np.float64)),
                                               _dp(f.view(np.float64))), "ft_backward2")
        return f.reshape(self.grid[2], self.grid[1], self.grid[0])

    def forward(self, f: np.ndarray, two: bool = False):
        """Coefficients of a complex grid (1/N scaling); two=True unpacks
        two real functions."""
        g = np.ascontiguousarray(f, np.complex128).reshape(-1)
        assert g.size == self.N
        c1 = np.empty(self.ngw, np.complex128)
        if not two:
            self._ok(self.lib.qbx_ft_forward(self.h, _dp(g.view(np.float64)),
                                             _dp(c1.view(np.float64))), "ft_forward")
            return c1
        c2 = np.empty(self.ngw, np.complex128)
        self._ok(self.lib.qbx_ft_forward2(self.h, _dp(g.view(np.float64)),
                                          _dp(c1.view(np.float64)), _dp(c2.view(np.float64))),
                 "ft_forward2")
        return c1, c2


def scf_step_batch(contexts, stress: bool = False, forces: bool = False):
    """qbx_scf_step_batch: one electronic step of every context, run
    concurrently; returns a list of energy dicts."""
    lib = load()
    n = len(contexts)
    arr = (_P * n)(*[c.h for c in contexts])
    e = np.zeros(n * NENERGY)
    rc = lib.qbx_scf_step_batch(arr, n, (2 if stress else 0) | (1 if forces else 0), _dp(e))
    if rc:
        msgs = [lib.qbx_last_error(c.h) for c in contexts]
        msg = next((m.decode() for m in msgs if m), "")
        raise QbxError(f"scf_step_batch: code {rc}: {msg}")
    return [dict(zip(ENERGY_NAMES, e[i * NENERGY:(i + 1) * NENERGY])) for i in range(n)]


def from_system(system, device: int = 0, precision: int = FP64,
                coeffs: Optional[np.ndarray] = None, gram: bool = True) -> Context:
    """Build a context for a qbx.systems.System and upload its seeded
    coefficients (keyed by sorted Miller index)."""
    ctx = Context(device, precision)
    ctx.set_cell(system.cell, system.ecut, system.nbands, system.xc)
    hkl = system.miller()
    if hkl.shape[0] != ctx.ngw:
        raise QbxError(f"basis size {ctx.ngw} differs from the generator's {hkl.shape[0]}")
    if not np.array_equal(ctx.miller(), hkl):
        ctx.set_coeff_order(hkl)
    for sp in system.species:
        ctx.add_species(sp.zval, sp.mesh_spacing, sp.local_potential(),
                        sp.projectors(), [d for _, d in sp.dmatrix()])
    counts = [len(system.positions(i)) for i in range(len(system.species))]
    tau = np.concatenate([system.positions(i) for i in range(len(system.species))])
    ctx.set_atoms(counts, tau)
    if coeffs is None:
        coeffs = system.coefficients(hkl)
    ctx.set_coeffs(coeffs)
    if system.kpoints:
        # the k points replace Gamma; their coefficients are keyed by the
        # sorted Miller list of each complex basis, the library's own order
        ctx.set_kpoints([k for k, _ in system.kpoints], [w for _, w in system.kpoints])
        for ik in range(len(system.kpoints)):
            hk = system.kmiller(ik)
            if not np.array_equal(ctx.kpoint_miller(ik), hk):
                raise QbxError(f"k point {ik}: basis differs from the generator's")
            ctx.set_kpoint_coeffs(ik, system.kcoefficients(ik, hk))
    if gram:
        ctx.gram()
    return ctx


# ---------------------------------------------------------- host-only helpers
def host_basis(cell, ecut: float):
    """(ngw, ngv, grid, hkl) from the library's host basis builder."""
    lib = load()
    a = np.ascontiguousarray(np.asarray(cell, float).ravel())
    ngw, ngv = _I(), _I()
    npg = (ctypes.c_int * 3)()
    rc = lib.qbx_host_basis(_dp(a), float(ecut), ctypes.byref(ngw), ctypes.byref(ngv), npg, None)
    if rc:
        raise QbxError(f"qbx_host_basis failed: {rc}")
    hkl = np.empty((ngw.value, 3), np.int32)
    rc = lib.qbx_host_basis(_dp(a), float(ecut), None, None, None, _ip(hkl))
    if rc:
        raise QbxError(f"qbx_host_basis failed: {rc}")
    return ngw.value, ngv.value, (npg[0], npg[1], npg[2]), hkl


def host_kbasis(cell, ecut: float, kpoint):
    """The complex basis at a k point from the library's host code: (Miller
    indices in coefficient order, index of the reference's first coefficient)."""
    lib = load()
    cell = np.ascontiguousarray(np.asarray(cell, float).reshape(9))
    k = np.ascontiguousarray(np.asarray(kpoint, float).reshape(3))
    n, first = _I(), _I()
    rc = lib.qbx_host_kbasis(_dp(cell), ecut, _dp(k), ctypes.byref(n), ctypes.byref(first), None)
    if rc:
        raise QbxError(f"qbx_host_kbasis: code {rc}")
    hkl = np.empty((n.value, 3), np.int32)
    lib.qbx_host_kbasis(_dp(cell), ecut, _dp(k), None, None, _ip(hkl))
    return hkl, first.value


def host_species_eval(sp, g: np.ndarray):
    """V_loc(G), dV_loc/dG and V_nl(G) per projector from the library."""
    lib = load()
    v = np.ascontiguousarray(sp.local_potential(), float)
    projs = sp.projectors()
    nproj = len(projs)
    pl = np.array([l for l, _ in projs], np.int32)
    pr = (np.ascontiguousarray(np.stack([p for _, p in projs]), float)
          if nproj else np.zeros(1))
    g = np.ascontiguousarray(g, float)
    vl = np.empty(g.size)
    dvl = np.empty(g.size)
    vnl = np.empty(max(1, nproj) * g.size)
    rc = lib.qbx_host_species_eval(int(sp.zval), float(sp.mesh_spacing), v.size, _dp(v),
                                   nproj, _ip(pl) if nproj else None, _dp(pr), g.size,
                                   _dp(g), _dp(vl), _dp(dvl), _dp(vnl))
    if rc:
        raise QbxError(f"qbx_host_species_eval failed: {rc}")
    return vl, dvl, vnl[:nproj * g.size].reshape(nproj, g.size)


def host_esr(system):
    lib = load()
    a = np.ascontiguousarray(np.asarray(system.cell, float).ravel())
    nsp = len(system.species)
    na = np.array([len(system.positions(i)) for i in range(nsp)], np.int32)
    zv = np.array([float(sp.zval) for sp in system.species])
    tau = np.ascontiguousarray(np.concatenate([system.positions(i) for i in range(nsp)]))
    e = _D()
    f = np.empty(3 * int(na.sum()))
    rc = lib.qbx_host_esr(_dp(a), nsp, _ip(na), _dp(zv), _dp(tau), ctypes.byref(e), _dp(f))
    if rc:
        raise QbxError(f"qbx_host_esr failed: {rc}")
    return e.value, f.reshape(-1, 3)
