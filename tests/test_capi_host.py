"""CPU tests of the C ABI: the library loads, exports every entry point that
include/qbx.h declares, refuses to create a context without a GPU, and its
host-side setup code (basis, species tables, E_sr) matches the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from qbx import capi, systems
from oracle import qbox_np


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "qbx.h")).read()
    return sorted(set(re.findall(r"\b(qbx_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(capi.SYMBOLS)
    assert lib.qbx_version() == 1


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = capi.load()
    h = ctypes.c_void_p()
    assert lib.qbx_create(ctypes.byref(h), 0, 0) == 8
    with pytest.raises(capi.QbxError):
        capi.Context()


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32", "si512"])
def test_host_basis_matches_oracle(name):
    s = systems.get(name)
    ngw, ngv, grid, hkl = capi.host_basis(s.cell, s.ecut)
    shape = qbox_np.dense_grid(np.array(s.cell), s.ecut)
    assert list(grid) == list(shape)
    assert ngw == s.miller().shape[0]
    np.testing.assert_array_equal(hkl, s.miller())
    if name != "si512":
        g = np.load(os.path.join(ROOT, "tests", "golden", f"ref_{name}.npz"))
        assert ngw == int(g["ngw"]) and ngv == int(g["ng_v"])
        assert list(grid) == list(g["grid"])


def test_basis_sizes_of_survey_configs():
    # 512-atom cell: 72 919 coefficients per band on a 140^3 grid
    s = systems.si512()
    ngw, ngv, grid, _ = capi.host_basis(s.cell, s.ecut)
    assert ngw == 72919 and tuple(grid) == (140, 140, 140) and ngv == 583904


@pytest.mark.parametrize("sp", [systems.SI, systems.O, systems.H])
def test_host_species_tables_match_oracle(sp):
    g = np.linspace(0.0, 12.0, 997)
    vl, dvl, vnl = capi.host_species_eval(sp, g)
    ref = qbox_np.Species(sp)
    v, dv = ref.dvlocg(g)
    np.testing.assert_allclose(vl, v, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(dvl, dv, rtol=1e-10, atol=1e-10)
    for iop in range(len(sp.projectors())):
        p, _ = ref.vnlg(iop, g)
        np.testing.assert_allclose(vnl[iop], p, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("name", ["si8", "h2o32"])
def test_host_esr_matches_reference(name):
    s = systems.get(name)
    e, f = capi.host_esr(s)
    zv = [sp.zval for sp in s.species]
    pos = [s.positions(i) for i in range(len(s.species))]
    e_ref, f_ref = qbox_np.esr_forces(s, zv, pos)
    assert abs(e - e_ref) < 1e-12 * max(1, abs(e_ref))
    np.testing.assert_allclose(f, np.concatenate(f_ref), atol=1e-12)
    g = np.load(os.path.join(ROOT, "tests", "golden", f"ref_{name}.npz"))
    assert abs(e - g["e_esr"][0]) < 1e-10


@pytest.mark.parametrize("name", ["si8k2", "h2o4k2"])
def test_host_kbasis_matches_oracle_and_reference(name):
    """The complex basis at each k point (host code of the library) equals
    the oracle's Miller set, has the reference's size (golden fixture) and
    the reference's first local coefficient (rod (0,0), lowest l)."""
    from conftest import golden
    from oracle import qbox_np
    s = systems.get(name)
    g = golden(name)
    base = qbox_np.ElectronicStep(s)
    for ik, (k, w) in enumerate(s.kpoints):
        hkl, first = capi.host_kbasis(s.cell, s.ecut, k)
        np.testing.assert_array_equal(hkl, s.kmiller(ik))
        assert hkl.shape[0] == int(g[f"k{ik}_ngw"])
        kp = qbox_np.KPoint(base, k, w, s.kmiller(ik), np.zeros((1, hkl.shape[0])))
        assert first == kp.first
