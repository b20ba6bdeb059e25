"""Molecular dynamics through the C ABI (qbx_md_run, qbx_move_atoms) against
the reference's own BOSampleStepper MD run (tests/golden/ref_si8_md.npz) and
between the library's own forms.

Tolerances: FP64 - energies printed by the reference to 8 decimals (6e-9),
positions 1e-10 bohr, velocities 1e-12, coefficients 1e-9; captured steps vs
eager 1e-11; mixed vs FP64 over two ionic steps 2e-6 Ha/atom on the energy
and 1e-5 bohr on the positions (the mixed forces differ by ~1e-5 Ha/bohr).
"""
import numpy as np
import pytest

from conftest import golden
from qbx import capi, systems

pytestmark = pytest.mark.gpu


def _masses(s):
    return [sp.mass for sp in s.species]


@pytest.mark.parametrize("graph", [False, True])
def test_md_matches_reference(graph):
    fx = golden("si8_md")
    s = systems.si8()
    ctx = capi.from_system(s, precision=capi.FP64)
    ctx.set_step_graph(graph)
    out = ctx.md_run(int(fx["niter"]), int(fx["nitscf"]), float(fx["dt"]), _masses(s))
    ion = out["ionic"]
    np.testing.assert_allclose(ion[:, 0], fx["etotal"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(ion[:, 1], fx["ekin_ion"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(ion[:, 2], fx["econst"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(out["positions"], fx["tau"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(out["velocities"], fx["vel"], rtol=0, atol=1e-12)
    c = ctx.get_coeffs()
    nb = fx["final_c_bands"].shape[0]
    np.testing.assert_allclose(c[:nb], fx["final_c_bands"], rtol=0, atol=1e-9)
    np.testing.assert_allclose((np.abs(c) ** 2).sum(1), fx["final_c_norm2"], rtol=1e-9)
    if graph:
        captured, launches, note = ctx.step_graph_info()
        assert note == "" and captured >= 1 and launches >= 2, (captured, launches, note)
    ctx.close()


def test_move_atoms_equals_set_atoms():
    """qbx_move_atoms (in place) gives the energy and forces of a context
    built at the new positions."""
    s = systems.si8()
    counts = [len(s.positions(i)) for i in range(len(s.species))]
    tau = np.concatenate([s.positions(i) for i in range(len(s.species))])
    tau2 = tau + 0.03 * np.random.default_rng(3).standard_normal(tau.shape)
    a = capi.from_system(s, precision=capi.FP64)
    b = capi.from_system(s, precision=capi.FP64)
    a.move_atoms(tau2)
    b.set_atoms(counts, tau2)
    ea = a.scf_step(forces=True)
    eb = b.scf_step(forces=True)
    assert abs(ea["etotal"] - eb["etotal"]) < 1e-11
    assert abs(ea["esr"] - eb["esr"]) < 1e-12
    np.testing.assert_allclose(ea["fion"], eb["fion"], rtol=0, atol=1e-11)
    a.close()
    b.close()


def test_md_mixed_close_to_fp64():
    s = systems.si64()
    natoms = len(s.atoms)
    runs = {}
    for prec in (capi.FP64, capi.MIXED):
        ctx = capi.from_system(s, precision=prec)
        ctx.set_step_graph(True)
        runs[prec] = ctx.md_run(2, 2, 20.0, _masses(s))
        ctx.close()
    a, b = runs[capi.FP64], runs[capi.MIXED]
    assert np.abs(a["ionic"][:, 0] - b["ionic"][:, 0]).max() / natoms < 2e-6
    assert np.abs(a["positions"] - b["positions"]).max() < 1e-5
