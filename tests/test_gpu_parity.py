"""GPU parity of the electronic step against the oracle and the reference.

Every call goes through the C ABI (libqbx.so via qbx.capi).  The oracle
(oracle/qbox_np.py) is pinned to the reference by tests/test_oracle.py; the
trajectory tests also compare with the reference's own energies and forces
stored in tests/golden/.

Tolerances: FP64 path - total energy 1e-8 Ha and forces 1e-6 Ha/bohr against
the reference; grids and H*psi 1e-10 absolute against the oracle.  Mixed
path (FP32 FFTs) - total energy within 1e-6 Ha/atom and forces within 1e-4
Ha/bohr of the FP64 path.
"""
import numpy as np
import pytest

from conftest import golden
from qbx import capi, systems
from oracle import qbox_np

pytestmark = pytest.mark.gpu

TERMS = ("ekin", "eps", "enl", "ehart", "exc", "esr", "eself", "etotal",
         "eigenvalue_sum")


@pytest.fixture(scope="module")
def si8_oracle():
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(True, forces=True)
    return s, es


def test_ft_backward_pair(si8_oracle):
    s, es = si8_oracle
    ctx = capi.from_system(s)
    c = ctx.get_coeffs()
    np.testing.assert_allclose(c, es.c, atol=1e-13)
    f = ctx.ft_backward_pair(0, 1)
    ref = es.wgrid.backward(es.c[0], es.c[1])
    np.testing.assert_allclose(f, ref, atol=1e-12)
    f = ctx.ft_backward_pair(3, -1)
    ref = es.wgrid.backward(es.c[3])
    np.testing.assert_allclose(f, ref, atol=1e-12)
    ctx.close()


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_density_potential_hpsi(si8_oracle, precision):
    s, es = si8_oracle
    ctx = capi.from_system(s, precision=precision)
    q = ctx.update_density()
    tol = 1e-12 if precision == capi.FP64 else 1e-6
    assert abs(q - s.nel) < (1e-9 if precision == capi.FP64 else 1e-4)
    rho = ctx.density()
    np.testing.assert_allclose(rho, es.rhor, atol=tol * np.abs(es.rhor).max())
    ctx.update_vhxc()
    vr = ctx.vr()
    np.testing.assert_allclose(vr, es.v_r, atol=(1e-10 if precision == capi.FP64 else 1e-5))
    e = ctx.energy(hpsi=True, forces=True)
    hc = ctx.get_hpsi()
    np.testing.assert_allclose(hc, es.hc, atol=(1e-11 if precision == capi.FP64 else 1e-5))
    etol = 1e-9 if precision == capi.FP64 else 1e-5
    for k in ("ekin", "eps", "enl", "ehart", "exc", "etotal"):
        assert abs(e[k] - getattr(es, k)) < etol * max(1, abs(getattr(es, k))), k
    np.testing.assert_allclose(e["fion"], np.concatenate(es.fion),
                               atol=(1e-9 if precision == capi.FP64 else 1e-4))
    ctx.close()


@pytest.mark.parametrize("name,nsteps", [("si8", 20), ("si64", 3), ("h2o32", 1)])
def test_fp64_trajectory_matches_reference(name, nsteps):
    g = golden(name)
    s = systems.get(name)
    ctx = capi.from_system(s, precision=capi.FP64)
    for it in range(nsteps):
        last = it == nsteps - 1
        r = ctx.scf_step(forces=(it == 0 or last))
        for k in TERMS:
            ref = g["e_" + k][it]
            tol = 1e-8 if k in ("etotal", "eigenvalue_sum") else 1e-8 * max(1, abs(ref))
            assert abs(r[k] - ref) < max(tol, 1e-8), (it, k, r[k], ref)
        if it == 0:
            np.testing.assert_allclose(r["fion"], g["fion_first"], atol=1e-6)
        if last and nsteps == int(g["nsteps"]):
            np.testing.assert_allclose(r["fion"], g["fion_last"], atol=1e-6)
    if nsteps == int(g["nsteps"]):
        c = ctx.get_coeffs()
        np.testing.assert_allclose(c[:4, g["g_idx"]], g["final_c_bands"], atol=1e-8)
    ctx.close()


def test_mixed_trajectory_within_budget():
    """Mixed precision stays within 1e-6 Ha/atom of the FP64 path over the
    20-step 8-atom trajectory, forces within 1e-4 Ha/bohr."""
    s = systems.si8()
    natoms = len(s.atoms)
    a = capi.from_system(s, precision=capi.FP64)
    b = capi.from_system(s, precision=capi.MIXED)
    for it in range(20):
        ra = a.scf_step(forces=(it == 19))
        rb = b.scf_step(forces=(it == 19))
    assert abs(ra["etotal"] - rb["etotal"]) / natoms < 1e-6, (ra["etotal"], rb["etotal"])
    np.testing.assert_allclose(rb["fion"], ra["fion"], atol=1e-4)
    a.close()
    b.close()


@pytest.mark.parametrize("backend", [0, 1])
def test_mixed_si64_within_budget(backend):
    """Mixed path with split-BF16 products (cuBLAS or tcgen05) against the
    FP64 path on the 64-atom PBE cell.  Each step starts both paths from the
    same coefficients (the FP64 trajectory's), so the energy difference is
    the error the mixed step itself makes: 1e-6 Ha/atom in the total energy,
    1e-4 Ha/bohr in the forces, and the mixed ortho_align leaves C
    orthonormal to 1e-6 (its rotation is an FP32-accurate product, so the
    overlap of the new C is exact to a few FP32 roundings; the next step's
    overlap Cholesky is FP64).  (Whole trajectories started from random
    coefficients are compared on the 8-atom cell, where they converge; far
    from the ground state the PSDA step amplifies any difference in C to
    first order in the energy.)"""
    s = systems.si64()
    natoms = len(s.atoms)
    a = capi.from_system(s, precision=capi.FP64)
    b = capi.from_system(s, precision=capi.MIXED)
    b.set_gemm_backend(backend)
    for it in range(3):
        b.set_coeffs(a.get_coeffs())
        ra = a.scf_step(forces=(it == 2))
        rb = b.scf_step(forces=(it == 2))
        assert abs(ra["etotal"] - rb["etotal"]) / natoms < 1e-6, (it, ra["etotal"], rb["etotal"])
    np.testing.assert_allclose(rb["fion"], ra["fion"], atol=1e-4)
    cb = b.get_coeffs()
    ov = 2.0 * (cb.conj() @ cb.T).real - np.outer(cb[:, 0].real, cb[:, 0].real)
    assert np.abs(ov - np.eye(s.nbands)).max() < 1e-6
    a.close()
    b.close()


def test_orthonormal_and_charge_invariants():
    """Known-answer invariants (src/SlaterDet.cpp:1272-1314 orthonormality,
    src/ChargeDensity.cpp:173-191 total charge) on the GPU path."""
    s = systems.si64()
    ctx = capi.from_system(s, precision=capi.FP64)
    for _ in range(2):
        r = ctx.scf_step()
        assert abs(r["total_charge"] - s.nel) < 1e-9
    c = ctx.get_coeffs()
    ov = 2.0 * (c.conj() @ c.T).real - np.outer(c[:, 0].real, c[:, 0].real)
    assert np.abs(ov - np.eye(s.nbands)).max() < 1e-10
    ctx.close()


def test_caller_coefficient_order():
    """qbx_set_coeff_order: a shuffled caller order gives identical physics."""
    s = systems.si8()
    hkl = s.miller()
    c = s.coefficients(hkl)
    perm = np.random.default_rng(7).permutation(hkl.shape[0])
    ctx = capi.Context()
    ctx.set_cell(s.cell, s.ecut, s.nbands, s.xc)
    ctx.set_coeff_order(hkl[perm])
    for sp in s.species:
        ctx.add_species(sp.zval, sp.mesh_spacing, sp.local_potential(),
                        sp.projectors(), [d for _, d in sp.dmatrix()])
    ctx.set_atoms([len(s.atoms)], s.positions(0))
    ctx.set_coeffs(c[:, perm])
    ctx.gram()
    r = ctx.scf_step()
    g = golden("si8")
    assert abs(r["etotal"] - g["e_etotal"][0]) < 1e-8
    ctx.close()


def test_errors_are_reported():
    ctx = capi.Context()
    with pytest.raises(capi.QbxError, match="set_cell"):
        ctx.update_density()
    with pytest.raises(capi.QbxError):
        ctx.set_cell(np.eye(3) * 10.0, 10.0, 4, "B3LYP")
    # a non-positive-definite overlap (two identical bands) fails in gram
    s = systems.si8()
    c = s.coefficients()
    c[1] = 0.0
    with pytest.raises(capi.QbxError, match="positive definite"):
        capi.from_system(s, coeffs=c)
    ctx.close()


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
def test_stress_matches_reference(name):
    """Stress tensor of the first step (EnergyFunctional::energy with
    compute_stress) against the reference's own sigma: 1e-9 Ha/bohr^3 in
    FP64; the mixed path within 1e-6 relative of the largest component."""
    g = golden(name)
    s = systems.get(name)
    ctx = capi.from_system(s, precision=capi.FP64)
    r = ctx.scf_step(forces=True, stress=True)
    np.testing.assert_allclose(r["sigma"], g["sigma_first"], rtol=0, atol=1e-9)
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(False)
    es.stress()
    for k, v in r["sigma_parts"].items():
        np.testing.assert_allclose(v, es.sigma_parts[k], rtol=0, atol=1e-9, err_msg=k)
    ctx.close()
    m = capi.from_system(s, precision=capi.MIXED)
    rm = m.scf_step(stress=True)
    scale = np.abs(g["sigma_first"]).max()
    np.testing.assert_allclose(rm["sigma"], g["sigma_first"], rtol=0, atol=1e-6 * scale)
    m.close()


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_jd_trajectory_matches_reference(precision):
    """wf_dyn JD (JDWavefunctionStepper::update): the eigenvalue sum of six
    steps from the seeded start against the reference's JD run; 1e-8 in
    FP64, 1e-5 relative in the mixed precision."""
    g = golden("si8_jd")
    s = systems.si8()
    ctx = capi.from_system(s, precision=precision)
    ctx.set_wf_dyn("JD")
    for it in range(int(g["nsteps"])):
        r = ctx.scf_step()
        ref = g["e_eigenvalue_sum"][it]
        tol = 1e-8 if precision == capi.FP64 else 1e-5 * max(1.0, abs(ref))
        assert abs(r["eigenvalue_sum"] - ref) < tol, (it, r["eigenvalue_sum"], ref)
    ctx.close()


def test_batch_of_systems_matches_single_steps():
    """qbx_scf_step_batch over six systems of the 32-system batch (different
    cells, cutoffs, grids and band counts), run concurrently, gives the
    energies of stepping each context on its own."""
    systs = systems.batch()[:6]
    ctxs = [capi.from_system(s, precision=capi.FP64) for s in systs]
    ref = [capi.from_system(s, precision=capi.FP64) for s in systs]
    for _ in range(2):
        eb = capi.scf_step_batch(ctxs)
        es = [c.scf_step() for c in ref]
        for a, b in zip(eb, es):
            assert abs(a["etotal"] - b["etotal"]) < 1e-10 * max(1.0, abs(b["etotal"]))
            assert abs(a["eigenvalue_sum"] - b["eigenvalue_sum"]) < 1e-9 * max(1.0, abs(b["eigenvalue_sum"]))
    for c in ctxs + ref:
        c.close()
