"""The numpy oracle (oracle/qbox_np.py) against the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference Qbox sources
compiled single-task (tests/golden/make_golden.py).  These tests pin the
oracle that the GPU parity tests compare against.
"""
import dataclasses

import numpy as np
import pytest

from conftest import golden
from qbx import systems
from oracle import qbox_np

TERMS = ("ekin", "eps", "enl", "ehart", "exc", "esr", "eself", "etotal",
         "eigenvalue_sum")


def _check_step0(es, g):
    n = np.prod(g["grid"])
    assert es.N == n
    assert tuple(es.grid_shape) == tuple(g["grid"])
    assert es.wb.size == g["ngw"] and es.vb.size == g["ng_v"]
    np.testing.assert_allclose(es.rhor[g["sample_idx"]], g["rhor_sample"],
                               rtol=0, atol=1e-13)
    np.testing.assert_allclose(es.v_r[g["sample_idx"]], g["vr_sample"],
                               rtol=0, atol=1e-11)
    np.testing.assert_allclose(es.hc[:4, g["g_idx"]], g["hc_bands"], atol=1e-13)
    np.testing.assert_allclose((np.abs(es.hc) ** 2).sum(1), g["hc_norm2"],
                               rtol=1e-11)


@pytest.mark.parametrize("name,nsteps", [("si8", 20), ("si64", 3),
                                         ("h2o32", 1)])
def test_oracle_matches_reference(name, nsteps):
    g = golden(name)
    es = qbox_np.ElectronicStep(systems.get(name))
    for it in range(nsteps):
        last = it == nsteps - 1
        r = es.step(forces=(it == 0 or last))
        if it == 0:
            _check_step0(es, g)
            np.testing.assert_allclose(np.concatenate(es.fion), g["fion_first"],
                                       atol=1e-12)
        for k in TERMS:
            ref = g["e_" + k][it]
            assert abs(r[k] - ref) < 1e-9 * max(1.0, abs(ref)), (it, k, r[k], ref)
    if nsteps == int(g["nsteps"]):
        np.testing.assert_allclose(np.concatenate(es.fion), g["fion_last"],
                                   atol=1e-12)
        np.testing.assert_allclose(es.c[:4, g["g_idx"]], g["final_c_bands"],
                                   atol=1e-12)


def test_invariants_si8():
    """Known-answer invariants of the reference (src/SlaterDet.cpp:1272-1314
    orthonormality; src/ChargeDensity.cpp:173-191 total charge)."""
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    for _ in range(3):
        es.step()
        ov = es.real_dot(es.c, es.c)
        assert np.abs(ov - np.eye(s.nbands)).max() < 1e-12
        assert abs(es.total_charge - s.nel) < 1e-10


def test_fft_roundtrip_and_gaussian():
    """forward(backward(c)) = c on the sphere, and the analytic transform of
    a Gaussian (src/testFourierTransform.cpp:157-162)."""
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    c = es.c[0]
    f = es.wgrid.backward(c)
    assert np.abs(f.imag).max() < 1e-12
    np.testing.assert_allclose(es.wgrid.forward(f.ravel()), c, atol=1e-14)
    # Gaussian exp(-a r^2) at the origin of the 20.52-bohr cell: periodic
    # images and the truncation at |G|^2 < 8 ecut are both below 1e-12
    s = systems.si64()
    es = qbox_np.ElectronicStep(s)
    a = 1.0
    vb = es.vb
    ghat = (np.pi / a) ** 1.5 * np.exp(-vb.g2 / (4 * a)) / es.omega
    f = es.vgrid.backward(ghat).real
    n0, n1, n2 = es.grid_shape
    x = np.arange(n0) / n0
    L = s.cell[0, 0]
    d = np.minimum(x, 1 - x) * L
    r2 = d[None, None, :] ** 2 + d[None, :, None] ** 2 + d[:, None, None] ** 2
    np.testing.assert_allclose(f, np.exp(-a * r2), atol=1e-11)


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
def test_oracle_stress_matches_reference(name):
    """Stress tensor (src/EnergyFunctional.cpp:397-1044 with compute_stress,
    src/XCPotential.cpp:467-640, src/NonLocalPotential.cpp:1790-2069) at
    the first step against the reference's own sigma."""
    g = golden(name)
    es = qbox_np.ElectronicStep(systems.get(name))
    es.update_density()
    es.update_vhxc()
    es.energy(False)
    np.testing.assert_allclose(es.stress(), g["sigma_first"], rtol=0, atol=1e-12)


def _strained(s, es, eps):
    m = np.eye(3) + eps
    s2 = dataclasses.replace(s, cell=np.asarray(s.cell) @ m,
                             atoms=[(i, p @ m) for i, p in s.atoms])
    e2 = qbox_np.ElectronicStep(s2, c=es.c, like=es)
    e2.update_density()
    e2.update_vhxc()
    return e2.energy(False)


def test_stress_is_the_strain_derivative():
    """sigma_ij = -(1/Omega) dE/d(eps_ij) at fixed coefficients and fixed
    plane-wave set, by central differences with strain 1e-4 (the check of
    test/si4stress/check_stress.sh, here without re-converging)."""
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(False)
    sig = es.stress()
    h = 1e-4
    for k, (i, j) in enumerate(qbox_np.VOIGT):
        eps = np.zeros((3, 3))
        eps[i, j] += h
        if i != j:
            eps[j, i] += h
        d = (_strained(s, es, eps) - _strained(s, es, -eps)) / (2 * h)
        fd = -d / es.omega / (1 if i == j else 2)
        assert abs(fd - sig[k]) < 1e-7, (k, fd, sig[k])


def test_forces_are_the_position_derivative():
    """fion = -dE/dtau at fixed coefficients, central differences 1e-3 bohr."""
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(False, forces=True)
    f = np.concatenate(es.fion)
    h = 1e-3
    for a, j in ((0, 0), (3, 1), (5, 2)):
        e = []
        for sgn in (1, -1):
            atoms = [(i, p.copy()) for i, p in s.atoms]
            atoms[a][1][j] += sgn * h
            s2 = dataclasses.replace(s, atoms=atoms)
            e2 = qbox_np.ElectronicStep(s2, c=es.c, like=es)
            e2.update_density()
            e2.update_vhxc()
            e.append(e2.energy(False))
        assert abs(-(e[0] - e[1]) / (2 * h) - f[a, j]) < 1e-6, (a, j)


def test_oracle_jd_matches_reference():
    """JDWavefunctionStepper::update (src/JDWavefunctionStepper.cpp:47-376):
    the eigenvalue sum of every step, and the energy of the correction block
    Z that the reference's energy functional holds after each update."""
    g = golden("si8_jd")
    es = qbox_np.ElectronicStep(systems.si8())
    for it in range(int(g["nsteps"])):
        r = es.step(wf_dyn="JD")
        assert abs(r["eigenvalue_sum"] - g["e_eigenvalue_sum"][it]) < 1e-9
        assert abs(es.etotal - g["e_etotal"][it]) < 1e-9


def test_oracle_md_matches_reference():
    """qbox_np.md_run (BOSampleStepper::step with atoms_dyn MD, PSDA, linear
    wavefunction extrapolation, velocity Verlet) against the reference's own
    stepper: printed energies to their 8 decimals, final positions and
    velocities and final coefficients to rounding."""
    fx = golden("si8_md")
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    out = qbox_np.md_run(es, int(fx["niter"]), int(fx["nitscf"]), float(fx["dt"]),
                         [sp.mass for sp in s.species])
    et = np.array([d["etotal"] for d in out["ionic"]])
    ec = np.array([d["econst"] for d in out["ionic"]])
    ek = np.array([d["ekin_ion"] for d in out["ionic"]])
    np.testing.assert_allclose(et, fx["etotal"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(ec, fx["econst"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(ek, fx["ekin_ion"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(np.concatenate(out["positions"]), fx["tau"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(np.concatenate(out["velocities"]), fx["vel"], rtol=0, atol=1e-14)
    c = out["c"]
    np.testing.assert_allclose(c[:fx["final_c_bands"].shape[0]], fx["final_c_bands"], rtol=0,
                               atol=1e-11)
    np.testing.assert_allclose((np.abs(c) ** 2).sum(1), fx["final_c_norm2"], rtol=1e-11)


def test_oracle_scf_mixing_matches_reference():
    """qbox_np.scf_run (BOSampleStepper::step(0) with nite > 0, Anderson and
    Kerker charge mixing) against the reference's own stepper: printed
    etotal_int and eigenvalue sums to their 8 decimals, final coefficients
    to rounding."""
    fx = golden("si8_gs")
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    out = qbox_np.scf_run(es, int(fx["nitscf"]), int(fx["nite"]), float(fx["mix_coeff"]),
                          float(fx["mix_rcut"]), int(fx["mix_ndim"]))
    np.testing.assert_allclose(out["etotal_int"], fx["etotal_int"], rtol=0, atol=6e-9)
    np.testing.assert_allclose(out["eigenvalue_sum"], fx["eigenvalue_sum"], rtol=0, atol=6e-9)
    g = fx["g_idx"]
    np.testing.assert_allclose(es.c[:fx["final_c_bands"].shape[0], g], fx["final_c_bands"],
                               rtol=0, atol=1e-11)


@pytest.mark.parametrize("name", ["si8k2", "h2o4k2"])
def test_oracle_kpoints_match_reference(name):
    """The k-point restatement (complex bases, one band per FFT, C^H C
    products, k-weighted sums) against the reference's PSDA run on the same k
    points: every energy term of each step to 1e-10 Ha, the density sample,
    H*psi and the final coefficients of each k point."""
    g = golden(name)
    ks = qbox_np.KPointStep(systems.get(name))
    assert len(ks.kpts) == int(g["nkp"])
    for it in range(int(g["nsteps"])):
        e = ks.step()
        if it == 0:
            np.testing.assert_allclose(ks.base.rhor[g["sample_idx"]], g["rhor_sample"],
                                       rtol=0, atol=1e-13)
            for ik, kp in enumerate(ks.kpts):
                assert kp.hkl.shape[0] == int(g[f"k{ik}_ngw"])
                gi = g[f"k{ik}_g_idx"]
                np.testing.assert_allclose(kp.hc[:4, gi], g[f"k{ik}_hc_bands"], atol=1e-13)
                np.testing.assert_allclose((np.abs(kp.hc) ** 2).sum(1), g[f"k{ik}_hc_norm2"],
                                           rtol=1e-11)
        for t in TERMS:
            assert abs(e[t] - g["e_" + t][it]) < 1e-10, (it, t, e[t], g["e_" + t][it])
    for ik, kp in enumerate(ks.kpts):
        gi = g[f"k{ik}_g_idx"]
        np.testing.assert_allclose(kp.c[:4, gi], g[f"k{ik}_final_c_bands"], atol=1e-12)
        np.testing.assert_allclose((np.abs(kp.c) ** 2).sum(1), g[f"k{ik}_final_c_norm2"],
                                   rtol=1e-12)


def test_oracle_diag_matches_reference():
    """ElectronicStep.diag against the reference's Wavefunction::diag after
    three PSDA steps of the 64-atom cell: eigenvalues 1e-10 Ha, rotated
    coefficients 1e-7 up to the sign of each band."""
    g = golden("si64_diag")
    es = qbox_np.ElectronicStep(systems.si64())
    for _ in range(int(g["nsteps"])):
        es.step()
    es.update_density()
    es.update_vhxc()
    es.energy(True)
    w = es.diag(True)
    np.testing.assert_allclose(w, g["eig"], atol=1e-10)
    c = es.c[:, g["g_idx"]]
    sign = np.sign((c.conj() * g["final_c_bands"]).sum(1).real)
    np.testing.assert_allclose(c * sign[:, None], g["final_c_bands"], atol=1e-7)
