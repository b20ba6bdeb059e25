"""The electronic step at k points off Gamma (complex bases) through the C ABI
against the oracle's restatement (oracle/qbox_np.py, KPointStep) and the
reference's own PSDA run on the same k points (tests/golden/ref_<name>.npz).

The k-point path is FP64: density, H*psi and energies agree with the oracle
to 1e-10 (relative to the largest value) and the energies with the reference
to 1e-8 Ha over the golden fixture's steps.
"""
import numpy as np
import pytest

from conftest import golden
from qbx import capi, systems
from oracle import qbox_np

pytestmark = pytest.mark.gpu

TERMS = ("ekin", "eps", "enl", "ehart", "exc", "esr", "eself", "etotal", "eigenvalue_sum")


@pytest.mark.parametrize("name", ["si8k2", "h2o4k2"])
def test_kpoint_step_matches_oracle(name):
    s = systems.get(name)
    ctx = capi.from_system(s, precision=capi.FP64)
    ks = qbox_np.KPointStep(s)
    for ik, kp in enumerate(ks.kpts):
        c = ctx.get_kpoint_coeffs(ik)
        np.testing.assert_allclose(c, kp.c, rtol=0, atol=1e-12)
    # the parts of the first step, one by one
    ctx.update_density()
    ks.update_density()
    rho = ctx.density().ravel()
    np.testing.assert_allclose(rho, ks.base.rhor, rtol=0, atol=1e-11 * np.abs(rho).max())
    ctx.update_vhxc()
    ks.update_vhxc()
    e = ctx.energy(hpsi=True)
    ks.energy(True)
    assert abs(e["ekin"] - ks.ekin) < 1e-9 and abs(e["enl"] - ks.enl) < 1e-11
    assert abs(e["etotal"] - ks.etotal) < 1e-9
    for ik, kp in enumerate(ks.kpts):
        hc = ctx.get_kpoint_hpsi(ik)
        np.testing.assert_allclose(hc, kp.hc, rtol=0, atol=1e-10 * np.abs(kp.hc).max())
    assert abs(ctx.eigenvalue_sum() - ks.eigenvalue_sum()) < 1e-9
    ctx.psda_update()
    ks.psda_update()
    for ik, kp in enumerate(ks.kpts):
        np.testing.assert_allclose(ctx.get_kpoint_coeffs(ik), kp.c, rtol=0, atol=1e-10)
    # whole steps (with Anderson extrapolation from the second update on)
    for it in range(3):
        eg = ctx.scf_step()
        eo = ks.step()
        for t in TERMS:
            assert abs(eg[t] - eo[t]) < 1e-8, (it, t, eg[t], eo[t])
    for ik, kp in enumerate(ks.kpts):
        np.testing.assert_allclose(ctx.get_kpoint_coeffs(ik), kp.c, rtol=0, atol=1e-9)
    ctx.close()


@pytest.mark.parametrize("name", ["si8k2", "h2o4k2"])
def test_kpoint_step_matches_reference(name):
    """Each PSDA step's energy terms equal the reference's at the same k
    points to 1e-8 Ha; the final coefficients match its sampled bands."""
    g = golden(name)
    s = systems.get(name)
    ctx = capi.from_system(s, precision=capi.FP64)
    for it in range(int(g["nsteps"])):
        e = ctx.scf_step()
        for t in TERMS:
            assert abs(e[t] - g["e_" + t][it]) < 1e-8, (it, t, e[t], g["e_" + t][it])
    for ik in range(int(g["nkp"])):
        c = ctx.get_kpoint_coeffs(ik)
        gi = g[f"k{ik}_g_idx"]
        np.testing.assert_allclose(c[:4, gi], g[f"k{ik}_final_c_bands"], rtol=0, atol=1e-9)
        np.testing.assert_allclose((np.abs(c) ** 2).sum(1), g[f"k{ik}_final_c_norm2"], rtol=1e-10)
    ctx.close()


def test_kpoints_run_fp64_in_a_mixed_context():
    """A mixed-precision context runs the k-point step in FP64: the same
    energies as an FP64 context."""
    s = systems.si8k2()
    a = capi.from_system(s, precision=capi.FP64)
    b = capi.from_system(s, precision=capi.MIXED)
    for _ in range(2):
        ea, eb = a.scf_step(), b.scf_step()
        assert abs(ea["etotal"] - eb["etotal"]) < 1e-11
    a.close()
    b.close()


def test_kpoint_errors_and_return_to_gamma():
    """Forces, stress and the Gamma-only drivers refuse k points with an
    error; set_kpoints([]) returns the context to its Gamma coefficients."""
    s = systems.si8k2()
    ctx = capi.from_system(s, precision=capi.FP64)
    with pytest.raises(capi.QbxError):
        ctx.scf_step(forces=True)
    with pytest.raises(capi.QbxError):
        ctx.set_kpoints([[0.0, 0.0, 0.0]], [1.0])
    assert len(ctx.get_kpoint_coeffs(1)) == s.nbands      # the refused set changed nothing
    ctx.set_kpoints([], [])
    ctx.gram()                   # the Gamma coefficients as from_system leaves them
    ref = capi.from_system(systems.si8(), precision=capi.FP64)
    ea, eb = ctx.scf_step(), ref.scf_step()
    assert abs(ea["etotal"] - eb["etotal"]) < 1e-10
    ctx.close()
    ref.close()


@pytest.mark.parametrize("name", ["si8k2", "h2o4k2"])
def test_kpoint_step_captured_equals_eager(name):
    """The k-point step as one CUDA graph (qbx_set_step_graph): the complex
    polar iteration in WHILE/IF conditional nodes, the Cholesky status in a
    device word.  Captured from its second use; every step equals the eager
    step of a twin context to 1e-12 Ha, and the reference's energies to 1e-8
    Ha over the fixture's steps."""
    g = golden(name)
    s = systems.get(name)
    eager = capi.from_system(s, precision=capi.FP64)
    graph = capi.from_system(s, precision=capi.FP64)
    graph.set_step_graph(True)
    nsteps = int(g["nsteps"])
    for it in range(nsteps):
        ra = eager.scf_step()
        rb = graph.scf_step()
        for k in TERMS:
            assert abs(ra[k] - rb[k]) < 1e-12 * max(1.0, abs(ra[k])), (it, k, ra[k], rb[k])
            assert abs(rb[k] - g["e_" + k][it]) < 1e-8 * max(1.0, abs(g["e_" + k][it])), (it, k)
    captured, launches, _ = graph.step_graph_info()
    assert captured >= 1 and launches >= 1, (captured, launches)
    for ik in range(len(s.kpoints)):
        np.testing.assert_allclose(graph.get_kpoint_coeffs(ik), eager.get_kpoint_coeffs(ik),
                                   atol=1e-12)
    eager.close()
    graph.close()
