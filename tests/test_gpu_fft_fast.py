"""The specialised staged FFTs (fft_fast_*.cu: compile-time lengths,
warp-synchronous radix stages) against the generic runtime-radix kernels of
fft.cu and against the oracle, through the C ABI.

QBX_FAST_FFT=0 at qbx_set_cell selects the generic kernels for a context.
Tolerances: FP64 1e-12 of the largest value (the same arithmetic in another
order); mixed precision 2e-6 of the largest value.
"""
import os

import numpy as np
import pytest

from qbx import capi, systems
from oracle import qbox_np

pytestmark = pytest.mark.gpu


def _ctx(s, precision, fast):
    os.environ["QBX_FAST_FFT"] = "1" if fast else "0"
    try:
        return capi.from_system(s, precision=precision)
    finally:
        os.environ.pop("QBX_FAST_FFT", None)


def _run(ctx):
    ctx.update_density()
    rho = ctx.density()
    ctx.update_vhxc()
    e = ctx.energy(hpsi=True)
    return rho, ctx.get_hpsi(), e


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_fast_matches_generic(name, precision):
    s = systems.get(name)
    a = _ctx(s, precision, True)
    b = _ctx(s, precision, False)
    ra, ha, ea = _run(a)
    rb, hb, eb = _run(b)
    tol = 1e-12 if precision == capi.FP64 else 2e-6
    np.testing.assert_allclose(ra, rb, rtol=0, atol=tol * np.abs(rb).max())
    np.testing.assert_allclose(ha, hb, rtol=0, atol=tol * np.abs(hb).max())
    etol = (1e-9 if precision == capi.FP64 else 1e-6) * len(s.atoms)
    assert abs(ea["etotal"] - eb["etotal"]) < etol
    a.close()
    b.close()


def test_fast_fp64_matches_oracle_si64():
    s = systems.si64()
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(True)
    ctx = _ctx(s, capi.FP64, True)
    rho, hc, e = _run(ctx)
    np.testing.assert_allclose(rho, es.rhor, rtol=0, atol=1e-12 * np.abs(es.rhor).max())
    np.testing.assert_allclose(hc, es.hc, rtol=0, atol=1e-11)
    assert abs(e["etotal"] - es.etotal) < 1e-8
    ctx.close()


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_autotune_keeps_results(precision):
    """qbx_autotune times the staged-FFT configurations and keeps the
    fastest; whatever it picks, the density and H*psi stay the same."""
    s = systems.si64()
    a = _ctx(s, precision, True)
    ra, ha, ea = _run(a)
    report = a.autotune()
    assert "chosen:" in report
    rb, hb, eb = _run(a)
    tol = 1e-12 if precision == capi.FP64 else 2e-6
    np.testing.assert_allclose(rb, ra, rtol=0, atol=tol * np.abs(ra).max())
    np.testing.assert_allclose(hb, ha, rtol=0, atol=tol * np.abs(ha).max())
    a.close()


@pytest.mark.parametrize("shape", [5, 6, 7, 8])
@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
def test_density_half_planes(name, shape, monkeypatch):
    """The half-plane density kernel (shape 5: two CTAs per plane), the
    whole-plane kernel reading the sticks through the column map (shape 6),
    the kernel accumulating in tensor memory (shape 7) and the kernel that
    queues the next band pair's sticks with cp.async (shape 8) give the
    default kernel's density (FP32, 2e-6 of the largest value)."""
    s = systems.get(name)
    ref = _ctx(s, capi.MIXED, True)
    monkeypatch.setenv("QBX_FAST_DENSITY_LANE_SHAPE", str(shape))
    half = _ctx(s, capi.MIXED, True)
    monkeypatch.delenv("QBX_FAST_DENSITY_LANE_SHAPE")
    ref.update_density()
    half.update_density()
    ra, rb = ref.density(), half.density()
    np.testing.assert_allclose(rb, ra, rtol=0, atol=2e-6 * np.abs(ra).max())
    ref.close()
    half.close()


@pytest.mark.parametrize("shape", [5, 6])
@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
def test_vpsi_sticks_through_column_map(name, shape, monkeypatch):
    """The H*psi plane kernel that reads and writes the sticks through the
    column map (lane shapes 5 and 6) gives the default kernel's H*psi (FP32,
    2e-6 of the largest value)."""
    s = systems.get(name)
    ref = _ctx(s, capi.MIXED, True)
    monkeypatch.setenv("QBX_FAST_LANE_SHAPE", str(shape))
    alt = _ctx(s, capi.MIXED, True)
    monkeypatch.delenv("QBX_FAST_LANE_SHAPE")
    ra, ha, ea = _run(ref)
    rb, hb, eb = _run(alt)
    np.testing.assert_allclose(hb, ha, rtol=0, atol=2e-6 * np.abs(ha).max())
    assert abs(ea["etotal"] - eb["etotal"]) < 1e-6 * len(s.atoms)
    ref.close()
    alt.close()


def test_density_tmem_si512(monkeypatch):
    """The tensor-memory density kernel (shape 7) on the 512-atom cell's
    140^3 grid, where each thread holds 2 rows x 35 points in 3 column
    blocks of tensor memory, gives the default kernel's density (FP32, 2e-6
    of the largest value)."""
    s = systems.si512().band_sample(32)
    ref = _ctx(s, capi.MIXED, True)
    monkeypatch.setenv("QBX_FAST_DENSITY_LANE_SHAPE", "7")
    tm = _ctx(s, capi.MIXED, True)
    monkeypatch.delenv("QBX_FAST_DENSITY_LANE_SHAPE")
    ref.update_density()
    tm.update_density()
    ra, rb = ref.density(), tm.density()
    np.testing.assert_allclose(rb, ra, rtol=0, atol=2e-6 * np.abs(ra).max())
    ref.close()
    tm.close()


@pytest.mark.parametrize("graph", [False, True])
def test_density_queued_sticks_si512(graph, monkeypatch):
    """Density shape 8 on the 512-atom cell's 140^3 grid, where its two
    tiles, accumulator and tables fill 227 840 bytes of shared memory: the
    step that stores psi(r) from it gives the default kernel's energies
    (1e-12 relative) and coefficients after two steps (1e-12), eager and
    captured."""
    s = systems.si512().band_sample(32)
    ctxs = []
    for shape in ("8", "3"):
        monkeypatch.setenv("QBX_FAST_DENSITY_LANE_SHAPE", shape)
        c = _ctx(s, capi.MIXED, True)
        c.set_step_graph(graph)
        ctxs.append(c)
    monkeypatch.delenv("QBX_FAST_DENSITY_LANE_SHAPE")
    a, b = ctxs
    for _ in range(3 if graph else 2):
        ea, eb = a.scf_step(), b.scf_step()
        for k in ("ekin", "enl", "etotal", "eigenvalue_sum"):
            assert abs(ea[k] - eb[k]) <= 1e-12 * abs(eb[k]) + 1e-12, (k, ea[k], eb[k])
    np.testing.assert_allclose(a.get_coeffs(), b.get_coeffs(), rtol=0, atol=1e-12)
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32"])
def test_z_sticks_in_register_lanes(name, monkeypatch):
    """The z-stick transforms held in register lanes (kz_bwd_lane,
    kz_fwd_lane) give the warp-per-stick kernels' density and H*psi (FP32,
    2e-6 of the largest value) and total energy (1e-6 Ha per atom)."""
    s = systems.get(name)
    ctxs = []
    for mode in ("1", "0"):
        monkeypatch.setenv("QBX_ZLANE", mode)
        ctxs.append(_ctx(s, capi.MIXED, True))
    monkeypatch.delenv("QBX_ZLANE")
    a, b = ctxs
    ra, ha, ea = _run(a)
    rb, hb, eb = _run(b)
    np.testing.assert_allclose(ra, rb, rtol=0, atol=2e-6 * np.abs(rb).max())
    np.testing.assert_allclose(ha, hb, rtol=0, atol=2e-6 * np.abs(hb).max())
    assert abs(ea["etotal"] - eb["etotal"]) < 1e-6 * len(s.atoms)
    a.close()
    b.close()


@pytest.mark.parametrize("staged", ["0", "1"])
@pytest.mark.parametrize("ppc", ["3", "16"])
@pytest.mark.parametrize("name", ["si64", "si512_32"])
def test_hpsi_from_psi_r_pairs_per_cta(name, ppc, staged, monkeypatch):
    """The H*psi plane kernel from the stored psi(r) with several band pairs
    per CTA (3: a launch's 16 pairs end in a partial CTA; 16: one CTA per
    plane), each prefetching the next pair's psi(r) plane into L2 or (staged)
    copying its rounds of rows into shared memory with cp.async, gives the
    one-pair-per-CTA kernel's step: energies to 1e-12 relative and the
    coefficients after two steps to 1e-12."""
    s = systems.si64() if name == "si64" else systems.si512().band_sample(32)
    ctxs = []
    for mode, st in ((ppc, staged), ("1", "0")):
        monkeypatch.setenv("QBX_FWD_PAIRS_PER_CTA", mode)
        monkeypatch.setenv("QBX_FWD_STAGED", st)
        ctxs.append(_ctx(s, capi.MIXED, True))
    monkeypatch.delenv("QBX_FWD_PAIRS_PER_CTA")
    monkeypatch.delenv("QBX_FWD_STAGED")
    a, b = ctxs
    for _ in range(2):
        ea, eb = a.scf_step(), b.scf_step()
        for k in ("ekin", "enl", "etotal", "eigenvalue_sum"):
            assert abs(ea[k] - eb[k]) <= 1e-12 * abs(eb[k]) + 1e-12, (k, ea[k], eb[k])
    np.testing.assert_allclose(a.get_coeffs(), b.get_coeffs(), rtol=0, atol=1e-12)
    a.close()
    b.close()


@pytest.mark.parametrize("graph", [False, True])
def test_stored_psi_r_gives_the_recomputed_step(graph, monkeypatch):
    """psi(r) kept in HBM from the density pass and reused by the H*psi pass
    of the same step (QBX_PSIR=1) gives the step that transforms every band
    pair backward twice (QBX_PSIR=0): energies to 1e-12 relative and the
    coefficients after three steps to 1e-12, eager and captured."""
    s = systems.si64()
    ctxs = []
    for mode in ("1", "0"):
        monkeypatch.setenv("QBX_PSIR", mode)
        c = _ctx(s, capi.MIXED, True)
        c.set_step_graph(graph)
        ctxs.append(c)
    monkeypatch.delenv("QBX_PSIR")
    a, b = ctxs
    for _ in range(3):
        ea, eb = a.scf_step(), b.scf_step()
        for k in ("ekin", "enl", "etotal", "eigenvalue_sum"):
            assert abs(ea[k] - eb[k]) <= 1e-12 * abs(eb[k]) + 1e-12, (k, ea[k], eb[k])
    np.testing.assert_allclose(a.get_coeffs(), b.get_coeffs(), rtol=0, atol=1e-12)
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["si8", "si64", "h2o32", "si512_32"])
def test_pruned_lane_kernels(name, monkeypatch):
    """The FP32 lane kernels that skip the lane registers beyond the sphere
    (QBX_FFT_PRUNE=1: the H*psi plane pass stores only the columns and
    sticks within prune_width, the z passes load and store only the z
    within it, the density pass loads only the columns and rows within it)
    give the unpruned kernels' density and H*psi (2e-6 of the largest value),
    and their two-step trajectory: energies to 1e-8 Ha per atom and the
    coefficients to 1e-7.  The density pass is the queued-sticks kernel
    (shape 8) and the H*psi pass the staged one, as at 140^3."""
    s = systems.si512().band_sample(32) if name == "si512_32" else systems.get(name)
    ctxs = []
    monkeypatch.setenv("QBX_FAST_DENSITY_LANE_SHAPE", "8")
    for mode in ("1", "0"):
        monkeypatch.setenv("QBX_FFT_PRUNE", mode)
        ctxs.append(_ctx(s, capi.MIXED, True))
    monkeypatch.delenv("QBX_FFT_PRUNE")
    monkeypatch.delenv("QBX_FAST_DENSITY_LANE_SHAPE")
    a, b = ctxs
    ra, ha, ea = _run(a)
    rb, hb, eb = _run(b)
    np.testing.assert_allclose(ra, rb, rtol=0, atol=2e-6 * np.abs(rb).max())
    np.testing.assert_allclose(ha, hb, rtol=0, atol=2e-6 * np.abs(hb).max())
    natoms = len(s.atoms)
    for _ in range(2):
        ea, eb = a.scf_step(), b.scf_step()
        for k in ("ekin", "enl", "etotal", "eigenvalue_sum"):
            assert abs(ea[k] - eb[k]) <= 1e-8 * natoms, (k, ea[k], eb[k])
    np.testing.assert_allclose(a.get_coeffs(), b.get_coeffs(), rtol=0, atol=1e-7)
    a.close()
    b.close()
