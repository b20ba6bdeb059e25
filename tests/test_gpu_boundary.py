"""The reference's class methods on caller arrays, through the C ABI, against
the oracle (oracle/qbox_np.py, pinned to the reference's own build).

* FourierTransform (qbx_ft_*): backward and forward, single and two-band,
  on the 8-atom cell's wavefunction basis and its density basis (4 ecut),
  in the default and in a shuffled caller order, and on a complex basis at
  a k point: 1e-12 of the values' scale (FP64).
* SlaterDet::compute_density, SlaterDet::rs_mul_add, NonLocalPotential::
  energy (E_nl, H*psi part, forces, sigma_enl), SlaterDet::ortho_align and
  SlaterDet::dot on the 8-atom cell, FP64: 1e-10 (grids, H*psi, forces,
  coefficients), 1e-10 relative (energies, dot).
"""
import numpy as np
import pytest

from qbx import capi, systems
from oracle import qbox_np

pytestmark = pytest.mark.gpu


def _numpy_backward_complex(hkl, grid, c):
    """Synthesis on a complex basis (+G only): numpy's inverse FFT times N."""
    n0, n1, n2 = grid
    N = n0 * n1 * n2
    h, k, l = hkl[:, 0], hkl[:, 1], hkl[:, 2]
    ip = ((l % n2) * n1 + (k % n1)) * n0 + (h % n0)
    z = np.zeros(N, complex)
    z[ip] = c
    return np.fft.ifftn(z.reshape(n2, n1, n0)) * N, ip


@pytest.mark.parametrize("which", ["wavefunction", "density", "shuffled"])
def test_fourier_transform_real_basis(which):
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    rng = np.random.default_rng(7)
    if which == "density":
        basis = qbox_np.Basis(s.cell, 4 * s.ecut)
        grid = qbox_np.Grid(basis, [es.wgrid.n0, es.wgrid.n1, es.wgrid.n2])
    else:
        basis, grid = es.wb, es.wgrid
    hkl = basis.hkl.copy()
    order = rng.permutation(len(hkl)) if which == "shuffled" else np.arange(len(hkl))
    ft = capi.FourierTransform(hkl[order], (grid.n0, grid.n1, grid.n2), real_basis=True)
    ng = len(hkl)
    c1 = rng.standard_normal(ng) + 1j * rng.standard_normal(ng)
    c2 = rng.standard_normal(ng) + 1j * rng.standard_normal(ng)
    g0 = basis.g0()
    c1[g0] = c1[g0].real
    c2[g0] = c2[g0].real
    ref1 = grid.backward(c1)
    ref2 = grid.backward(c1, c2)
    scale = np.abs(ref2).max()
    np.testing.assert_allclose(ft.backward(c1[order]), ref1, atol=1e-12 * scale)
    np.testing.assert_allclose(ft.backward(c1[order], c2[order]), ref2, atol=1e-12 * scale)
    f = rng.standard_normal(grid.N) + 1j * rng.standard_normal(grid.N)
    np.testing.assert_allclose(ft.forward(f), grid.forward(f)[order], atol=1e-12)
    a, b = ft.forward(f, two=True)
    ra, rb = grid.forward(f, two=True)
    np.testing.assert_allclose(a, ra[order], atol=1e-12)
    np.testing.assert_allclose(b, rb[order], atol=1e-12)
    # forward(backward(c)) = c on the sphere
    np.testing.assert_allclose(ft.forward(ft.backward(c1[order])), c1[order], atol=1e-12)
    ft.close()


def test_fourier_transform_complex_basis():
    s = systems.si8k2()
    hkl = s.kmiller(0)
    grid = qbox_np.dense_grid(s.cell, s.ecut)
    ft = capi.FourierTransform(hkl, grid, real_basis=False)
    rng = np.random.default_rng(11)
    c = rng.standard_normal(len(hkl)) + 1j * rng.standard_normal(len(hkl))
    ref, ip = _numpy_backward_complex(hkl, grid, c)
    np.testing.assert_allclose(ft.backward(c), ref, atol=1e-12 * np.abs(ref).max())
    N = grid[0] * grid[1] * grid[2]
    f = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    z = (np.fft.fftn(f.reshape(grid[2], grid[1], grid[0])) / N).ravel()
    np.testing.assert_allclose(ft.forward(f), z[ip], atol=1e-12)
    with pytest.raises(capi.QbxError):
        ft.backward(c, c)          # two-band transforms need a real basis
    ft.close()


def test_fourier_transform_rejects_a_basis_larger_than_the_grid():
    with pytest.raises(capi.QbxError):
        capi.FourierTransform(np.array([[8, 0, 0]]), (16, 16, 16))


@pytest.fixture(scope="module")
def si8_state():
    s = systems.si8()
    es = qbox_np.ElectronicStep(s)
    es.update_density()
    es.update_vhxc()
    es.energy(True, forces=True)
    ctx = capi.from_system(s)
    ctx.update_density()
    ctx.update_vhxc()
    ctx.energy(hpsi=True, forces=True)
    yield s, es, ctx
    ctx.close()


def test_compute_density_and_rs_mul_add(si8_state):
    s, es, ctx = si8_state
    rho = np.full(es.wgrid.N, 0.25)
    ctx.compute_density(0.5, rho)
    np.testing.assert_allclose(rho, 0.25 + 0.5 * es.rhor.ravel(), atol=1e-12)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(es.wgrid.N)
    dc = np.ones((s.nbands, ctx.ngw), complex)
    ctx.rs_mul_add(v, dc)
    ref = np.ones((s.nbands, es.wb.size), complex)
    es.rs_mul_add(v, ref)
    np.testing.assert_allclose(dc, ref, atol=1e-11)


def test_nonlocal_energy_alone(si8_state):
    s, es, ctx = si8_state
    dc = np.zeros((s.nbands, ctx.ngw), complex)
    out = ctx.nonlocal_energy(dc, forces=True, stress=True)
    hc = np.zeros_like(es.c)
    enl, fnl = es.nonlocal_energy(hc, forces=True)
    assert abs(out["enl"] - enl) < 1e-10 * max(1.0, abs(enl))
    np.testing.assert_allclose(dc, hc, atol=1e-11)
    np.testing.assert_allclose(out["fion"], np.concatenate(fnl), atol=1e-10)
    _, parts = ctx.stress()
    np.testing.assert_allclose(out["sigma_enl"], parts["enl"], atol=1e-12)
    # the whole H*psi is kinetic + local + nonlocal
    local = np.zeros_like(dc)
    ctx.rs_mul_add(ctx.vr(), local)
    kin = 0.5 * es.wb.g2[None, :] * es.c
    np.testing.assert_allclose(ctx.get_hpsi(), kin + local + dc, atol=1e-11)


def test_ortho_align_and_dot():
    s = systems.si8()
    rng = np.random.default_rng(5)
    es = qbox_np.ElectronicStep(s)
    c_ref = es.c.copy()
    c = es.c + 0.05 * (rng.standard_normal(es.c.shape) + 1j * rng.standard_normal(es.c.shape))
    ctx = capi.from_system(s, coeffs=c, gram=False)
    d = ctx.dot(c_ref)
    ref = np.trace(es.real_dot(c, c_ref))
    assert abs(d - ref) < 1e-10 * abs(ref)
    ctx.ortho_align(c_ref)
    es.c = c.copy()
    es.ortho_align(c_ref)
    np.testing.assert_allclose(ctx.get_coeffs(), es.c, atol=1e-10)
    ctx.close()


def test_diag_matches_reference():
    """Wavefunction::diag(dwf, true) after three PSDA steps of the 64-atom
    cell (tests/golden/ref_si64_diag.npz, the reference's own run):
    eigenvalues to 1e-10 Ha, rotated coefficients to 1e-7 up to the sign of
    each band (the smallest eigenvalue gap is 7e-4 Ha)."""
    from conftest import golden
    g = golden("si64_diag")
    s = systems.si64()
    ctx = capi.from_system(s)
    for _ in range(int(g["nsteps"])):
        ctx.scf_step()
    ctx.update_density()
    ctx.update_vhxc()
    ctx.energy(hpsi=True)
    w = ctx.diag(eigvec=True)
    np.testing.assert_allclose(w, g["eig"], atol=1e-10)
    c = ctx.get_coeffs()[:, g["g_idx"]]
    ref = g["final_c_bands"]
    sign = np.sign((c.conj() * ref).sum(1).real)
    np.testing.assert_allclose(c * sign[:, None], ref, atol=1e-7)
    ctx.close()
