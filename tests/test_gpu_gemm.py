"""The tcgen05 split-precision GEMM against numpy (FP64) and against the
same split products through cuBLAS, through the C ABI."""
import os

import numpy as np
import pytest

from qbx import capi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    """A context whose tcgen05 GEMMs run one CTA per 128 x 128 tile
    (QBX_TC_PAIR=0), the reference for the CTA-pair kernels."""
    os.environ["QBX_TC_PAIR"] = "0"
    try:
        c = capi.Context()
    finally:
        os.environ.pop("QBX_TC_PAIR", None)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_default():
    c = capi.Context()
    yield c
    c.close()


@pytest.fixture(scope="module", params=["1", "2"])
def ctx_pair(request):
    """A context whose tcgen05 GEMMs run on CTA pairs instead of one CTA
    per 128 x 128 tile: 256 x 128 tiles (QBX_TC_PAIR=1) or 256 x 256 tiles
    (QBX_TC_PAIR=2)."""
    os.environ["QBX_TC_PAIR"] = request.param
    try:
        c = capi.Context()
    finally:
        os.environ.pop("QBX_TC_PAIR", None)
    c.pair_mode = request.param
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 128, 1000), (128, 256, 4099),
                                   (256, 256, 65543), (1024, 1024, 23848)])
def test_tcgen05_split_gemm(ctx_default, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n)) / np.sqrt(k)
    ref = a.T @ b
    d_tc = ctx_default.split_gemm_tn(a, b, backend=1)
    d_cb = ctx_default.split_gemm_tn(a, b, backend=0)
    scale = np.abs(ref).max()
    # three BF16 split terms: ~2^-16 per product term, random in sign
    assert np.abs(d_tc - ref).max() < 2e-5 * scale + 1e-6
    assert np.abs(d_cb - ref).max() < 2e-5 * scale + 1e-6
    assert np.abs(d_tc - d_cb).max() < 1e-5 * scale + 1e-6


def test_tcgen05_overlap_of_orthonormal_columns(ctx_default):
    """C^T C of orthonormal columns: off-diagonal error ~1e-8, as the mixed
    path needs for its overlap matrix."""
    rng = np.random.default_rng(3)
    k, n = 20000, 256
    q, _ = np.linalg.qr(rng.standard_normal((k, n)))
    s = ctx_default.split_gemm_tn(q, q, backend=1)
    off = s - np.diag(np.diag(s))
    assert np.abs(off).max() < 2e-7
    assert np.abs(np.diag(s) - 1.0).max() < 1e-4


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 130, 1000), (145838, 256, 1024),
                                   (1000, 1024, 2048)])
def test_tcgen05_tf32_split_gemm(ctx_default, m, n, k):
    """TF32 hi/lo splits (kind::tf32), the form of the tall updates: ~22
    significant bits per product term, so FP32-level accuracy; partial tiles
    in m and n."""
    rng = np.random.default_rng(m + 3 * n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n))
    ref = a.T @ b
    d = ctx_default.split_gemm_tn(a, b, backend=2)
    scale = np.abs(ref).max()
    assert np.abs(d - ref).max() < 2e-6 * scale


@pytest.mark.parametrize("m,n,k,backend", [(128, 128, 64, 1), (384, 256, 5000, 1),
                                           (1024, 1024, 23848, 1), (2048, 1024, 20000, 1),
                                           (300, 130, 1000, 2), (145838, 256, 1024, 2),
                                           (1000, 1024, 2048, 2)])
def test_cta_pair_gemm_matches_single_cta(ctx, ctx_pair, m, n, k, backend):
    """The CTA-pair kernel (cta_group::2, B split between the two CTAs'
    shared memory) gives the one-CTA kernel's products.  With 256 x 128
    tiles it runs the same K blocks in the same accumulation chains, so the
    two agree to 1e-6 of the largest value; with 256 x 256 tiles the
    correction terms share the hi*hi chain, and both stay within the
    split-precision bound of the FP64 product.  The shapes cover an odd
    number of M tiles (the pair's second CTA reads zeros), partial tiles, the
    split-K and the direct (tall update) epilogues, BF16 and TF32."""
    rng = np.random.default_rng(7 * m + n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n)) / np.sqrt(k)
    ref = a.T @ b
    d2 = ctx_pair.split_gemm_tn(a, b, backend=backend)
    d1 = ctx.split_gemm_tn(a, b, backend=backend)
    scale = np.abs(ref).max()
    bound = 2e-5 if backend == 1 else 2e-6
    assert np.abs(d2 - d1).max() <= (1e-6 if ctx_pair.pair_mode == "1" else bound) * scale
    assert np.abs(d2 - ref).max() < bound * scale + 1e-6
    assert np.abs(d1 - ref).max() < bound * scale + 1e-6


@pytest.mark.parametrize("pair", ["1", "2"])
def test_cta_pair_gemm_step_si512_sample(pair, monkeypatch):
    """Two mixed electronic steps of a 32-band sample of the 512-atom cell
    with every tcgen05 GEMM on CTA pairs (the lower-triangle overlaps, the
    split-K inner products, the tall updates) give the one-CTA steps'
    energies to 1e-8 Ha per atom (256 x 128 tiles, the same chains) or
    2e-7 Ha per atom (256 x 256 tiles, corrections in the hi*hi chain), and
    coefficients to 1e-7 or 1e-6."""
    from qbx import systems
    s = systems.si512().band_sample(32)
    etol, ctol = (1e-8, 1e-7) if pair == "1" else (2e-7, 1e-6)
    ctxs = []
    for mode in (pair, "0"):
        monkeypatch.setenv("QBX_TC_PAIR", mode)
        ctxs.append(capi.from_system(s, precision=capi.MIXED))
    monkeypatch.delenv("QBX_TC_PAIR")
    a, b = ctxs
    for _ in range(2):
        ea, eb = a.scf_step(), b.scf_step()
        for key in ("ekin", "enl", "etotal", "eigenvalue_sum"):
            assert abs(ea[key] - eb[key]) <= etol * len(s.atoms), (key, ea[key], eb[key])
    np.testing.assert_allclose(a.get_coeffs(), b.get_coeffs(), rtol=0, atol=ctol)
    a.close()
    b.close()


@pytest.mark.parametrize("m,n,k,backend", [(128, 256, 1024, 3), (145838, 1024, 1024, 3),
                                           (300, 130, 1000, 4), (145838, 1024, 1024, 4),
                                           (1000, 256, 2048, 3)])
def test_tall_update_with_mn_major_a(ctx_default, m, n, k, backend):
    """The tall-update form of the CTA-pair kernel: A read as an MN-major
    operand (its rows contiguous, as the plain split of a wavefunction block
    lies), B K-major.  BF16 (3) and TF32 (4) splits against the FP64
    product, within the split-precision bound; partial tiles and the
    512-atom shape (145 838 rows, 1 024 bands)."""
    rng = np.random.default_rng(11 * m + n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n)) / np.sqrt(k)
    d = ctx_default.split_gemm_tn(a, b, backend=backend)
    ref = a.T @ b
    scale = np.abs(ref).max()
    bound = 2e-5 if backend == 3 else 2e-6
    assert np.abs(d - ref).max() < bound * scale + 1e-6
