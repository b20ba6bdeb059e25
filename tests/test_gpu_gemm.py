"""The tcgen05 split-precision GEMM against numpy (FP64) and against the
same split products through cuBLAS, through the C ABI."""
import numpy as np
import pytest

from qbx import capi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context()
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 128, 1000), (128, 256, 4099),
                                   (256, 256, 65543), (1024, 1024, 23848)])
def test_tcgen05_split_gemm(ctx, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n)) / np.sqrt(k)
    ref = a.T @ b
    d_tc = ctx.split_gemm_tn(a, b, backend=1)
    d_cb = ctx.split_gemm_tn(a, b, backend=0)
    scale = np.abs(ref).max()
    # three BF16 split terms: ~2^-16 per product term, random in sign
    assert np.abs(d_tc - ref).max() < 2e-5 * scale + 1e-6
    assert np.abs(d_cb - ref).max() < 2e-5 * scale + 1e-6
    assert np.abs(d_tc - d_cb).max() < 1e-5 * scale + 1e-6


def test_tcgen05_overlap_of_orthonormal_columns(ctx):
    """C^T C of orthonormal columns: off-diagonal error ~1e-8, as the mixed
    path needs for its overlap matrix."""
    rng = np.random.default_rng(3)
    k, n = 20000, 256
    q, _ = np.linalg.qr(rng.standard_normal((k, n)))
    s = ctx.split_gemm_tn(q, q, backend=1)
    off = s - np.diag(np.diag(s))
    assert np.abs(off).max() < 2e-7
    assert np.abs(np.diag(s) - 1.0).max() < 1e-4


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (300, 130, 1000), (145838, 256, 1024),
                                   (1000, 1024, 2048)])
def test_tcgen05_tf32_split_gemm(ctx, m, n, k):
    """TF32 hi/lo splits (kind::tf32), the form of the tall updates: ~22
    significant bits per product term, so FP32-level accuracy; partial tiles
    in m and n."""
    rng = np.random.default_rng(m + 3 * n + k)
    a = rng.standard_normal((k, m)) / np.sqrt(k)
    b = rng.standard_normal((k, n))
    ref = a.T @ b
    d = ctx.split_gemm_tn(a, b, backend=2)
    scale = np.abs(ref).max()
    assert np.abs(d - ref).max() < 2e-6 * scale
