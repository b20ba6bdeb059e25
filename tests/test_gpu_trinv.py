"""The inverse of a lower-triangular Cholesky factor that ortho_align and the
polar iteration's Cholesky step use on the mixed path (qbx_lower_inverse):
blocked for n = 32 x a power of two (32 x 32 diagonal inverses by forward
substitution, then FP64 GEMMs doubling the block), a triangular solve of I
otherwise.  Checked against numpy's inverse of the same factor, with NaN in
the upper triangle (which must not be read).
"""
import numpy as np
import pytest

from qbx import capi, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.from_system(systems.get("si8"), precision=capi.MIXED)
    yield c
    c.close()


def _factor(n, spread, seed):
    """Cholesky factor of an SPD matrix with eigenvalues spread over
    [1, spread], NaN above the diagonal."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = q @ np.diag(np.geomspace(1.0, spread, n)) @ q.T
    l = np.linalg.cholesky(0.5 * (s + s.T))
    l[np.triu_indices(n, 1)] = np.nan
    return l


@pytest.mark.parametrize("n", [32, 64, 128, 1024, 96, 100])
@pytest.mark.parametrize("spread", [1.5, 1e4])
def test_lower_inverse_matches_numpy(ctx, n, spread):
    l = _factor(n, spread, n)
    got, blocked = ctx.lower_inverse(l)
    assert blocked == (n in (32, 64, 128, 1024))
    lc = np.tril(np.nan_to_num(l, nan=0.0))
    ref = np.linalg.inv(lc)
    assert np.isfinite(got).all()
    assert np.all(got[np.triu_indices(n, 1)] == 0.0)
    # both inverses carry the factor's condition number (sqrt(spread))
    # times the rounding unit
    tol = 64 * np.sqrt(spread) * np.finfo(float).eps * np.abs(ref).max()
    assert np.abs(got - ref).max() <= tol, (np.abs(got - ref).max(), tol)
    assert np.abs(got @ lc - np.eye(n)).max() <= 64 * np.sqrt(spread) * np.finfo(float).eps * n
