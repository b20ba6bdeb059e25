"""qbx_density_static, the density entry point that allocates no device
memory, against the context's own qbx_update_density.

Callers that cannot call cudaMalloc when they need the density (a host
callback, a plug-in inside another framework that has already divided the
device memory) hand the library their own device coefficients and density
grid; the stick scratch comes from a static device array inside the
library.  This file is named to be collected last, so that a run stopping at
its first failure has already run every other test.

Tolerance: the FP64 density matches the existing entry point to 1e-12 of
its maximum (only the twiddle tables differ: computed on the device here,
on the host there), the mixed-precision density to 2e-6, as the other
mixed-precision density tests allow.
"""
import numpy as np
import pytest

from qbx import capi, systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,precision", [("si8", capi.FP64), ("si64", capi.FP64),
                                            ("si64", capi.MIXED)])
def test_density_static_matches_update_density(name, precision):
    import torch
    s = systems.get(name)
    ctx = capi.from_system(s, precision=precision)
    ctx.update_density()
    ref = ctx.density()
    # the coefficients in the library's default order, in caller-owned
    # device memory
    ctx.set_coeff_order(None)
    c = torch.from_numpy(ctx.get_coeffs().view(np.float64).copy()).cuda()
    rho = torch.empty(ref.size, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    tol = (1e-12 if precision == capi.FP64 else 2e-6) * np.abs(ref).max()
    for _ in range(2):
        rho.fill_(np.nan)
        torch.cuda.synchronize()
        ctx.density_static(c.data_ptr(), s.nbands, rho.data_ptr())
        np.testing.assert_allclose(rho.cpu().numpy(), ref, rtol=0, atol=tol)
    # explicit occupations: one electron less in the last band
    occ = np.full(s.nbands, 2.0)
    occ[-1] = 1.0
    ctx.density_static(c.data_ptr(), s.nbands, rho.data_ptr(), occ)
    omega = abs(np.linalg.det(np.asarray(s.cell, float)))
    q = rho.sum().item() * omega / ref.size
    qtol = (1e-9 if precision == capi.FP64 else 1e-6) * s.nel
    assert abs(q - (s.nel - 1.0)) < qtol, q
    ctx.close()


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_density_static_odd_band_count_allocates_nothing(precision):
    """nst = nbands - 1 (odd): the last band pair has one band.  The result
    must equal qbx_update_density of a context holding those nst bands, and
    after the first call (which may load the library's kernels) a call must
    leave the device's free memory unchanged."""
    import dataclasses
    import torch
    s = systems.si64()
    ctx = capi.from_system(s, precision=precision)
    ctx.set_coeff_order(None)
    c_all = ctx.get_coeffs()
    nst = s.nbands - 1
    s_odd = dataclasses.replace(s, nbands=nst, nel_override=2 * nst)
    ref_ctx = capi.from_system(s_odd, precision=precision, coeffs=None, gram=False)
    ref_ctx.set_coeff_order(None)
    ref_ctx.set_coeffs(c_all[:nst])
    ref_ctx.update_density()
    ref = ref_ctx.density()
    ref_ctx.close()
    c = torch.from_numpy(c_all[:nst].view(np.float64).copy()).cuda()
    rho = torch.empty(ref.size, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    tol = (1e-12 if precision == capi.FP64 else 2e-6) * np.abs(ref).max()
    ctx.density_static(c.data_ptr(), nst, rho.data_ptr())
    for _ in range(2):
        rho.fill_(np.nan)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        ctx.density_static(c.data_ptr(), nst, rho.data_ptr())
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
        np.testing.assert_allclose(rho.cpu().numpy(), ref, rtol=0, atol=tol)
    with pytest.raises(ValueError, match="occupations"):
        ctx.density_static(c.data_ptr(), nst, rho.data_ptr(), np.full(s.nbands, 2.0))
    ctx.close()


def test_density_static_rejects_bad_arguments():
    s = systems.si8()
    ctx = capi.from_system(s)
    with pytest.raises(capi.QbxError, match="null"):
        ctx.density_static(0, s.nbands, 0)
    ctx.close()
