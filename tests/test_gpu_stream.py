"""The streamed SlaterDet (qbx_stream_in / qbx_scf_step_async /
qbx_stream_out / qbx_stream_wait): coefficients in pinned host memory pass
through the GPU each step with the copies on their own streams.  Each step's
downloaded result equals the synchronous API's (set, step, get) from the same
inputs, captured or not."""
import numpy as np
import pytest
import torch

from qbx import capi, systems

pytestmark = pytest.mark.gpu


def _pinned(n):
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()


@pytest.mark.parametrize("graph", [True, False])
def test_streamed_steps_equal_synchronous_steps(graph):
    s = systems.si64()
    a = capi.from_system(s, precision=capi.MIXED)
    b = capi.from_system(s, precision=capi.MIXED)
    for ctx in (a, b):
        ctx.set_step_graph(graph)
        for _ in range(3):             # capture and warm both the same way
            ctx.scf_step()
    c0 = b.get_coeffs()
    a.set_coeffs_async(np.ascontiguousarray(c0).view(np.float64))   # same start, history kept
    nf = c0.size * 2
    pin_in = _pinned(nf)
    pin_in[:] = c0.view(np.float64).ravel()
    outs = [_pinned(nf) for _ in range(3)]
    for i in range(3):
        a.stream_in(pin_in)
        a.scf_step_async()
        a.stream_out(outs[i])
    ea = a.stream_wait()
    for i in range(3):
        b.set_coeffs_async(np.ascontiguousarray(c0).view(np.float64))
        eb = b.scf_step()
        cb = b.get_coeffs()
        ca = outs[i].view(np.complex128).reshape(cb.shape)
        np.testing.assert_allclose(ca, cb, rtol=0, atol=1e-13)
    for k in ("ekin", "enl", "etotal", "eigenvalue_sum"):
        assert abs(ea[k] - eb[k]) < 1e-10, (k, ea[k], eb[k])
    a.close()
    b.close()
