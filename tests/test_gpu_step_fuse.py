"""The mixed PSDA step with its fused passes against the same step with each
pass on its own (QBX_STEP_FUSE, read at context creation), through the C ABI.

Fused (the default): energy()'s split of C also forms each band's kinetic
energy for the preconditioner (Preconditioner::update,
src/Preconditioner.cpp:88-143); the captured step forms the eigenvalue sum in
the split of H C; the PSDA step (src/PSDAWavefunctionStepper.cpp:82-212)
writes the cleaned-up new C's BF16 and TF32 splits and the column sums of its
squares that ortho_align reads.  Separate: the one-band-per-CTA
preconditioner kernel, the eigenvalue-sum reduction, the plain PSDA step, the
cleanup and the split kernel.

Only the order of the FP64 sums differs, so energies, theta and C agree to
rounding over several steps: the bounds of the captured-versus-eager test of
the mixed path (1e-9).
"""
import numpy as np
import pytest

from qbx import capi, systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [False, True])
def test_fused_step_matches_separate_passes(monkeypatch, graph):
    s = systems.get("si64")
    monkeypatch.setenv("QBX_STEP_FUSE", "0")
    sep = capi.from_system(s, precision=capi.MIXED)
    monkeypatch.setenv("QBX_STEP_FUSE", "1")
    fus = capi.from_system(s, precision=capi.MIXED)
    if graph:
        sep.set_step_graph(True)
        fus.set_step_graph(True)
    for _ in range(5):
        ea = sep.scf_step()
        eb = fus.scf_step()
        for k in ("etotal", "eigenvalue_sum", "ekin", "enl", "exc"):
            assert abs(ea[k] - eb[k]) <= 1e-9 * max(1.0, abs(ea[k])), (k, ea[k], eb[k])
        assert abs(ea["theta"] - eb["theta"]) <= 1e-9
    ca, cb = sep.get_coeffs(), fus.get_coeffs()
    assert np.abs(ca - cb).max() <= 1e-9
    # C stays orthonormal on the fused path (its overlap's diagonal comes
    # from the PSDA step's column sums): S = 2 Re C^* C^T - c(0) c(0)^T on
    # the half sphere, within the mixed path's 1e-6
    ovl = 2.0 * (cb.conj() @ cb.T).real - np.outer(cb[:, 0].real, cb[:, 0].real)
    assert np.abs(ovl - np.eye(cb.shape[0])).max() <= 1e-6
    assert np.abs(cb[:, 0].imag).max() <= 1e-12   # SlaterDet::cleanup on the new C
    if graph:
        captured, launches, note = fus.step_graph_info()
        assert note == "" and captured >= 1 and launches >= 3, (captured, launches, note)
    sep.close()
    fus.close()
