"""The precision form (64-atom PBE cell over 30 PSDA steps) and the batching
form (uneven small cells stepped together) against the reference.

Fixtures come from the reference's own CPU build (tests/golden/make_golden.py):
ref_si64_30.npz holds the energies of 30 PSDA steps of the 64-atom cell,
ref_batch4.npz the energies of two steps of four systems of the 32-system
batch.

Tolerances: FP64 path - every energy term 1e-8 Ha (relative to the term for
terms above 1 Ha) at every step.  Mixed path - 1e-6 Ha/atom at every step
when it evaluates the FP64 path's coefficients (the error the mixed step
makes).  A whole mixed trajectory started from random coefficients follows
the FP64 one only to first order in its step errors: over these 30 steps
the difference wanders between -2e-6 and +1.3e-5 Ha/atom (largest in the
first steps, whatever the product precisions - BF16 or TF32 H*C updates,
short or long accumulation chains), so its last step is held to 5e-6
Ha/atom.
"""
import numpy as np
import pytest

from conftest import golden
from qbx import capi, systems

pytestmark = pytest.mark.gpu

TERMS = ("ekin", "eps", "enl", "ehart", "exc", "esr", "eself", "etotal", "eigenvalue_sum")


def _close(r, g, it, tol=1e-8):
    for k in TERMS:
        ref = g["e_" + k][it]
        assert abs(r[k] - ref) < tol * max(1, abs(ref)), (it, k, r[k], ref)


def test_si64_30_steps_fp64_matches_reference():
    g = golden("si64_30")
    s = systems.si64()
    ctx = capi.from_system(s, precision=capi.FP64)
    for it in range(int(g["nsteps"])):
        _close(ctx.scf_step(), g, it)
    c = ctx.get_coeffs()
    np.testing.assert_allclose(c[:4, g["g_idx"]], g["final_c_bands"], atol=1e-8)
    ctx.close()


def test_si64_30_steps_mixed_against_reference():
    g = golden("si64_30")
    s = systems.si64()
    natoms = len(s.atoms)
    nsteps = int(g["nsteps"])
    f64 = capi.from_system(s, precision=capi.FP64)
    same_c = capi.from_system(s, precision=capi.MIXED)
    traj = capi.from_system(s, precision=capi.MIXED)
    worst_same = 0.0
    for it in range(nsteps):
        same_c.set_coeffs(f64.get_coeffs())
        ra = f64.scf_step()
        rb = same_c.scf_step()
        worst_same = max(worst_same, abs(rb["etotal"] - g["e_etotal"][it]) / natoms)
        assert abs(ra["etotal"] - g["e_etotal"][it]) < 1e-8
        rt = traj.scf_step()
    assert worst_same < 1e-6, worst_same
    assert abs(rt["etotal"] - g["e_etotal"][-1]) / natoms < 5e-6, (rt["etotal"], g["e_etotal"][-1])
    for c in (f64, same_c, traj):
        c.close()


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_batch_systems_match_reference(precision):
    """Four systems of the batch (8-64 atoms, 20-30 Ry, bands = 2 x atoms)
    stepped together by qbx_scf_step_batch, each captured as a graph from
    its second step, against the reference run of each alone."""
    g = golden("batch4")
    allsys = systems.batch()
    picked = [int(i) for i in g["picked"]]
    ctxs = [capi.from_system(allsys[i], precision=precision) for i in picked]
    for c in ctxs:
        c.set_step_graph(True)
    for it in range(int(g["nsteps"])):
        rs = capi.scf_step_batch(ctxs)
        for i, r in zip(picked, rs):
            gi = {k[len(f"s{i}_"):]: v for k, v in g.items() if k.startswith(f"s{i}_")}
            if precision == capi.FP64:
                _close(r, gi, it)
            elif it == 0:
                # the first step evaluates the reference's own starting
                # coefficients
                natoms = len(allsys[i].atoms)
                assert abs(r["etotal"] - gi["e_etotal"][0]) / natoms < 1e-6, (i, r["etotal"])
    for c in ctxs:
        c.close()
