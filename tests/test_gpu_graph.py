"""The electronic step captured as a CUDA graph (qbx_set_step_graph) against
the same step run eagerly, through the C ABI.

A captured step replays the eager step's kernels in the same order with the
same arguments; the differences are that its scalars stay on the device
(Anderson theta formed there, the polar iteration decided by conditional
graph nodes) and are read back once at the end.  The energies of every step
and the final coefficients therefore agree to rounding: 1e-12 relative on
the total energy and eigenvalue sum, 1e-12 absolute on C (FP64) and the same
bounds times 1e3 for the mixed path, whose split-K GEMM partial sums may be
added in another order by cuBLAS's graph-captured algorithms.
"""
import numpy as np
import pytest

from qbx import capi, systems

pytestmark = pytest.mark.gpu


def _pair(s, precision):
    a = capi.from_system(s, precision=precision)
    b = capi.from_system(s, precision=precision)
    b.set_step_graph(True)
    return a, b


@pytest.mark.parametrize("name,precision", [("si8", capi.FP64), ("si64", capi.FP64),
                                            ("si64", capi.MIXED)])
def test_graph_step_matches_eager(name, precision):
    s = systems.get(name)
    eager, graph = _pair(s, precision)
    tol = 1e-12 if precision == capi.FP64 else 1e-9
    for _ in range(5):
        ea = eager.scf_step()
        eb = graph.scf_step()
        for k in ("etotal", "eigenvalue_sum", "ekin", "enl", "exc"):
            assert abs(ea[k] - eb[k]) <= tol * max(1.0, abs(ea[k])), (k, ea[k], eb[k])
        assert abs(ea["theta"] - eb["theta"]) <= 1e-9
    ca, cb = eager.get_coeffs(), graph.get_coeffs()
    assert np.abs(ca - cb).max() <= (1e-12 if precision == capi.FP64 else 1e-9)
    captured, launches, note = graph.step_graph_info()
    assert note == "", note
    # configurations: first step (no extrapolation) runs eagerly once; the
    # extrapolated step is captured on its second use and launched from then on
    assert captured >= 1 and launches >= 3, (captured, launches)
    eager.close()
    graph.close()


def test_graph_step_with_forces():
    """The forces variant of the captured step: forces read back from the
    graph's pinned copy equal the eager step's."""
    s = systems.get("si8")
    eager, graph = _pair(s, capi.FP64)
    for _ in range(4):
        ea = eager.scf_step(forces=True)
        eb = graph.scf_step(forces=True)
        assert abs(ea["etotal"] - eb["etotal"]) <= 1e-12 * abs(ea["etotal"])
        np.testing.assert_allclose(eb["fion"], ea["fion"], rtol=0, atol=1e-12)
    captured, launches, note = graph.step_graph_info()
    assert note == "" and captured >= 1 and launches >= 2, (captured, launches, note)
    eager.close()
    graph.close()


@pytest.mark.parametrize("single_graph", [False, True])
def test_graph_batch_paths(single_graph, monkeypatch):
    """With every context's step captured, qbx_scf_step_batch launches each
    context's graph from one thread, or (QBX_BATCH_GRAPH=1) one graph whose
    branches are the contexts' steps; either way the energies equal
    stepping each context eagerly."""
    systs = systems.batch()[:6]
    if single_graph:
        monkeypatch.setenv("QBX_BATCH_GRAPH", "1")
    ctxs = [capi.from_system(s, precision=capi.FP64) for s in systs]
    monkeypatch.delenv("QBX_BATCH_GRAPH", raising=False)
    ref = [capi.from_system(s, precision=capi.FP64) for s in systs]
    for c in ctxs:
        c.set_step_graph(True)
    for it in range(5):
        eb = capi.scf_step_batch(ctxs)
        es = [c.scf_step() for c in ref]
        for a, b in zip(eb, es):
            assert abs(a["etotal"] - b["etotal"]) < 1e-10 * max(1.0, abs(b["etotal"]))
            assert abs(a["eigenvalue_sum"] - b["eigenvalue_sum"]) < 1e-9 * max(1.0, abs(b["eigenvalue_sum"]))
    for c in ctxs:
        captured, launches, note = c.step_graph_info()
        assert note == "" and captured >= 1 and launches >= 2, (captured, launches, note)
    batch_launches = ctxs[0].step_graph_info_full()[2]
    if single_graph:
        assert batch_launches >= 2      # the steps ran as branches of one graph
    else:
        assert batch_launches == 0
    for c in ctxs + ref:
        c.close()


def test_graph_dropped_on_atoms_change():
    """Moving the atoms re-uploads the geometry and drops the captured
    graphs; stepping continues (eagerly, then captured again)."""
    s = systems.get("si8")
    ctx = capi.from_system(s, precision=capi.FP64)
    ctx.set_step_graph(True)
    for _ in range(3):
        ctx.scf_step()
    assert ctx.step_graph_info()[0] >= 1
    counts = [len(s.positions(i)) for i in range(len(s.species))]
    tau = np.concatenate([s.positions(i) for i in range(len(s.species))])
    tau = tau + 0.01 * np.random.default_rng(7).standard_normal(tau.shape)
    ctx.set_atoms(counts, tau)
    assert ctx.step_graph_info()[0] == 0
    for _ in range(3):
        ctx.scf_step()
    assert ctx.step_graph_info()[0] >= 1
    ctx.close()


def _polar_cases(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    near = q + 0.02 * rng.standard_normal((n, n)) / np.sqrt(n)      # ||I - x^T x|| < 1
    far = q @ np.diag(np.linspace(0.3, 2.5, n)) @ q.T               # Higham steps first
    return {"bjorck": near, "higham": far}


@pytest.mark.parametrize("name", ["si8", "si64"])
@pytest.mark.parametrize("graph", [False, True])
def test_polar_matches_oracle(name, graph):
    """qbx_polar (DoubleMatrix::polar) against the oracle's restatement, in
    both branches, eagerly and as a graph with conditional nodes."""
    from oracle import qbox_np
    s = systems.get(name)
    ctx = capi.from_system(s, precision=capi.FP64)
    for kind, x in _polar_cases(s.nbands, 11).items():
        ref = qbox_np.polar(x.copy(), 1e-6, 20)
        got, iters = ctx.polar(x, 1e-6, 20, graph=graph)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10, err_msg=kind)
        assert np.abs(got.T @ got - np.eye(s.nbands)).max() < 1e-9, kind
        assert 1 <= iters <= 20, (kind, iters)
    ctx.close()


@pytest.mark.parametrize("graph", [False, True])
def test_polar_mixed_higham_by_cholesky(graph):
    """The mixed path's Higham steps form x^-T from the Cholesky factor of
    x^T x instead of a pivoted LU of x^T: the polar factor is the oracle's
    to 1e-8 and orthogonal to 1e-9, for the near-orthogonal case, the
    symmetric one (polar factor I) and a rotated one with singular values
    from 0.1 to 3, eagerly and captured."""
    from oracle import qbox_np
    s = systems.get("si64")
    ctx = capi.from_system(s, precision=capi.MIXED)
    n = s.nbands
    cases = _polar_cases(n, 11)
    rng = np.random.default_rng(5)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    cases["rotated"] = u @ np.diag(np.linspace(0.1, 3.0, n)) @ v.T
    for kind, x in cases.items():
        ref = qbox_np.polar(x.copy(), 1e-6, 20)
        got, iters = ctx.polar(x, 1e-6, 20, graph=graph)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-8, err_msg=kind)
        assert np.abs(got.T @ got - np.eye(n)).max() < 1e-9, kind
        assert 1 <= iters <= 20, (kind, iters)
    ctx.close()
