"""beagleB200UpdatePrePartialsWithDerivatives: the pre-order walk and the edge
derivatives of its branches in one kernel (4-state) against the two separate
calls and the oracle, for every category count the fused walk takes, tips as
states and as partials, with and without rescaling; lists without sibling
pairs, lists longer than one launch takes, other state counts (run as the
separate calls), and a captured graph."""
import numpy as np
import pytest

from helpers import TOL, gpu_flags, grad_err, rel, run_oracle

pytestmark = pytest.mark.gpu

ASYNCH = 1 << 3


def _pair(b200, pr, precision, **kw):
    pref, req = gpu_flags(precision)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref | kw.get("extra", 0),
                       requirementFlags=req)
    pr.load(inst)
    return inst


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("C,rescale,amb", [(1, True, 0.0), (2, False, 0.03), (4, True, 0.03),
                                           (8, True, 0.0)])
@pytest.mark.parametrize("form", [1, 2, 3])
def test_fused_matches_separate_calls_and_oracle(b200, syn, oracle, monkeypatch, precision, C,
                                                 rescale, amb, form):
    """form 1: the fused walk; 2: its pairs-only, 2-patterns-a-thread form
    (FP32 only: an FP64 instance forced to it runs form 1); 3: the fused walk
    with its matrices staged in shared memory."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", f"-1,-1,-1,{form}")
    pr = syn.make_problem(S=4, N=33, P=1300, C=C, seed=500 + C, rescale=rescale, ambiguous=amb)
    inst = _pair(b200, pr, precision)
    l0, g0 = pr.evaluate(inst)
    l1, sums = pr.evaluate(inst, fused=True)
    g1 = pr.branch_gradient(sums)
    _, lo, go = run_oracle(oracle, pr)
    tol = TOL[precision]
    # the fused post-order call: its FP64 sums run in another order, and the
    # separate call's autotuner may have picked another post-order kernel shape
    assert rel(l1, l0) <= (1e-13 if precision == "double" else 1e-6)
    assert grad_err(g1, g0) <= tol["grad"] * 1e-2, grad_err(g1, g0)
    assert grad_err(g1, go) <= tol["grad"], grad_err(g1, go)
    # the pre-order buffers the fused walk wrote are the separate walk's, up to
    # the rounding of a different FMA order: a few ulp per op, compounded over
    # the tree's depth (relative, or absolute below the smallest normal number)
    ulps, tiny = (1e-13, 1e-300) if precision == "double" else (1e-5, 1.2e-38)
    for v in (0, pr.N, pr.B - 1):
        pr.evaluate(inst, fused=True)
        a = inst.getPartials(pr.pre(v))
        pr.evaluate(inst)
        b = inst.getPartials(pr.pre(v))
        assert np.all(np.abs(a - b) <= ulps * np.abs(b) + tiny), v
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("form", [1, 3])
def test_fused_without_sibling_pairs(b200, syn, monkeypatch, precision, form):
    """Pre-order ops sorted by depth, then by node: siblings are not adjacent,
    so every op runs on its own (three loads, one store)."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", f"-1,-1,-1,{form}")
    pr = syn.make_problem(S=4, N=40, P=900, C=4, seed=61, rescale=True)
    inst = _pair(b200, pr, precision)
    l0, g0 = pr.evaluate(inst)
    ops = pr.pre_ops()
    depth = {pr.pre(pr.root): 0}
    for op in ops:
        depth[op[0]] = depth[op[3]] + 1
    ops = ops[np.lexsort((ops[:, 0] % 7, [depth[o[0]] for o in ops]))]
    adjacent = sum(1 for a, b in zip(ops, ops[1:]) if a[3] == b[3])
    assert adjacent < len(ops) // 4
    nodes = ops[:, 0] - pr.pre(0)
    sums, _ = inst.updatePrePartialsWithDerivatives(ops, nodes, np.full(pr.B, pr.B), [0])
    assert inst.tunedVariants()["fused"] == form
    g1 = np.empty(pr.B)
    g1[nodes] = sums
    assert grad_err(g1, g0) <= TOL[precision]["grad"] * 1e-2
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,N,form", [(4, 150, 1), (4, 300, 1), (4, 150, 3), (4, 300, 3),
                                      (20, 12, 1)])
def test_fused_long_lists_and_other_state_counts(b200, syn, oracle, monkeypatch, precision, S,
                                                 N, form):
    """More than 256 ops (N = 150: 298; N = 300: 598): the fused walk (forced,
    form 1 or the staged form 3, whose shared-memory chunks are also cut
    between sibling pairs) runs as consecutive launches cut between sibling
    pairs.  S = 20 runs the
    tensor-core fused walk in FP32 (its derivative from the unscaled row and
    split products, so it agrees with the separate calls to the mixed path's
    tolerance) and the two separate calls in FP64.  Same results as the
    separate calls and the oracle."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", f"-1,-1,-1,{form}")
    pr = syn.make_problem(S=S, N=N, P=500, C=4, seed=7 + S + N, rescale=True)
    inst = _pair(b200, pr, precision)
    tr = S > 4
    l0, g0 = pr.evaluate(inst, transposed_pre=tr)
    l1, sums = pr.evaluate(inst, transposed_pre=tr, fused=True)
    g1 = pr.branch_gradient(sums)
    tol = TOL[precision]
    # the fused post-order call: its FP64 sums run in another order, and the
    # separate call's autotuner may have picked another post-order kernel shape
    assert rel(l1, l0) <= (1e-13 if precision == "double" else 1e-6)
    assert grad_err(g1, g0) <= (1e-12 if precision == "double" else
                                tol["grad"] * (1e-2 if S == 4 else 1.0))
    if S == 4:
        assert inst.tunedVariants()["fused"] == form   # the fused walk ran
    _, lo, go = run_oracle(oracle, pr)
    assert rel(l1, lo) <= tol["lnl"]
    assert grad_err(g1, go) <= tol["grad"]
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_fused_graph_replay(b200, syn, precision):
    pr = syn.make_problem(S=4, N=30, P=2000, C=4, seed=88, rescale=True)
    plain = _pair(b200, pr, precision)
    gi = _pair(b200, pr, precision, extra=ASYNCH)
    graph, raw = pr.capture(gi, fused=True)
    rng = np.random.default_rng(2)
    tol = TOL[precision]
    for step in range(3):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(plain, lengths=t)
        l1, _ = pr.evaluate_graph(gi, graph, raw, lengths=t)
        assert rel(l1, l0) <= tol["lnl"], step
        assert grad_err(pr.branch_gradient(raw), g0) <= tol["grad"], step
    plain.finalize()
    gi.finalize()
