"""beagleB200UpdatePrePartialsWithDerivatives for 4 < S <= 64 on the FP32
path: the tensor-core fused walk (k_tc.cu k_prederiv_tc; autotuner variant 1
of the fused call, forced here) against the two separate calls on the same
instance and against the oracle.  The state counts cover every padded width
of the tensor-core kernels (N = 16, 32, 48, 64) and both K layouts; tips come
as compact states (with missing states) and as partials; rescaling on and
off; C from 1 to 8 (clusters of up to 8 CTAs); pre-order matrices transposed
by the caller and by the library; a captured graph.  The sibling-pair form
(k_prederiv_tc_pairs, autotuner variant 2, 17 to 32 padded states) against
the single-op walk, the oracle, lists without pairs (variant 1 runs instead)
and a captured graph."""
import numpy as np
import pytest

from helpers import TOL, gpu_flags, grad_err, rel, run_oracle

pytestmark = pytest.mark.gpu

ASYNCH = 1 << 3
FUSED_TC = "-1,-1,-1,1"
FUSED_PAIRS = "-1,-1,-1,2"
SEPARATE = "-1,-1,-1,0"
CASES = [(5, 3), (13, 2), (20, 4), (33, 2), (48, 8), (61, 4), (61, 1)]


def _inst(b200, pr, auto_transpose=False, extra=0):
    pref, req = gpu_flags("single", auto_transpose=auto_transpose)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref | extra, requirementFlags=req)
    pr.load(inst)
    return inst


def _fused(inst, pr, transposed):
    _, sums = pr.evaluate(inst, transposed_pre=transposed, fused=True)
    return inst.getLogLikelihood(), pr.branch_gradient(sums)


@pytest.mark.parametrize("S,C", CASES, ids=[f"S{s}C{c}" for s, c in CASES])
def test_tc_fused_matches_separate_and_oracle(b200, syn, oracle, monkeypatch, S, C):
    # odd C: every tip as partials (1 % ambiguous cells); even C: compact
    # tip states, 5 % of them missing
    pr = syn.make_problem(S=S, N=11, P=900, C=C, seed=900 + S + C, rescale=True,
                          ambiguous=0.01 if C % 2 else 0.0)
    rng = np.random.default_rng(S + C)
    pr.tip_states[rng.random(pr.tip_states.shape) < 0.05] = S
    inst = _inst(b200, pr)
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", SEPARATE)
    l0, g0 = _fused(inst, pr, True)
    pre0 = [inst.getPartials(pr.pre(v)) for v in (0, pr.N, pr.B - 1)]
    sc0 = [inst.getScaleFactors(pr.N - 1 + v) for v in (0, pr.N, pr.B - 1)]
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_TC)
    l1, g1 = _fused(inst, pr, True)
    assert inst.tunedVariants()["fused"] == 1          # the tensor-core fused walk ran
    _, lo, go = run_oracle(oracle, pr)
    tol = TOL["single"]
    assert rel(l1, l0) <= 1e-12
    assert rel(l1, lo) <= tol["lnl"]
    assert grad_err(g1, g0) <= tol["grad"], grad_err(g1, g0)
    assert grad_err(g1, go) <= tol["grad"], grad_err(g1, go)
    # the pre-order partials and scale factors it wrote are the walk's
    for k, v in enumerate((0, pr.N, pr.B - 1)):
        a = inst.getPartials(pr.pre(v))
        assert np.max(np.abs(a - pre0[k])) <= 2e-4 * np.max(np.abs(pre0[k])), v
        s = inst.getScaleFactors(pr.N - 1 + v)
        assert np.max(np.abs(s - sc0[k]) / np.maximum(1.0, np.abs(sc0[k]))) <= 2e-4, v
    inst.finalize()


# Without rescaling only small state counts stay inside FP32's range on these
# trees: 61-state partials of a 9-taxon tree fall to about 1e-42 (subnormal),
# where neither FP32 nor the split products carry 1e-4 relative accuracy.
@pytest.mark.parametrize("S", [13, 20])
def test_tc_fused_without_rescaling_and_auto_transpose(b200, syn, oracle, monkeypatch, S):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_TC)
    pr = syn.make_problem(S=S, N=9, P=513, C=4, seed=950 + S, rescale=False)
    _, lo, go = run_oracle(oracle, pr)
    for auto in (False, True):
        inst = _inst(b200, pr, auto_transpose=auto)
        l1, g1 = _fused(inst, pr, not auto)
        assert inst.tunedVariants()["fused"] == 1
        assert rel(l1, lo) <= TOL["single"]["lnl"]
        assert grad_err(g1, go) <= TOL["single"]["grad"], (auto, grad_err(g1, go))
        inst.finalize()


def test_tc_fused_graph_replay(b200, syn, monkeypatch):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_TC)
    pr = syn.make_problem(S=61, N=10, P=700, C=4, seed=977, rescale=True)
    plain = _inst(b200, pr)
    gi = _inst(b200, pr, extra=ASYNCH)
    graph, grad = pr.capture_step(gi, transposed_pre=True, fused=True)
    rng = np.random.default_rng(3)
    for step in range(3):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(plain, transposed_pre=True, lengths=t)
        l1, _ = pr.evaluate_graph_step(gi, graph, grad, lengths=t)
        assert rel(l1, l0) <= TOL["single"]["lnl"], step
        assert grad_err(pr.branch_gradient(grad), g0) <= TOL["single"]["grad"], step
    plain.finalize()
    gi.finalize()


PAIR_CASES = [(17, 1, 0.01), (20, 4, 0.0), (20, 8, 0.01), (29, 3, 0.0), (32, 2, 0.0)]


@pytest.mark.parametrize("S,C,amb", PAIR_CASES, ids=[f"S{s}C{c}" for s, c, _ in PAIR_CASES])
def test_tc_fused_pairs_match_single_op_walk_and_oracle(b200, syn, oracle, monkeypatch, S, C, amb):
    # tips as compact states with 5 % missing, or with 1 % ambiguous cells as
    # partials; the pair step does per op the arithmetic of the single-op walk
    pr = syn.make_problem(S=S, N=13, P=1100, C=C, seed=700 + S + C, rescale=True, ambiguous=amb)
    rng = np.random.default_rng(S * C)
    pr.tip_states[rng.random(pr.tip_states.shape) < 0.05] = S
    inst = _inst(b200, pr)
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_TC)
    l1, g1 = _fused(inst, pr, True)
    pre1 = [inst.getPartials(pr.pre(v)) for v in (0, pr.N, pr.B - 1)]
    sc1 = [inst.getScaleFactors(pr.N - 1 + v) for v in (0, pr.N, pr.B - 1)]
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_PAIRS)
    l2, g2 = _fused(inst, pr, True)
    assert inst.tunedVariants()["fused"] == 2          # the pair walk ran
    assert rel(l2, l1) <= 1e-12
    assert grad_err(g2, g1) <= 1e-9, grad_err(g2, g1)
    for k, v in enumerate((0, pr.N, pr.B - 1)):
        a = inst.getPartials(pr.pre(v))
        assert np.max(np.abs(a - pre1[k])) <= 1e-6 * np.max(np.abs(pre1[k])), v
        assert np.array_equal(inst.getScaleFactors(pr.N - 1 + v), sc1[k]), v
    _, lo, go = run_oracle(oracle, pr)
    assert rel(l2, lo) <= TOL["single"]["lnl"]
    assert grad_err(g2, go) <= TOL["single"]["grad"], grad_err(g2, go)
    inst.finalize()


def test_tc_fused_pairs_without_rescaling(b200, syn, oracle, monkeypatch):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_PAIRS)
    pr = syn.make_problem(S=20, N=9, P=513, C=4, seed=931, rescale=False)
    _, lo, go = run_oracle(oracle, pr)
    for auto in (False, True):
        inst = _inst(b200, pr, auto_transpose=auto)
        l2, g2 = _fused(inst, pr, not auto)
        assert inst.tunedVariants()["fused"] == 2
        assert rel(l2, lo) <= TOL["single"]["lnl"]
        assert grad_err(g2, go) <= TOL["single"]["grad"], (auto, grad_err(g2, go))
        inst.finalize()


def test_tc_fused_pairs_refuse_lists_without_pairs(b200, syn, monkeypatch):
    """Pre-order ops sorted by depth, then by node, so siblings are not
    adjacent: the pair form refuses the list and the single-op walk runs."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_PAIRS)
    pr = syn.make_problem(S=20, N=30, P=600, C=4, seed=932, rescale=True)
    inst = _inst(b200, pr)
    l0, g0 = pr.evaluate(inst, transposed_pre=True)
    ops = pr.pre_ops(transposed_matrices=True)
    depth = {pr.pre(pr.root): 0}
    for op in ops:
        depth[op[0]] = depth[op[3]] + 1
    ops = ops[np.lexsort((ops[:, 0] % 7, [depth[o[0]] for o in ops]))]
    nodes = ops[:, 0] - pr.pre(0)
    sums, _ = inst.updatePrePartialsWithDerivatives(ops, nodes, np.full(pr.B, pr.B), [0])
    assert inst.tunedVariants()["fused"] == 1
    g1 = np.empty(pr.B)
    g1[nodes] = sums
    assert grad_err(g1, g0) <= TOL["single"]["grad"], grad_err(g1, g0)
    inst.finalize()


def test_tc_fused_pairs_graph_replay(b200, syn, monkeypatch):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", FUSED_PAIRS)
    pr = syn.make_problem(S=20, N=10, P=700, C=4, seed=933, rescale=True)
    plain = _inst(b200, pr)
    gi = _inst(b200, pr, extra=ASYNCH)
    graph, grad = pr.capture_step(gi, transposed_pre=True, fused=True)
    assert gi.tunedVariants()["fused"] == 2
    rng = np.random.default_rng(4)
    for step in range(3):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(plain, transposed_pre=True, lengths=t)
        l1, _ = pr.evaluate_graph_step(gi, graph, grad, lengths=t)
        assert rel(l1, l0) <= TOL["single"]["lnl"], step
        assert grad_err(pr.branch_gradient(grad), g0) <= TOL["single"]["grad"], step
    plain.finalize()
    gi.finalize()
