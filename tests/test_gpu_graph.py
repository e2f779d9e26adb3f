"""CUDA graphs of an instance's evaluation (beagleB200BeginCapture /
EndCapture / LaunchGraph): partials, scaling, root lnL, pre-order partials and
edge derivatives captured once, then per step new transition matrices and a
graph launch, against plain evaluations with the same branch lengths."""
import numpy as np
import pytest

from helpers import TOL, grad_err, gpu_flags, rel

pytestmark = pytest.mark.gpu

ASYNCH = 1 << 3


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,C", [(4, 4), (20, 2)])
def test_graph_replay_matches_plain_evaluation(b200, syn, precision, S, C):
    pr = syn.make_problem(S=S, N=14, P=900, C=C, seed=70 + S, rescale=True)
    pref, req = gpu_flags(precision)
    plain = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    graphed = b200.create(*pr.create_args(), preferenceFlags=pref | ASYNCH,
                          requirementFlags=req)
    for x in (plain, graphed):
        pr.load(x)
    tr = S > 4
    graph, grad = pr.capture(graphed, transposed_pre=tr)
    rng = np.random.default_rng(1)
    tol = TOL[precision]
    for step in range(4):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(plain, transposed_pre=tr, lengths=t)
        l1, g1 = pr.evaluate_graph(graphed, graph, grad, lengths=t)
        assert rel(l1, l0) <= tol["lnl"], (step, l1, l0)
        assert grad_err(g1, g0) <= tol["grad"], step
    # a call that waits for results is refused while capturing
    graphed.beginCapture()
    with pytest.raises(Exception):
        graphed.getLogLikelihood()
    graphed.endCapture()
    plain.finalize()
    graphed.finalize()
