"""CUDA graphs of an instance's evaluation (beagleB200BeginCapture /
EndCapture / LaunchGraph): partials, scaling, root lnL, pre-order partials and
edge derivatives captured once, then per step new transition matrices and a
graph launch; or the whole step with the matrices, launched with new branch
lengths (beagleB200LaunchGraphWithLengths) -- against plain evaluations with
the same branch lengths."""
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


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,C,fused", [(4, 4, False), (4, 4, True), (20, 2, False)])
def test_whole_step_graph_with_new_lengths(b200, syn, precision, S, C, fused):
    """The transition-matrix update captured too: the graph reads the branch
    lengths on the device, and beagleB200LaunchGraphWithLengths replaces them
    per step (one call and one wait a step); a count that does not match the
    capture is refused; plain LaunchGraph replays the lengths last given."""
    pr = syn.make_problem(S=S, N=14, P=900, C=C, seed=90 + S, rescale=True)
    pref, req = gpu_flags(precision)
    plain = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    graphed = b200.create(*pr.create_args(), preferenceFlags=pref | ASYNCH,
                          requirementFlags=req)
    for x in (plain, graphed):
        pr.load(x)
    tr = S > 4
    graph, grad = pr.capture_step(graphed, transposed_pre=tr, fused=fused)
    rng = np.random.default_rng(2)
    tol = TOL[precision]
    for step in range(4):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(plain, transposed_pre=tr, lengths=t, fused=fused)
        l1, g1 = pr.evaluate_graph_step(graphed, graph, grad, lengths=t)
        if fused:
            g0, g1 = pr.branch_gradient(g0), pr.branch_gradient(g1)
        assert rel(l1, l0) <= (1e-13 if precision == "double" else tol["lnl"]), (step, l1, l0)
        assert grad_err(g1, g0) <= tol["grad"], step
    with pytest.raises(Exception):
        graphed.launchGraphWithLengths(graph, pr.lengths[:-1])
    # plain replay: the lengths last given (here the last step's)
    l2, _ = pr.evaluate(plain, transposed_pre=tr, lengths=t, fused=fused)
    graphed.launchGraph(graph)
    assert rel(graphed.getLogLikelihood(), l2) <= (1e-13 if precision == "double" else tol["lnl"])
    plain.finalize()
    graphed.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_graph_lengths_buffer_reusable_at_once(b200, syn, precision):
    """beagleB200LaunchGraphWithLengths copies the lengths on the host before
    it returns, pinned memory included: a caller that writes the next step's
    lengths into the same pinned buffer right after the call (before any
    wait), several launches deep, still gets each launch's own lengths."""
    import torch
    pr = syn.make_problem(S=4, N=12, P=700, C=4, seed=97, rescale=True)
    pref, req = gpu_flags(precision)
    plain = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    graphed = b200.create(*pr.create_args(), preferenceFlags=pref | ASYNCH,
                          requirementFlags=req)
    for x in (plain, graphed):
        pr.load(x)
    graph, grad = pr.capture_step(graphed, fused=True)
    buf = torch.empty(pr.B, dtype=torch.float64).pin_memory().numpy()
    rng = np.random.default_rng(4)
    steps = [pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B)) for _ in range(6)]
    for t in steps:                       # six launches queued, the buffer reused each time
        buf[:] = t
        graphed.launchGraphWithLengths(graph, buf)
        buf[:] = 123.0                    # overwritten before the launch could have run
    lnl_last = graphed.getLogLikelihood()  # the last launch's result
    l0, _ = pr.evaluate(plain, lengths=steps[-1], fused=True)
    tol = 1e-13 if precision == "double" else TOL[precision]["lnl"]
    assert rel(lnl_last, l0) <= tol, (lnl_last, l0)
    plain.finalize()
    graphed.finalize()
