"""Subtree checkpointing of post-order partials (beagle-lib_b200/checkpoint.py):
the checkpointed schedule, on a pool of a fraction of the full buffer count,
gives the lnL and gradient of the full schedule.  On the CPU through the
oracle (the schedule logic: buffer reuse inside one op list, recomputation,
block order); on the GPU through the C ABI, plain and captured as a graph."""
import numpy as np
import pytest

from helpers import SCALERS_LOG, TOL, gpu_flags, grad_err, rel

ASYNCH = 1 << 3


def _oracle_eval(oracle, args, problem, runner):
    inst = oracle.OracleInstance(*args, flags=SCALERS_LOG)
    problem.load(inst)
    return runner(inst)


@pytest.mark.parametrize("S,N,C,rescale", [(4, 24, 4, True), (4, 17, 1, False),
                                           (5, 12, 2, True)])
def test_checkpointed_schedule_matches_full_on_oracle(pkg, syn, oracle, S, N, C, rescale):
    ck = pkg.checkpoint
    pr = syn.make_problem(S=S, N=N, P=40, C=C, seed=900 + N, rescale=rescale)
    l0, g0 = _oracle_eval(oracle, pr.create_args(), pr, lambda i: pr.evaluate(i))
    full = ck.CheckpointPlan(pr, 1).full_buffers()
    for block in (1, 2, 3, 5, N):
        plan = ck.CheckpointPlan(pr, block)
        l1, g1 = _oracle_eval(oracle, plan.create_args(), pr, lambda i: plan.evaluate(i))
        assert rel(l1, l0) <= 1e-13, (block, l1, l0)
        assert grad_err(g1, g0) <= 1e-12, block
        if 1 < block < N:
            assert plan.n_buffers < full, (block, plan.n_buffers, full)


def test_plan_structure(pkg, syn):
    """Every branch gets one derivative; the pool stays within its size; the
    smallest plan for a 128-taxon tree needs under half the full buffers."""
    ck = pkg.checkpoint
    pr = syn.make_problem(S=4, N=128, P=8, C=1, seed=5)
    plan = ck.smallest_plan(pr)
    seen = np.concatenate([s[1] for s in plan.steps if s[0] == "deriv"])
    assert sorted(seen.tolist()) == list(range(pr.B))
    hi = pr.N + plan.pool
    for s in plan.steps:
        arrs = [s[1]] if s[0] != "deriv" else [s[2], s[3]]
        for a in arrs:
            a = np.asarray(a)
            if a.ndim == 2:
                bufs = a[:, [0, 3, 5]]
            else:
                bufs = a
            assert bufs.max() < hi
    assert plan.n_buffers * 2 < plan.full_buffers()
    fit = ck.plan_for_budget(pr, plan.n_buffers + 20)
    assert fit.n_buffers <= plan.n_buffers + 20 and fit.calls <= plan.calls
    with pytest.raises(ValueError):
        ck.plan_for_budget(pr, pr.N + 2)


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [False, True], ids=["calls", "fused"])
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,N,C", [(4, 40, 4), (20, 20, 2), (61, 12, 4)])
def test_checkpointed_gpu_matches_full(b200, pkg, syn, precision, S, N, C, fused):
    """fused: each block's pre-order walk and derivatives as one
    beagleB200UpdatePrePartialsWithDerivatives call."""
    ck = pkg.checkpoint
    pr = syn.make_problem(S=S, N=N, P=1500, C=C, seed=950 + S, rescale=True)
    pref, req = gpu_flags(precision)
    tr = S > 4
    full = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(full)
    l0, g0 = pr.evaluate(full, transposed_pre=tr)
    plan = ck.smallest_plan(pr, transposed_pre=tr)
    assert plan.n_buffers < plan.full_buffers()
    inst = b200.create(*plan.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(inst)
    l1, g1 = plan.evaluate(inst, fused=fused)
    tol = TOL[precision]
    assert rel(l1, l0) <= tol["lnl"], (l1, l0)
    assert grad_err(g1, g0) <= tol["grad"]
    # captured as one graph on an ASYNCH instance, replayed with new lengths
    gi = b200.create(*plan.create_args(), preferenceFlags=pref | ASYNCH, requirementFlags=req)
    pr.load(gi)
    graph, gradient = plan.capture(gi, fused=fused)
    rng = np.random.default_rng(3)
    for step in range(2):
        t = pr.lengths * (1 + 0.05 * rng.standard_normal(pr.B))
        l0, g0 = pr.evaluate(full, transposed_pre=tr, lengths=t)
        gi.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, t)
        gi.launchGraph(graph)
        l2 = gi.getLogLikelihood()
        assert rel(l2, l0) <= tol["lnl"], (step, l2, l0)
        assert grad_err(gradient(), g0) <= tol["grad"], step
    for x in (full, inst, gi):
        x.finalize()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("variant", [1, 7, 9, 11, 12, 13])
def test_checkpointed_buffer_reuse_each_s4_walk(b200, pkg, syn, monkeypatch, precision, variant):
    """The checkpointed schedule reuses buffers inside one op list (a result's
    buffer becomes a later op's destination): every S = 4 walk shape, the
    level-reordering ones included, must keep those write-after-read orders."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", f"{variant},{variant},1")
    ck = pkg.checkpoint
    pr = syn.make_problem(S=4, N=48, P=700, C=4, seed=77, rescale=True)
    pref, req = gpu_flags(precision)
    full = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(full)
    l0, g0 = pr.evaluate(full)
    plan = ck.CheckpointPlan(pr, 3)
    inst = b200.create(*plan.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(inst)
    l1, g1 = plan.evaluate(inst)
    tol = TOL[precision]
    assert rel(l1, l0) <= tol["lnl"], (l1, l0)
    assert grad_err(g1, g0) <= tol["grad"]
    full.finalize()
    inst.finalize()
