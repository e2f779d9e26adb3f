"""Batched calls (beagleB200Batch*): a heterogeneous batch of trees (4 and
20 states; 1, 3, 4 and 8 categories; uneven tree sizes and pattern counts)
evaluated with one batched call per step, against the same problems evaluated
one instance at a time and against the oracle."""
import numpy as np
import pytest

from helpers import TOL, grad_err, gpu_flags, rel, run_oracle

pytestmark = pytest.mark.gpu


def _problems(syn):
    probs = syn.batched_problems(count=10, seed=7, max_patterns=3000)
    # members the batched kernels do not take (3 categories; 20 states) run
    # their single-instance launches on the batch's stream
    probs.append(syn.make_problem(S=4, N=11, P=500, C=3, seed=3, rescale=True))
    probs.append(syn.make_problem(S=20, N=9, P=300, C=4, seed=4, rescale=True))
    return probs


def _create(b200, pr, precision, asynch=False):
    pref, req = gpu_flags(precision, auto_transpose=True)
    if asynch:
        pref |= 1 << 3                      # BEAGLE_FLAG_COMPUTATION_ASYNCH
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(inst)
    return inst


@pytest.mark.parametrize("asynch", [False, True], ids=["synch", "asynch"])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_matches_single_instances_and_oracle(b200, pkg, syn, oracle, precision, asynch):
    """ASYNCH members: the batched result calls defer their values to
    beagleB200BatchWait (batch_evaluate calls it at the end of a step)."""
    probs = _problems(syn)
    singles = [_create(b200, pr, precision) for pr in probs]
    ref = [pr.evaluate(inst, transposed_pre=False) for pr, inst in zip(probs, singles)]
    members = [_create(b200, pr, precision, asynch) for pr in probs]
    batch = pkg.binding.Batch(b200, members)
    for rep in range(2):                    # the second pass reuses the batch's tables
        lnl, grads = syn.batch_evaluate(batch, probs)
        tol = TOL[precision]
        for k, (pr, (l1, g1)) in enumerate(zip(probs, ref)):
            assert rel(lnl[k], l1) <= (1e-12 if precision == "double" else tol["lnl"]), k
            assert grad_err(grads[k], g1) <= (1e-10 if precision == "double" else tol["grad"]), k
    for k in (0, 3, len(probs) - 1):
        _, lo, go = run_oracle(oracle, probs[k])
        assert rel(lnl[k], lo) <= TOL[precision]["lnl"]
        assert grad_err(grads[k], go) <= TOL[precision]["grad"]
    batch.finalize()
    # members work on their own streams again (an ASYNCH instance delivers
    # its lnL through getLogLikelihood)
    l_after, _ = probs[0].evaluate(members[0], transposed_pre=False)
    if asynch:
        l_after = members[0].getLogLikelihood()
    assert rel(l_after, ref[0][0]) <= 1e-6
    for x in singles + members:
        x.finalize()


def test_batch_rejects_bad_members(b200, pkg, syn):
    pr = syn.make_problem(S=4, N=6, P=100, C=2, seed=1)
    a = _create(b200, pr, "double")
    b = _create(b200, pr, "single")
    with pytest.raises(pkg.binding.BeagleError):
        pkg.binding.Batch(b200, [a, b])          # mixed precision
    batch = pkg.binding.Batch(b200, [a])
    with pytest.raises(pkg.binding.BeagleError):
        pkg.binding.Batch(b200, [a])             # already in a batch
    batch.finalize()
    a.finalize()
    b.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_graph_replay(b200, pkg, syn, precision):
    """One batched evaluation captured as a CUDA graph of the batch (batched
    kernels, the 3-category and 20-state members' own launches, uploads and
    result copies), replayed with new branch lengths against plain batched
    evaluations of a second batch."""
    probs = _problems(syn)
    plain = pkg.binding.Batch(b200, [_create(b200, pr, precision, True) for pr in probs])
    graphed = pkg.binding.Batch(b200, [_create(b200, pr, precision, True) for pr in probs])
    graph, lnl_g, sums_g = syn.batch_capture(graphed, probs)
    rng = np.random.default_rng(5)
    tol = TOL[precision]
    for step in range(3):
        ts = [p.lengths * (1 + 0.05 * rng.standard_normal(p.B)) for p in probs]
        lnl0, sums0 = syn.batch_evaluate(plain, probs, lengths=ts)
        syn.batch_evaluate_graph(graphed, probs, graph, lengths=ts)
        for i in range(len(probs)):
            assert rel(lnl_g[i], lnl0[i]) <= tol["lnl"], (step, i)
            assert grad_err(sums_g[i], sums0[i]) <= tol["grad"], (step, i)
    # a result call that would wait is refused while capturing
    graphed.beginCapture()
    with pytest.raises(Exception):
        graphed.wait()
    graphed.endCapture()
    plain.finalize()
    graphed.finalize()


@pytest.mark.parametrize("fused", [False, True], ids=["calls", "fused"])
@pytest.mark.parametrize("asynch", [False, True], ids=["synch", "asynch"])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_checkpointed_matches_single_instances(b200, pkg, syn, precision, asynch, fused):
    """Every member with its own subtree checkpoint plan (pooled buffers,
    per-block recomputation), the plans run side by side through batched
    calls, against full evaluations one instance at a time."""
    probs = _problems(syn)
    singles = [_create(b200, pr, precision) for pr in probs]
    ref = [pr.evaluate(inst, transposed_pre=False) for pr, inst in zip(probs, singles)]
    plans = [pkg.checkpoint.smallest_plan(pr) for pr in probs]
    pref, req = gpu_flags(precision, auto_transpose=True)
    if asynch:
        pref |= 1 << 3
    members = []
    for pr, pl in zip(probs, plans):
        assert pl.n_buffers < pl.full_buffers()
        inst = b200.create(*pl.create_args(), preferenceFlags=pref, requirementFlags=req)
        pr.load(inst)
        members.append(inst)
    batch = pkg.binding.Batch(b200, members)
    tol = TOL[precision]
    for _ in range(2):
        lnl, grads = pkg.checkpoint.batch_checkpointed_evaluate(batch, plans, fused=fused)
        for i, (l0, g0) in enumerate(ref):
            assert rel(lnl[i], l0) <= tol["lnl"], (i, lnl[i], l0)
            assert grad_err(grads[i], g0) <= tol["grad"], i
    batch.finalize()
    for x in singles + members:
        x.finalize()


@pytest.mark.parametrize("asynch", [False, True], ids=["synch", "asynch"])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_fused_matches_single_instances_and_oracle(b200, pkg, syn, oracle, precision,
                                                         asynch):
    """beagleB200BatchUpdatePrePartialsWithDerivatives: the batched fused walks
    (4-state members with 1/4/8 categories; FP32 20-state members on the
    tensor cores) and the members' own calls (3 categories; FP64 20 states)
    against separate single-instance calls and the oracle."""
    probs = _problems(syn)
    singles = [_create(b200, pr, precision) for pr in probs]
    ref = [pr.evaluate(inst, transposed_pre=False) for pr, inst in zip(probs, singles)]
    members = [_create(b200, pr, precision, asynch) for pr in probs]
    batch = pkg.binding.Batch(b200, members)
    tol = TOL[precision]
    for rep in range(2):
        lnl, grads = syn.batch_evaluate(batch, probs, fused=True)
        for k, (l1, g1) in enumerate(ref):
            assert rel(lnl[k], l1) <= (1e-12 if precision == "double" else tol["lnl"]), k
            assert grad_err(grads[k], g1) <= (1e-10 if precision == "double" else tol["grad"]), \
                (k, grad_err(grads[k], g1))
    for k in (0, 3, len(probs) - 1):
        _, lo, go = run_oracle(oracle, probs[k])
        assert rel(lnl[k], lo) <= tol["lnl"]
        assert grad_err(grads[k], go) <= tol["grad"]
    batch.finalize()
    for x in singles + members:
        x.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_whole_step_graph(b200, pkg, syn, precision):
    """The whole batched step -- transition matrices, post-order walks,
    scaling, root lnL, the fused pre-order walks with derivatives -- captured
    once; each launch takes every member's new branch lengths
    (beagleB200BatchLaunchGraphWithLengths).  Against plain batched
    evaluations with the same lengths; the caller's length arrays are
    overwritten right after each launch call (they are copied on the host)."""
    probs = _problems(syn)
    plain = pkg.binding.Batch(b200, [_create(b200, pr, precision, True) for pr in probs])
    graphed = pkg.binding.Batch(b200, [_create(b200, pr, precision, True) for pr in probs])
    graph, lnl_g, sums_g = syn.batch_capture_step(graphed, probs, fused=True)
    rng = np.random.default_rng(9)
    tol = TOL[precision]
    for step in range(3):
        ts = [p.lengths * (1 + 0.05 * rng.standard_normal(p.B)) for p in probs]
        lnl0, g0 = syn.batch_evaluate(plain, probs, lengths=ts, fused=True)
        flat = np.concatenate(ts)
        graphed.launchGraphWithLengths(graph, flat)
        flat[:] = 1e9                         # the call has its own copy
        graphed.wait()
        g1 = syn.batch_gradients(probs, sums_g, fused=True)
        for i in range(len(probs)):
            assert rel(lnl_g[i], lnl0[i]) <= (1e-12 if precision == "double" else tol["lnl"]), \
                (step, i)
            assert grad_err(g1[i], g0[i]) <= (1e-10 if precision == "double" else tol["grad"]), \
                (step, i)
    with pytest.raises(pkg.binding.BeagleError):
        graphed.launchGraphWithLengths(graph, np.ones(3))     # count must match the capture
    plain.finalize()
    graphed.finalize()


@pytest.mark.slow
def test_batch_configuration_shapes_checkpointed(b200, pkg, syn, oracle):
    """Trees drawn as the batched configuration draws them, at its own
    pattern range (log-uniform 100-50,000): every member with a subtree
    checkpoint plan, the plans side by side through batched calls on the
    mixed path, against the same plans one instance at a time on the FP64
    path, and two members against the oracle.  The mixed path runs each
    block's pre-order walk and derivatives as one batched fused call."""
    probs = syn.batched_problems(count=16, seed=2100, max_patterns=50000)
    plans = [pkg.checkpoint.quick_plan(pr) for pr in probs]
    assert max(p.P for p in probs) > 20000

    def members(precision, asynch):
        pref, req = gpu_flags(precision, auto_transpose=True)
        out = []
        for pr, pl in zip(probs, plans):
            inst = b200.create(*pl.create_args(), preferenceFlags=pref | (asynch << 3),
                               requirementFlags=req)
            pr.load(inst)
            out.append(inst)
        return out

    m32 = members("single", 1)
    batch = pkg.binding.Batch(b200, m32)
    lnl32, g32 = pkg.checkpoint.batch_checkpointed_evaluate(batch, plans, fused=True)
    lnl32 = np.array(lnl32)
    g32 = [np.array(g) for g in g32]
    batch.finalize()
    for x in m32:
        x.finalize()
    m64 = members("double", 0)
    tol = TOL["single"]
    for i, (pl, inst) in enumerate(zip(plans, m64)):
        l64, g64 = pl.evaluate(inst)
        assert rel(lnl32[i], l64) <= tol["lnl"], (i, lnl32[i], l64)
        assert grad_err(g32[i], g64) <= tol["grad"], (i, grad_err(g32[i], g64))
        inst.finalize()
    small = sorted(range(len(probs)), key=lambda i: probs[i].P * probs[i].N)[:2]
    for i in small:
        _, lo, go = run_oracle(oracle, probs[i])
        assert rel(lnl32[i], lo) <= tol["lnl"]
        assert grad_err(g32[i], go) <= tol["grad"]


@pytest.mark.parametrize("unpaired", [False, True], ids=["pairs", "one_member_unpaired"])
def test_batch_tc_fused_pair_walk_and_unpaired_lists(b200, pkg, syn, unpaired):
    """FP32 20-state members in one (S, C) group: the batched sibling-pair
    tensor-core walk when every member's list is made of sibling pairs, the
    batched single-op walk for the whole group when one member's list is
    sorted by depth (siblings not adjacent).  Gradients against separate
    single-instance calls."""
    probs = [syn.make_problem(S=20, N=12 + 3 * k, P=400 + 150 * k, C=4, seed=960 + k,
                              rescale=True) for k in range(3)]
    singles = [_create(b200, pr, "single") for pr in probs]
    ref = [pr.evaluate(inst) for pr, inst in zip(probs, singles)]
    members = [_create(b200, pr, "single") for pr in probs]
    batch = pkg.binding.Batch(b200, members)
    syn.batch_evaluate(batch, probs, fused=True)   # leaves every member's post-order side in place
    plan = batch._plan
    pre, nodes = list(plan["pre"]), list(plan["fnodes"])
    if unpaired:
        pr = probs[1]
        ops = pre[1]
        depth = {pr.pre(pr.root): 0}
        for op in ops:
            depth[op[0]] = depth[op[3]] + 1
        ops = ops[np.lexsort((ops[:, 0] % 7, [depth[o[0]] for o in ops]))]
        pre[1] = ops
        nodes[1] = (ops[:, 0] - pr.pre(0)).astype(np.int32)
    sums, _ = batch.updatePrePartialsWithDerivatives(pre, nodes, plan["dmat"], plan["zeros"])
    batch.wait()
    for k, pr in enumerate(probs):
        g = np.empty(pr.B)
        g[nodes[k]] = sums[k]
        assert grad_err(g, ref[k][1]) <= TOL["single"]["grad"], (k, grad_err(g, ref[k][1]))
    batch.finalize()
    for x in singles + members:
        x.finalize()


@pytest.mark.parametrize("kind", ["all_4state", "mixed"])
@pytest.mark.parametrize("asynch", [False, True], ids=["synch", "asynch"])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_post_root_matches_single_instances(b200, pkg, syn, oracle, precision, asynch,
                                                  kind):
    """beagleB200BatchUpdatePartialsWithRootLogLikelihood: 4-state members with
    1, 2, 4 and 8 categories run the batched fused walk (k_post4root_batch);
    with a 20-state member (or 3 categories) the batch runs the batched calls
    of the three steps.  lnL and every member's cumulative scale buffer
    against separate single-instance calls; two members against the oracle."""
    probs = [syn.make_problem(S=4, N=8 + 9 * k, P=300 + 700 * k, C=(1, 2, 4, 8)[k % 4],
                              seed=980 + k, rescale=True) for k in range(5)]
    if kind == "mixed":
        probs.append(syn.make_problem(S=20, N=9, P=300, C=4, seed=990, rescale=True))
        probs.append(syn.make_problem(S=4, N=11, P=500, C=3, seed=991, rescale=True))
    singles = [_create(b200, pr, precision) for pr in probs]
    ref = []
    for pr, inst in zip(probs, singles):
        inst.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, pr.lengths)
        inst.updatePartials(pr.post_ops(), -1)
        inst.resetScaleFactors(pr.cumulative)
        inst.accumulateScaleFactors(np.arange(pr.N - 1, dtype=np.int32), pr.cumulative)
        ref.append(inst.calculateRootLogLikelihoods([pr.root], [0], [0], [pr.cumulative]))
    members = [_create(b200, pr, precision, asynch) for pr in probs]
    batch = pkg.binding.Batch(b200, members)
    n = len(probs)
    batch.updateTransitionMatrices([0] * n, [np.arange(p.B, dtype=np.int32) for p in probs],
                                   [p.lengths for p in probs])
    tol = 1e-12 if precision == "double" else TOL[precision]["lnl"]
    for rep in range(2):
        lnl = batch.updatePartialsWithRootLogLikelihood(
            [p.post_ops() for p in probs], [p.cumulative for p in probs],
            [p.root for p in probs], [0] * n, [0] * n)
        batch.wait()
        for k in range(n):
            assert rel(lnl[k], ref[k]) <= tol, (rep, k, lnl[k], ref[k])
    for k, (pr, inst, m) in enumerate(zip(probs, singles, members)):
        a, b = m.getScaleFactors(pr.cumulative), inst.getScaleFactors(pr.cumulative)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b))), k
    for k in (0, 3):
        _, lo, _ = run_oracle(oracle, probs[k])
        assert rel(lnl[k], lo) <= TOL[precision]["lnl"], k
    batch.finalize()
    for x in singles + members:
        x.finalize()
