"""Subtree checkpointing of post-order partials for lnL + gradient evaluations
whose partials buffers would not fit in device memory.

A full evaluation (``synthetic.Problem.evaluate``, the call sequence of the
reference's ``examples/hmctest/hmctest.cpp:398-703``) keeps 3N - 3 partials
buffers alive for an N-taxon tree: N - 1 post-order and 2N - 2 pre-order.
Here only the post-order partials of *checkpoint* nodes survive the forward
pass.  The tree is cut at the checkpoints into blocks: a block is a checkpoint
(or the root) plus the internal nodes below it down to the next checkpoints or
tips.  The backward pass visits the blocks depth first and, for each block,

1. recomputes the post-order partials of its inner nodes from the kept
   checkpoints and tips (one ``updatePartials`` call);
2. computes the pre-order partials of every node below the block root (one
   ``updatePrePartials`` call);
3. computes the edge derivatives of every branch in the block (one
   ``calculateEdgeDerivatives`` call);

then frees the block's buffers, except the pre-order partials of the
checkpoints at its lower edge: those are the roots of the blocks below.

Physical buffers come from a pool indexed after the tips and are reused within
one call: BEAGLE executes an operation list in order, so a buffer whose last
reader is op k may be op k + 1's destination.  The schedule is a plain list of
BEAGLE calls, so it runs unchanged on any object with the ``beagle.h`` method
names (``binding.Instance``, the oracle), and an ASYNCH instance can capture
it as one CUDA graph.

Scale buffers (one FP64 value per pattern and node) are not pooled; a
recomputed post-order op rewrites its node's factors with the values the
forward pass wrote.  Recomputation adds at most one post-order pass.
"""

import heapq

import numpy as np

from .synthetic import OP_NONE, postorder


class _Pool:
    """Lowest-free-first allocator of partials buffer ids starting at ``base``;
    records the peak number in use."""

    def __init__(self, base):
        self.base = base
        self.free = []
        self.top = 0
        self.used = 0
        self.peak = 0

    def alloc(self):
        if self.free:
            b = heapq.heappop(self.free)
        else:
            b = self.base + self.top
            self.top += 1
        self.used += 1
        self.peak = max(self.peak, self.used)
        return b

    def release(self, b):
        heapq.heappush(self.free, b)
        self.used -= 1


def choose_checkpoints(problem, block):
    """Bottom-up cut: an internal node becomes a checkpoint when the number of
    not-yet-covered internal nodes in its subtree (itself included) reaches
    ``block``.  Blocks then hold between 1 and 2*block - 1 internal nodes.  The
    root is always a checkpoint."""
    if block < 1:
        raise ValueError("block must be >= 1")
    N = problem.N
    ch = problem.children
    acc = {}
    cps = set()
    for v in postorder(ch, problem.root):
        a = 1
        for c in ch[v]:
            c = int(c)
            if c >= N and c not in cps:
                a += acc[c]
        acc[v] = a
        if a >= block:
            cps.add(v)
    cps.add(problem.root)
    return cps


class CheckpointPlan:
    """The schedule of BEAGLE calls for one checkpointed lnL + gradient
    evaluation of ``problem`` with blocks of about ``block`` internal nodes.

    Buffer ids: tips 0..N-1 as in ``synthetic.Problem``; pool buffers N ..
    N + pool - 1.  Matrix and scale-buffer ids are the Problem's.
    """

    def __init__(self, problem, block, transposed_pre=False):
        self.pb = pb = problem
        self.block = block
        self.transposed_pre = transposed_pre
        N, ch = pb.N, pb.children
        self.checkpoints = cps = choose_checkpoints(pb, block)
        pool = _Pool(N)
        post = {}                       # node -> buffer holding its post-order partials
        for t in range(N):
            post[t] = t

        def rescale_post(v):
            return v - N if pb.rescale else OP_NONE

        def rescale_pre(v):
            return (N - 1) + v if pb.rescale else OP_NONE

        def post_op(v):
            c1, c2 = (int(x) for x in ch[v])
            return [post[v], rescale_post(v), OP_NONE, post[c1], c1, post[c2], c2]

        # Forward: every internal node once; inner nodes freed after their parent.
        fwd = []
        for v in postorder(ch, pb.root):
            post[v] = pool.alloc()
            fwd.append(post_op(v))
            for c in ch[v]:
                c = int(c)
                if c >= N and c not in cps:
                    pool.release(post.pop(c))
        self.forward_ops = np.array(fwd, dtype=np.int32)
        self.root_buffer = post[pb.root]
        steps = []
        # The root's post-order partials serve only the root lnL.
        pool.release(post.pop(pb.root))
        pre = {pb.root: pool.alloc()}
        self.root_pre_buffer = pre[pb.root]

        stack = [pb.root]
        self.n_blocks = 0
        self.blocks = []        # per block: (post ops, pre ops, deriv step)
        while stack:
            r = stack.pop()
            self.n_blocks += 1
            # The block: inner nodes (not checkpoints) and its lower edge.
            inner, edge = [], []
            walk = [int(c) for c in ch[r]]
            while walk:
                v = walk.pop()
                if v < N or v in cps:
                    edge.append(v)
                else:
                    inner.append(v)
                    walk.extend(int(c) for c in ch[v])
            inner_set = set(inner)
            # 1. recompute the inner nodes' post-order partials
            rec = []
            for v in postorder(ch, r):
                if v in inner_set:
                    post[v] = pool.alloc()
                    rec.append(post_op(v))
            # postorder() descends into checkpoints too; keep only this block's
            # nodes, which it emits children first.
            block_post = np.array(rec, dtype=np.int32).reshape(-1, 7)
            if rec:
                steps.append(("post", block_post))
            # 2. pre-order partials of every node below r in the block
            pre_ops, branches = [], []
            order = [r]
            i = 0
            while i < len(order):
                p = order[i]
                i += 1
                if p != r and p not in inner_set:
                    continue
                a, b = (int(x) for x in ch[p])
                for v, sib in ((a, b), (b, a)):
                    pre[v] = pool.alloc()
                    m = pb.B + 1 + v if transposed_pre else v
                    pre_ops.append([pre[v], rescale_pre(v), OP_NONE, pre[p], m, post[sib], sib])
                    branches.append(v)
                    order.append(v)
            steps.append(("pre", np.array(pre_ops, dtype=np.int32)))
            # 3. edge derivatives of the block's branches
            br = np.array(branches, dtype=np.int32)
            steps.append(("deriv", br, np.array([post[v] for v in branches], dtype=np.int32),
                          np.array([pre[v] for v in branches], dtype=np.int32)))
            self.blocks.append((block_post, steps[-2][1], steps[-1]))
            # Free: r's pre-order partials, inner nodes' post and pre, tips' pre,
            # and the edge checkpoints' post (their branch is done).  The edge
            # checkpoints' pre-order partials root the blocks below.
            pool.release(pre.pop(r))
            for v in inner:
                pool.release(post.pop(v))
                pool.release(pre.pop(v))
            for v in edge:
                if v < N:
                    pool.release(pre.pop(v))
                else:
                    pool.release(post.pop(v))
            # depth first, first child's block on top
            stack.extend(v for v in reversed(edge) if v >= N)
        self.steps = steps
        self.pool = pool.peak
        self.calls = 1 + sum(1 for s in steps)

    # ------------------------------------------------------------------ sizes

    @property
    def n_buffers(self):
        """Partials + compact buffers the instance needs (tips + pool)."""
        return self.pb.N + self.pool

    def create_args(self):
        pb = self.pb
        nc = len(pb.compact_tips())
        return (pb.N, self.n_buffers - nc, nc, pb.S, pb.P, 1, pb.n_matrices, pb.C, pb.n_scale)

    def full_buffers(self):
        """Tip + internal buffers of the full (uncheckpointed) schedule that
        the pool replaces: N tips + (N - 1) post + (2N - 2) pre."""
        return self.pb.N + (self.pb.N - 1) + self.pb.B

    # ------------------------------------------------------------- evaluation

    def evaluate(self, inst, lengths=None, fused=False):
        """One lnL + gradient evaluation; returns (lnL, gradient[B]).  The
        instance holds the problem's data (``Problem.load``).  With ``fused``
        each block's pre-order walk and derivatives are one
        beagleB200UpdatePrePartialsWithDerivatives call (its sums come in
        the block's branch order, the pre-order ops' order)."""
        pb = self.pb
        t = pb.lengths if lengths is None else lengths
        inst.updateTransitionMatrices(0, np.arange(pb.B, dtype=np.int32), None, None, t)
        return self._after_matrices(inst, fused)

    def _after_matrices(self, inst, fused=False):
        pb = self.pb
        if self.transposed_pre:
            idx = np.arange(pb.B, dtype=np.int32)
            inst.transposeTransitionMatrices(idx, idx + pb.B + 1)
        inst.updatePartials(self.forward_ops, OP_NONE)
        cum = OP_NONE
        if pb.rescale:
            cum = pb.cumulative
            inst.resetScaleFactors(cum)
            inst.accumulateScaleFactors(np.arange(pb.N - 1, dtype=np.int32), cum)
        lnl = inst.calculateRootLogLikelihoods([self.root_buffer], [0], [0], [cum])
        self._set_root_pre(inst)
        grad = np.zeros(pb.B)
        parts = []
        steps = self.steps
        for i, s in enumerate(steps):
            if s[0] == "post":
                inst.updatePartials(s[1], OP_NONE)
            elif s[0] == "pre":
                if fused:                  # with the "deriv" step that follows it
                    _, br, pst, _ = steps[i + 1]
                    sums, _ = inst.updatePrePartialsWithDerivatives(
                        s[1], pst, np.full(len(br), pb.B, dtype=np.int32), [0])
                    parts.append((br, sums))
                else:
                    inst.updatePrePartials(s[1], OP_NONE)
            elif not fused:
                _, br, pst, prb = s
                _, sums, _ = inst.calculateEdgeDerivatives(
                    pst, prb, np.full(len(br), pb.B, dtype=np.int32), [0], per_site=False,
                    sums=True, sumsq=False)
                parts.append((br, sums))
        self._parts = parts
        return lnl, self._gather(grad)

    def _gather(self, grad):
        for br, sums in self._parts:
            grad[br] = sums
        return grad

    def _set_root_pre(self, inst):
        pb = self.pb
        code = inst.setRootPrePartials([self.root_pre_buffer], [0], check=False)
        if code == -7:                       # BEAGLE_ERROR_NO_IMPLEMENTATION
            inst.setPartials(self.root_pre_buffer, pb.root_pre_partials())
        elif code < 0:
            raise RuntimeError(f"setRootPrePartials returned {code}")

    def capture(self, inst, fused=False):
        """Record the evaluation after the transition matrices as a CUDA graph
        of an ASYNCH instance; returns (graph, gradient getter).  The getter,
        called after ``getLogLikelihood`` following a launch, assembles the
        gradient from the per-block sums the graph delivers."""
        self.evaluate(inst, fused=fused)
        inst.getLogLikelihood()
        inst.beginCapture()
        try:
            self._after_matrices(inst, fused)
        finally:
            graph = inst.endCapture()
        parts = self._parts

        def gradient():
            g = np.zeros(self.pb.B)
            for br, sums in parts:
                g[br] = sums
            return g

        return graph, gradient


def quick_plan(problem, transposed_pre=False):
    """One plan with blocks of about sqrt(N / 2) internal nodes: within a few
    buffers of the smallest plan, built in one pass (for many trees)."""
    return CheckpointPlan(problem, max(2, int(round((problem.N / 2) ** 0.5))), transposed_pre)


def plan_for_budget(problem, max_buffers, transposed_pre=False):
    """The plan with the fewest calls whose tip + pool buffers fit in
    ``max_buffers``; raises ValueError when no block size fits."""
    best = None
    for block in range(1, problem.N):
        plan = CheckpointPlan(problem, block, transposed_pre)
        if plan.n_buffers <= max_buffers and (best is None or plan.calls < best.calls):
            best = plan
    if best is None:
        raise ValueError(f"no checkpoint plan fits in {max_buffers} buffers")
    return best


def smallest_plan(problem, transposed_pre=False):
    """The plan with the fewest buffers (ties: fewer calls)."""
    best = None
    for block in range(1, problem.N):
        plan = CheckpointPlan(problem, block, transposed_pre)
        if best is None or (plan.n_buffers, plan.calls) < (best.n_buffers, best.calls):
            best = plan
    return best


def batch_checkpointed_evaluate(batch, plans, lengths=None, fused=False):
    """One lnL + gradient evaluation of every member of a batch, each with its
    own checkpoint plan (members in plan order; S > 4 members need
    PREORDER_TRANSPOSE_AUTO).  The members' schedules run side by side: one
    batched forward walk, scale accumulation and root lnL, then for block
    i = 0, 1, ... one batched recomputation, pre-order walk and derivative call
    over every member that has an i-th block (the others pass empty lists);
    with ``fused`` the pre-order walk and the derivatives of each block index
    are one beagleB200BatchUpdatePrePartialsWithDerivatives call.
    Returns (lnL[n], [gradient_m])."""
    n = len(plans)
    pbs = [pl.pb for pl in plans]
    resc = [p.rescale for p in pbs]
    if any(resc) and not all(resc):
        raise ValueError("a batch rescales all members or none")
    zeros, none = [0] * n, [OP_NONE] * n
    idx = [np.arange(p.B, dtype=np.int32) for p in pbs]
    ts = [p.lengths if lengths is None else lengths[i] for i, p in enumerate(pbs)]
    batch.updateTransitionMatrices(zeros, idx, ts)
    batch.updatePartials([pl.forward_ops for pl in plans], none)
    cums = none
    if all(resc):
        cums = [p.cumulative for p in pbs]
        batch.accumulateScaleFactors([np.arange(p.N - 1, dtype=np.int32) for p in pbs], cums,
                                     reset=True)
    lnl = batch.calculateRootLogLikelihoods([pl.root_buffer for pl in plans], zeros, zeros, cums)
    batch.setRootPrePartials([pl.root_pre_buffer for pl in plans], zeros)
    grads = [np.zeros(p.B) for p in pbs]
    empty_ops = np.zeros((0, 7), dtype=np.int32)
    empty_idx = np.zeros(0, dtype=np.int32)
    parts = []
    for i in range(max(len(pl.blocks) for pl in plans)):
        blk = [pl.blocks[i] if i < len(pl.blocks) else None for pl in plans]
        batch.updatePartials([b[0] if b else empty_ops for b in blk], none)
        post = [b[2][2] if b else empty_idx for b in blk]
        pre = [b[2][3] if b else empty_idx for b in blk]
        dmat = [np.full(len(q), p.B, dtype=np.int32) for q, p in zip(post, pbs)]
        if fused:
            sums, _ = batch.updatePrePartialsWithDerivatives(
                [b[1] if b else empty_ops for b in blk], post, dmat, zeros)
        else:
            batch.updatePrePartials([b[1] if b else empty_ops for b in blk])
            sums, _ = batch.calculateEdgeDerivatives(post, pre, dmat, zeros)
        parts.append([(b[2][1] if b else empty_idx, sm) for b, sm in zip(blk, sums)])
    batch.wait()
    for step in parts:
        for m, (br, sm) in enumerate(step):
            grads[m][br] = sm
    return lnl, grads
