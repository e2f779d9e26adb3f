"""Seeded synthetic phylogenetic workloads and the BEAGLE call sequence that
evaluates lnL and the branch-length gradient.

There is no public dataset for this path; these generators stand in for one,
with the shapes and distributions the benchmark configurations name.  They play
the role of the reference's ``examples/synthetictest`` (random-join trees,
``synthetictest.cpp:986-1021``) and ``examples/hmctest`` (the pre-order /
edge-derivative call sequence, ``hmctest.cpp:398-703``), with numpy
``PCG64(seed)`` streams instead of the reference's LCG.

Buffer conventions used by :class:`Problem` for a rooted binary tree with N
tips (node ids: tips 0..N-1, internal N..2N-2, root 2N-2, B = 2N-2 branches):

* post-order partials of node v: buffer v;
* pre-order partials of node v: buffer (2N-1) + v;
* transition matrix of the branch above node v: matrix v (v < B); the
  rate-scaled generator Q*r_c used as the derivative matrix: matrix B; the
  transposed P of node v (pre-order operand under the GPU's manual-transpose
  convention for S > 4): matrix B + 1 + v;
* scale buffers: post-order node v -> v - N, pre-order node v -> (N-1) + v,
  cumulative -> 3N - 3.
"""

import numpy as np
from dataclasses import dataclass, field

OP_NONE = -1

# NCBI standard genetic code (table 1), codons ordered TCAG at each position.
_AA = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG"
_NUC = "TCAG"


def random_tree(n_taxa, rng):
    """Random-join rooted binary tree (the topology process of
    synthetictest.cpp:986-1021): each new tip is joined, through a new parent,
    to a uniformly chosen existing node.  Returns (parent, children) with tips
    0..N-1, internal nodes N..2N-2 and the root relabelled 2N-2."""
    N = n_taxa
    parent = {0: -1}
    children = {}
    nodes = [0]
    next_internal = N
    for tip in range(1, N):
        sib = nodes[int(rng.integers(len(nodes)))]
        newp = next_internal
        next_internal += 1
        gp = parent[sib]
        parent[newp] = gp
        if gp >= 0:
            kids = children[gp]
            kids[kids.index(sib)] = newp
        children[newp] = [sib, tip]
        parent[sib] = newp
        parent[tip] = newp
        nodes += [tip, newp]
    root = next(v for v, p in parent.items() if p < 0)
    want = 2 * N - 2
    if root != want:                                  # swap labels root <-> 2N-2
        def rl(v):
            return want if v == root else (root if v == want else v)
        parent = {rl(v): (rl(p) if p >= 0 else -1) for v, p in parent.items()}
        children = {rl(v): [rl(c) for c in kids] for v, kids in children.items()}
    par = np.full(2 * N - 1, -1, dtype=np.int64)
    for v, p in parent.items():
        par[v] = p
    ch = np.zeros((2 * N - 1, 2), dtype=np.int64) - 1
    for v, kids in children.items():
        ch[v] = kids
    return par, ch


def postorder(ch, root):
    out, stack = [], [(root, False)]
    while stack:
        v, done = stack.pop()
        if ch[v, 0] < 0:
            continue
        if done:
            out.append(v)
        else:
            stack.append((v, True))
            stack.append((int(ch[v, 1]), False))
            stack.append((int(ch[v, 0]), False))
    return out


def preorder_nonroot(ch, root):
    out, stack = [], [root]
    while stack:
        v = stack.pop()
        for c in ch[v]:
            if c >= 0:
                out.append(int(c))
                stack.append(int(c))
    return out


def eigen_reversible(Q, pi):
    """Eigensystem of a reversible Q through the symmetric form
    D^1/2 Q D^-1/2; returns (V, V^-1, lambda) with Q = V diag(lambda) V^-1."""
    d = np.sqrt(pi)
    A = d[:, None] * Q / d[None, :]
    A = 0.5 * (A + A.T)
    lam, U = np.linalg.eigh(A)
    V = U / d[:, None]
    Vi = U.T * d[None, :]
    return V, Vi, lam


def _normalise(R, pi):
    Q = R * pi[None, :]
    np.fill_diagonal(Q, 0.0)
    np.fill_diagonal(Q, -Q.sum(axis=1))
    mu = -np.dot(pi, np.diag(Q))
    return Q / mu


def gtr_model(rng):
    """4-state GTR: exchangeabilities ~ U(0.5, 2), frequencies ~ Dirichlet(1,1,1,1)."""
    pi = rng.dirichlet(np.ones(4))
    R = np.zeros((4, 4))
    iu = np.triu_indices(4, 1)
    R[iu] = rng.uniform(0.5, 2.0, size=len(iu[0]))
    R = R + R.T
    return _normalise(R, pi), pi


def amino_model(rng, S=20):
    """S-state model: symmetric exchangeabilities ~ Gamma(1,1), pi ~ Dirichlet(1 x S)."""
    pi = rng.dirichlet(np.ones(S))
    R = np.zeros((S, S))
    iu = np.triu_indices(S, 1)
    R[iu] = rng.gamma(1.0, 1.0, size=len(iu[0]))
    R = R + R.T
    return _normalise(R, pi), pi


def codon_model(rng):
    """Goldman-Yang style 61-state codon model: kappa ~ U(1,4), omega ~ U(0.1,1),
    codon frequencies ~ Dirichlet(1 x 61); single-nucleotide changes only."""
    kappa = rng.uniform(1.0, 4.0)
    omega = rng.uniform(0.1, 1.0)
    codons = [a + b + c for a in _NUC for b in _NUC for c in _NUC]
    sense = [(cd, _AA[i]) for i, cd in enumerate(codons) if _AA[i] != "*"]
    S = len(sense)
    pi = rng.dirichlet(np.ones(S))
    R = np.zeros((S, S))
    purine = set("AG")
    for i, (ci, ai) in enumerate(sense):
        for j, (cj, aj) in enumerate(sense):
            if i == j:
                continue
            diff = [k for k in range(3) if ci[k] != cj[k]]
            if len(diff) != 1:
                continue
            x, y = ci[diff[0]], cj[diff[0]]
            r = 1.0
            if (x in purine) == (y in purine):
                r *= kappa
            if ai != aj:
                r *= omega
            R[i, j] = r
    return _normalise(R, pi), pi


def discrete_gamma(alpha, ncat):
    """Mean-of-category discrete gamma rates (Yang 1994), equal weights."""
    if ncat == 1:
        return np.ones(1), np.ones(1)
    from scipy.special import gammainc
    from scipy.stats import gamma
    cuts = gamma.ppf(np.arange(1, ncat) / ncat, alpha, scale=1.0 / alpha)
    edges = np.concatenate([[0.0], cuts, [np.inf]])
    cdf1 = gammainc(alpha + 1.0, edges * alpha)
    rates = ncat * np.diff(cdf1)
    rates *= ncat / rates.sum()
    return rates, np.full(ncat, 1.0 / ncat)


@dataclass
class Problem:
    """One likelihood+gradient workload (a tree, a model and data) and the
    BEAGLE call sequence over it."""
    N: int
    S: int
    P: int
    C: int
    parent: np.ndarray
    children: np.ndarray
    lengths: np.ndarray            # [B] branch length above node v
    Q: np.ndarray
    pi: np.ndarray
    V: np.ndarray
    Vi: np.ndarray
    lam: np.ndarray
    rates: np.ndarray
    catw: np.ndarray
    patw: np.ndarray
    tip_states: np.ndarray         # [N][P] (S = missing)
    tip_partials: dict = field(default_factory=dict)   # tip -> [P*S] for ambiguous tips
    rescale: bool = False
    seed: int = 0
    name: str = ""

    @property
    def B(self):
        return 2 * self.N - 2

    @property
    def root(self):
        return 2 * self.N - 2

    @property
    def n_buffers(self):
        return 2 * (2 * self.N - 1)

    @property
    def n_matrices(self):
        return 2 * self.B + 1

    @property
    def n_scale(self):
        return 3 * self.N - 2

    @property
    def cumulative(self):
        return 3 * self.N - 3

    def pre(self, v):
        return 2 * self.N - 1 + v

    def compact_tips(self):
        return [t for t in range(self.N) if t not in self.tip_partials]

    def create_args(self):
        """(tipCount, partialsBufferCount, compactBufferCount, S, P, eigen, matrices,
        categories, scale buffers) for beagleCreateInstance."""
        nc = len(self.compact_tips())
        return (self.N, self.n_buffers - nc, nc, self.S, self.P, 1, self.n_matrices,
                self.C, self.n_scale)

    def post_ops(self):
        """Post-order ops (dest, write scale, read scale, child 1, its matrix,
        child 2, its matrix); built once per problem (the topology is fixed)."""
        if getattr(self, "_post_ops", None) is None:
            self._post_ops = self._build_post_ops()
        return self._post_ops.copy()

    def _build_post_ops(self):
        ops = []
        for v in postorder(self.children, self.root):
            c1, c2 = (int(x) for x in self.children[v])
            ws = v - self.N if self.rescale else OP_NONE
            ops.append([v, ws, OP_NONE, c1, c1, c2, c2])
        return np.array(ops, dtype=np.int32)

    def pre_ops(self, transposed_matrices=False):
        """Pre-order ops (dest, write, read, pre(parent), P_node, sibling, P_sib).
        With ``transposed_matrices`` the node's matrix index points at its
        transposed copy (B + 1 + v).  Built once per problem and flag."""
        cache = self.__dict__.setdefault("_pre_ops", {})
        if transposed_matrices not in cache:
            cache[transposed_matrices] = self._build_pre_ops(transposed_matrices)
        return cache[transposed_matrices].copy()

    def _build_pre_ops(self, transposed_matrices):
        ops = []
        for v in preorder_nonroot(self.children, self.root):
            p = int(self.parent[v])
            sib = int(self.children[p, 0] if self.children[p, 1] == v else self.children[p, 1])
            ws = (self.N - 1) + v if self.rescale else OP_NONE
            m = self.B + 1 + v if transposed_matrices else v
            ops.append([self.pre(v), ws, OP_NONE, self.pre(p), m, sib, sib])
        return np.array(ops, dtype=np.int32)

    def scaled_q(self):
        """[C][S][S] derivative matrices Q * r_c (hmctest.cpp:398-407)."""
        return np.stack([self.Q * r for r in self.rates])

    def root_pre_partials(self):
        return np.broadcast_to(self.pi, (self.C, self.P, self.S)).reshape(-1).copy()

    def set_root_pre(self, inst):
        """Pre-order root partials = state frequencies (hmctest.cpp:550-559),
        through beagleSetRootPrePartials where the instance implements it."""
        if getattr(inst, "_no_root_pre", False):
            inst.setPartials(self.pre(self.root), self.root_pre_partials())
            return
        code = inst.setRootPrePartials([self.pre(self.root)], [0], check=False)
        if code == -7:                       # BEAGLE_ERROR_NO_IMPLEMENTATION
            inst._no_root_pre = True
            inst.setPartials(self.pre(self.root), self.root_pre_partials())
        elif code < 0:
            raise RuntimeError(f"setRootPrePartials returned {code}")

    def load(self, inst, transposed_pre=False):
        """Set tips, model and weights on an instance (any object with the
        beagle.h method names of ``binding.Instance``)."""
        for t in range(self.N):
            if t in self.tip_partials:
                inst.setTipPartials(t, self.tip_partials[t])
            else:
                inst.setTipStates(t, self.tip_states[t])
        inst.setEigenDecomposition(0, self.V.reshape(-1), self.Vi.reshape(-1), self.lam)
        inst.setStateFrequencies(0, self.pi)
        inst.setCategoryWeights(0, self.catw)
        inst.setCategoryRates(self.rates)
        inst.setPatternWeights(self.patw)
        inst.setTransitionMatrix(self.B, self.scaled_q().reshape(-1), 0.0)

    def evaluate(self, inst, gradient=True, transposed_pre=False, lengths=None, mark=None,
                 fused=False):
        """One lnL (+ gradient) evaluation: the call sequence the benchmark times.

        updateTransitionMatrices (all B branches) -> updatePartials (N-1 ops) ->
        scale accumulation -> root lnL -> root pre-partials -> updatePrePartials
        (B ops) -> calculateEdgeDerivatives (all B branches, sums only).
        With ``fused`` the post-order walk, scale accumulation and root lnL are
        one beagleB200UpdatePartialsWithRootLogLikelihood call, and the last
        two are one beagleB200UpdatePrePartialsWithDerivatives call, whose
        sums come in pre-order op order (``fused_branches()`` names the branch
        of each; ``branch_gradient`` reorders them).
        Returns (lnL, gradient[B] or None)."""
        mark = mark or (lambda name: None)
        t = self.lengths if lengths is None else lengths
        idx = np.arange(self.B, dtype=np.int32)
        mark("start")
        inst.updateTransitionMatrices(0, idx, None, None, t)
        mark("matrices")
        return self._after_matrices(inst, gradient, transposed_pre, mark, fused)

    def fused_branches(self):
        """Branch (node) of each pre-order op: the order of the fused call's sums."""
        return self.pre_ops()[:, 0] - self.pre(0)

    def branch_gradient(self, sums):
        """Fused-call sums (op order) as gradient[B] in branch order."""
        g = np.empty(self.B)
        g[self.fused_branches()] = sums
        return g

    def _after_matrices(self, inst, gradient, transposed_pre, mark, fused=False):
        idx = np.arange(self.B, dtype=np.int32)
        cum = self.cumulative if self.rescale else OP_NONE
        if fused:
            # post-order walk, cumulative scale factors and root lnL in one call
            lnl = inst.updatePartialsWithRootLogLikelihood(self.post_ops(), cum, self.root, 0, 0)
            mark("post")
            mark("scale")
            mark("root")
        else:
            inst.updatePartials(self.post_ops(), OP_NONE)
            mark("post")
            if self.rescale:
                inst.resetScaleFactors(cum)
                inst.accumulateScaleFactors(np.arange(self.N - 1, dtype=np.int32), cum)
            mark("scale")
            lnl = inst.calculateRootLogLikelihoods([self.root], [0], [0], [cum])
            mark("root")
        if not gradient:
            return lnl, None
        if transposed_pre:
            inst.transposeTransitionMatrices(idx, idx + self.B + 1)
        self.set_root_pre(inst)
        mark("rootpre")
        if fused:
            nodes = self.fused_branches()
            sums, _ = inst.updatePrePartialsWithDerivatives(
                self.pre_ops(transposed_pre), nodes, np.full(self.B, self.B, dtype=np.int32), [0])
            mark("deriv")
            return lnl, sums
        inst.updatePrePartials(self.pre_ops(transposed_pre), OP_NONE)
        mark("pre")
        nonroot = np.arange(self.B, dtype=np.int32)
        _, sums, _ = inst.calculateEdgeDerivatives(
            nonroot, nonroot + self.pre(0), np.full(self.B, self.B, dtype=np.int32),
            [0], per_site=False, sums=True, sumsq=False)
        mark("deriv")
        return lnl, sums

    def capture(self, inst, transposed_pre=False, fused=False):
        """Record one evaluation after the transition matrices (partials,
        scaling, root lnL, pre-order partials, edge derivatives) as a CUDA
        graph of an ASYNCH instance; returns (graph, gradient array the graph
        fills: branch order, or op order with ``fused``).  Runs the sequence
        once first, as the capture requires."""
        self.evaluate(inst, transposed_pre=transposed_pre, fused=fused)
        inst.getLogLikelihood()
        inst.beginCapture()
        try:
            _, grad = self._after_matrices(inst, True, transposed_pre, lambda name: None, fused)
        finally:
            graph = inst.endCapture()
        return graph, grad

    def capture_step(self, inst, transposed_pre=False, fused=False):
        """Record one whole evaluation, the transition matrices included, as a
        CUDA graph of an ASYNCH instance; the graph reads the branch lengths
        on the device, and ``evaluate_graph_step`` replaces them per launch.
        Returns (graph, gradient array the graph fills)."""
        self.evaluate(inst, transposed_pre=transposed_pre, fused=fused)
        inst.getLogLikelihood()
        inst.beginCapture()
        try:
            _, grad = self.evaluate(inst, transposed_pre=transposed_pre, fused=fused)
        finally:
            graph = inst.endCapture()
        return graph, grad

    def evaluate_graph_step(self, inst, graph, grad, lengths=None):
        """One evaluation through a graph from ``capture_step``: the new branch
        lengths and the graph in one call, then lnL and the gradient."""
        t = self.lengths if lengths is None else lengths
        inst.launchGraphWithLengths(graph, t)
        lnl = inst.getLogLikelihood()            # waits; delivers the gradient too
        return lnl, grad

    def evaluate_graph(self, inst, graph, grad, lengths=None):
        """One evaluation through a captured graph: new transition matrices
        (outside the graph), the graph, then lnL and the gradient."""
        t = self.lengths if lengths is None else lengths
        inst.updateTransitionMatrices(0, np.arange(self.B, dtype=np.int32), None, None, t)
        inst.launchGraph(graph)
        lnl = inst.getLogLikelihood()            # waits; delivers the gradient too
        return lnl, grad

    def algorithmic_bytes(self, w):
        """Compulsory traffic per phase of one evaluation, with w bytes per real:
        each operation reads each input once and writes each output once
        (synthetictest.cpp:2567-2580 generalised to the pre-order and derivative
        passes).  Partials buffer L = P*C*S*w (S unpadded), compact tip = 4P,
        scale factors 8P per rescaled node (FP64 on this resource)."""
        L = self.P * self.C * self.S * w
        tip = 4 * self.P
        compact = set(self.compact_tips())

        def rd(v):
            return tip if v in compact else L

        sc = 8 * self.P if self.rescale else 0
        post = sum(rd(op[3]) + rd(op[5]) + L + sc for op in self.post_ops())
        pre = sum(L + rd(op[5]) + L + sc for op in self.pre_ops())
        deriv = sum(L + rd(v) for v in range(self.B))
        mats = self.B * self.C * self.S * self.S * w
        # fused pre-order + derivative walk: a sibling pair reads its parent
        # row and both children's post-order rows once, writes two rows
        ops = self.pre_ops()
        fused, k = 0, 0
        while k < len(ops):
            a = ops[k]
            if k + 1 < len(ops) and ops[k + 1][3] == a[3]:
                b = ops[k + 1]
                fused += L + rd(a[5]) + rd(b[5]) + 2 * L + 2 * sc
                k += 2
            else:
                fused += L + rd(a[5]) + rd(a[0] - self.pre(0)) + L + sc
                k += 1
        # scale accumulation: reset (write), N - 1 buffers and the cumulative
        # buffer read, the cumulative buffer written; root lnL: the root row,
        # cumulative and pattern weights read, site values written
        scale = (self.N + 2) * 8 * self.P if self.rescale else 0
        root = L + (8 * self.P if self.rescale else 0) + 16 * self.P
        return dict(matrices=mats, post=post, pre=pre, deriv=deriv, fused=fused, scale=scale,
                    root=root)


GRAD_FLOOR = 0.1     # absolute floor of the per-branch error, in units of rms(gradient)


def gradient_errors(g, gref):
    """Errors of a branch gradient against a reference gradient.

    ``branch``: the worst per-branch relative error,
    max_b |g_b - gref_b| / (|gref_b| + 0.1 rms(gref)).  Branch b's own
    magnitude sets its bar; the floor of a tenth of the gradient's rms only
    keeps a branch whose reference derivative sits near zero (a sum over
    patterns that cancels) from dividing by nothing.
    ``branch_unfloored``: max_b |g_b - gref_b| / |gref_b| over branches with
    gref_b != 0.  ``max_norm``: max_b |g_b - gref_b| / max_b |gref_b|."""
    g = np.asarray(g, dtype=np.float64)
    r = np.asarray(gref, dtype=np.float64)
    d = np.abs(g - r)
    rms = float(np.sqrt(np.mean(r * r))) if r.size else 0.0
    floor = max(GRAD_FLOOR * rms, 1e-300)
    nz = r != 0
    return {"branch": float(np.max(d / (np.abs(r) + floor))) if r.size else 0.0,
            "branch_unfloored": float(np.max(d[nz] / np.abs(r[nz]))) if nz.any() else 0.0,
            "max_norm": float(np.max(d) / max(float(np.max(np.abs(r))), 1e-300))
            if r.size else 0.0}


def make_problem(S, N, P, C, seed, mean_length=0.1, ambiguous=0.0, rescale=False,
                 alpha=0.5, weights=(1, 5), name=""):
    """Build a Problem: random-join tree, Exp(mean_length) branch lengths, a
    GTR (S=4), random-exchangeability (S=20 or other) or GY codon (S=61) model,
    discrete-gamma rates, uniform tip states (``ambiguous`` fraction of tip
    cells given as all-ones partials), pattern weights ~ U{lo..hi}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    par, ch = random_tree(N, rng)
    B = 2 * N - 2
    lengths = rng.exponential(mean_length, size=B)
    if S == 4:
        Q, pi = gtr_model(rng)
    elif S == 61:
        Q, pi = codon_model(rng)
    else:
        Q, pi = amino_model(rng, S)
    V, Vi, lam = eigen_reversible(Q, pi)
    rates, catw = discrete_gamma(alpha, C)
    patw = rng.integers(weights[0], weights[1] + 1, size=P).astype(np.float64)
    states = rng.integers(0, S, size=(N, P))
    tip_partials = {}
    if ambiguous > 0:
        amb = rng.random((N, P)) < ambiguous
        for t in range(N):
            part = np.zeros((P, S))
            part[np.arange(P), states[t]] = 1.0
            part[amb[t]] = 1.0
            tip_partials[t] = part.reshape(-1)
    return Problem(N=N, S=S, P=P, C=C, parent=par, children=ch, lengths=lengths, Q=Q,
                   pi=pi, V=V, Vi=Vi, lam=lam, rates=rates, catw=catw, patw=patw,
                   tip_states=states, tip_partials=tip_partials, rescale=rescale,
                   seed=seed, name=name)


# The benchmark configurations (sizes and distributions of each workload).
CONFIGS = {
    "gtr4_n16_p1000": dict(S=4, N=16, P=1000, C=4, seed=1000, mean_length=0.1,
                           ambiguous=0.05, rescale=False),
    "gtr4_n128_p100k": dict(S=4, N=128, P=100000, C=4, seed=1001, mean_length=0.05,
                            rescale=True),
    "aa20_n64_p20k": dict(S=20, N=64, P=20000, C=4, seed=1002, mean_length=0.1,
                          rescale=True),
    "codon61_n32_p10k": dict(S=61, N=32, P=10000, C=4, seed=1003, mean_length=0.1,
                             rescale=True),
}


def config_problem(name, **over):
    kw = dict(CONFIGS[name])
    kw.update(over)
    return make_problem(name=name, **kw)


def batched_problems(count=256, seed=2000, max_patterns=50000):
    """Heterogeneous batch: per partition N ~ U{16..256}, S in {4 (70%), 20 (30%)},
    C in {1,4,8}, P log-uniform in [100, max_patterns]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        S = 4 if rng.random() < 0.7 else 20
        N = int(rng.integers(16, 257))
        C = int(rng.choice([1, 4, 8]))
        P = int(np.exp(rng.uniform(np.log(100), np.log(max_patterns))))
        out.append(make_problem(S=S, N=N, P=P, C=C, seed=seed + 1 + i,
                                mean_length=0.1, rescale=True, name=f"part{i}"))
    return out


def _batch_plan(batch, problems):
    plan = getattr(batch, "_plan", None)
    if plan is None or plan["problems"] is not problems:
        n = len(problems)
        resc = [p.rescale for p in problems]
        if any(resc) and not all(resc):
            raise ValueError("a batch rescales all members or none")
        nonroot = [np.arange(p.B, dtype=np.int32) for p in problems]
        plan = batch._plan = dict(
            problems=problems, n=n, rescale=all(resc),
            idx=nonroot, post=[p.post_ops() for p in problems],
            pre=[p.pre_ops(False) for p in problems],
            cums=[p.cumulative if p.rescale else OP_NONE for p in problems],
            scales=[np.arange(p.N - 1, dtype=np.int32) for p in problems],
            roots=[p.root for p in problems], roots_pre=[p.pre(p.root) for p in problems],
            pre_idx=[nr + p.pre(0) for nr, p in zip(nonroot, problems)],
            fnodes=[p.fused_branches().astype(np.int32) for p in problems],
            dmat=[np.full(p.B, p.B, dtype=np.int32) for p in problems], zeros=[0] * n,
            none=[OP_NONE] * n)
    return plan


def batch_gradients(problems, sums, fused):
    """Per-member gradients in branch order from a batched evaluation's sums
    (op order with ``fused``)."""
    if not fused:
        return [np.asarray(g) for g in sums]
    return [p.branch_gradient(g) for p, g in zip(problems, sums)]


def batch_evaluate(batch, problems, lengths=None, fused=False):
    """One lnL + gradient evaluation of every problem of a batch (members in
    the same order), the call sequence of Problem.evaluate with one batched
    call per step; with ``fused`` the post-order walk, scaling and root lnL
    are one beagleB200BatchUpdatePartialsWithRootLogLikelihood call and the
    pre-order walk and the derivatives one
    beagleB200BatchUpdatePrePartialsWithDerivatives call.  S > 4 members
    need PREORDER_TRANSPOSE_AUTO (their pre-order ops carry untransposed
    matrices).  Returns (lnL[n], [gradient_m] in branch order)."""
    plan = _batch_plan(batch, problems)
    ts = [p.lengths if lengths is None else lengths[i] for i, p in enumerate(problems)]
    batch.updateTransitionMatrices(plan["zeros"], plan["idx"], ts)
    lnl, sums = _batch_after_matrices(batch, plan, fused)
    batch.wait()
    return lnl, batch_gradients(problems, sums, fused)


def _batch_after_matrices(batch, plan, fused=False):
    if fused:
        # the post-order walk, scaling and root lnL as one batched call
        lnl = batch.updatePartialsWithRootLogLikelihood(plan["post"], plan["cums"],
                                                        plan["roots"], plan["zeros"],
                                                        plan["zeros"])
    else:
        batch.updatePartials(plan["post"], plan["none"])
        if plan["rescale"]:
            batch.accumulateScaleFactors(plan["scales"], plan["cums"], reset=True)
        lnl = batch.calculateRootLogLikelihoods(plan["roots"], plan["zeros"], plan["zeros"],
                                                plan["cums"])
    batch.setRootPrePartials(plan["roots_pre"], plan["zeros"])
    if fused:
        sums, _ = batch.updatePrePartialsWithDerivatives(plan["pre"], plan["fnodes"],
                                                         plan["dmat"], plan["zeros"])
        return lnl, sums
    batch.updatePrePartials(plan["pre"])
    sums, _ = batch.calculateEdgeDerivatives(plan["idx"], plan["pre_idx"], plan["dmat"],
                                             plan["zeros"])
    return lnl, sums


def batch_capture(batch, problems, fused=False):
    """Record one batched evaluation after the transition matrices as a CUDA
    graph of the batch (every member ASYNCH); returns (graph, lnL array,
    gradient arrays: branch order, or op order with ``fused``) that each
    launch fills at the next wait.  Runs the sequence once first, as the
    capture requires."""
    batch_evaluate(batch, problems, fused=fused)
    plan = batch._plan
    batch.beginCapture()
    try:
        lnl, sums = _batch_after_matrices(batch, plan, fused)
    finally:
        graph = batch.endCapture()
    return graph, lnl, sums


def batch_capture_step(batch, problems, fused=False):
    """Record one whole batched evaluation, the transition matrices
    included, as a CUDA graph of the batch; the graph reads the branch
    lengths on the device and ``batch_evaluate_graph_step`` replaces them per
    launch.  Returns (graph, lnL array, gradient arrays) as batch_capture."""
    batch_evaluate(batch, problems, fused=fused)
    plan = batch._plan
    batch.beginCapture()
    try:
        batch.updateTransitionMatrices(plan["zeros"], plan["idx"],
                                       [p.lengths for p in problems])
        lnl, sums = _batch_after_matrices(batch, plan, fused)
    finally:
        graph = batch.endCapture()
    return graph, lnl, sums


def batch_evaluate_graph_step(batch, problems, graph, lengths=None):
    """One batched evaluation through a graph from ``batch_capture_step``: all
    members' new branch lengths (concatenated in member order) and the graph
    in one call, then the wait that delivers lnL and the gradients into the
    captured arrays."""
    ts = [p.lengths if lengths is None else lengths[i] for i, p in enumerate(problems)]
    batch.launchGraphWithLengths(graph, np.concatenate(ts))
    batch.wait()


def batch_evaluate_graph(batch, problems, graph, lengths=None):
    """One batched evaluation through a captured graph: new transition
    matrices (outside the graph), the graph, then the wait that delivers lnL
    and the gradients into the captured arrays."""
    plan = batch._plan
    ts = [p.lengths if lengths is None else lengths[i] for i, p in enumerate(problems)]
    batch.updateTransitionMatrices(plan["zeros"], plan["idx"], ts)
    batch.launchGraph(graph)
    batch.wait()
