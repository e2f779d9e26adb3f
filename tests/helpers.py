"""Shared helpers of the parity tests: running one Problem through an
instance (this library, the compiled reference, or the numpy oracle) and the
tolerances the comparisons use."""
import numpy as np

# Flag bits of beagle.h.
SINGLE, DOUBLE = 1 << 0, 1 << 1
SCALERS_RAW, SCALERS_LOG = 1 << 9, 1 << 10
PROCESSOR_CPU, PROCESSOR_GPU = 1 << 15, 1 << 16
FRAMEWORK_CUDA = 1 << 22
PRE_MANUAL, PRE_AUTO = 1 << 30, 1 << 31

# Tolerances: relative lnL error, and the worst per-branch relative error of
# the branch gradient, max_b |g_b - g_ref,b| / (|g_ref,b| + 0.1 rms(g_ref))
# (synthetic.gradient_errors: each branch against its own magnitude, with a
# floor of a tenth of the gradient's rms for branches whose derivative sums
# to nearly zero).  FP64 plain path 1e-10 (lnL) and 1e-8 (gradient); mixed
# FP32 path 1e-6 (lnL) and 1e-4 (gradient).
TOL = {
    "double": dict(lnl=1e-10, grad=1e-8),
    "single": dict(lnl=1e-6, grad=1e-4),
}


def gpu_flags(precision, log_scalers=True, auto_transpose=False):
    pref = (DOUBLE if precision == "double" else SINGLE) | PROCESSOR_GPU
    pref |= SCALERS_LOG if log_scalers else SCALERS_RAW
    pref |= PRE_AUTO if auto_transpose else PRE_MANUAL
    req = (DOUBLE if precision == "double" else SINGLE) | FRAMEWORK_CUDA
    return pref, req


def run_b200(lib, problem, precision, gradient=True, log_scalers=True, auto_transpose=False):
    pref, req = gpu_flags(precision, log_scalers, auto_transpose)
    inst = lib.create(*problem.create_args(), preferenceFlags=pref, requirementFlags=req)
    problem.load(inst)
    transposed = problem.S > 4 and not auto_transpose
    lnl, grad = problem.evaluate(inst, gradient=gradient, transposed_pre=transposed)
    return inst, lnl, grad


def run_oracle(oracle, problem, gradient=True, log_scalers=True):
    flags = SCALERS_LOG if log_scalers else SCALERS_RAW
    inst = oracle.OracleInstance(*problem.create_args(), flags=flags)
    problem.load(inst)
    lnl, grad = problem.evaluate(inst, gradient=gradient)
    return inst, lnl, grad


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def grad_err(g, gref):
    """Worst per-branch relative error (floored), as the tolerances define it."""
    from importlib import import_module
    return import_module("beagle-lib_b200").synthetic.gradient_errors(g, gref)["branch"]


def partitioned_args(problem, nparts):
    """create_args with room for per-partition matrices, scale buffers and
    cumulative buffers."""
    args = list(problem.create_args())
    args[6] = max(args[6], nparts * problem.B + 1 + 2 * nparts)
    args[8] = max(args[8], nparts * (problem.N - 1) + nparts)
    return args


def run_partitioned(inst, problem, nparts, rescale=True, pre=True):
    """Contiguous pattern partitions, each with its own branch-length scaling
    (matrices q * B + v), scale buffers (q * (N - 1) + v - N) and cumulative
    buffer (nparts * (N - 1) + q): post-order partition ops in one call, the
    per-partition root lnL, then (unscaled) pre-order partition ops in one call.
    Returns (byPartition, total).  S > 4 GPU instances need
    PREORDER_TRANSPOSE_AUTO (the pre-order ops carry untransposed matrices)."""
    from importlib import import_module
    syn = import_module("beagle-lib_b200").synthetic
    pr = problem
    bounds = np.linspace(0, pr.P, nparts + 1).astype(int)
    parts = np.repeat(np.arange(nparts), np.diff(bounds)).astype(np.int32)
    inst.setPatternPartitions(nparts, parts)
    idx = np.arange(pr.B, dtype=np.int32)
    for q in range(nparts):
        inst.updateTransitionMatrices(0, q * pr.B + idx, None, None, pr.lengths * (1 + 0.3 * q))
    cum0 = nparts * (pr.N - 1)
    for q in range(nparts):
        inst.resetScaleFactorsByPartition(cum0 + q, q)
    ops = []
    for v in syn.postorder(pr.children, pr.root):
        c1, c2 = (int(x) for x in pr.children[v])
        for q in range(nparts):
            ws = q * (pr.N - 1) + (v - pr.N) if rescale else -1
            ops.append([v, ws, -1, c1, q * pr.B + c1, c2, q * pr.B + c2, q, cum0 + q])
    inst.updatePartialsByPartition(np.array(ops, dtype=np.int32))
    byp, tot = inst.calculateRootLogLikelihoodsByPartition(
        [pr.root] * nparts, [0] * nparts, [0] * nparts, [cum0 + q for q in range(nparts)],
        list(range(nparts)))
    if pre:
        pr.set_root_pre(inst)
        pops = []
        for v in syn.preorder_nonroot(pr.children, pr.root):
            par = int(pr.parent[v])
            sib = int(pr.children[par, 0] if pr.children[par, 1] == v else pr.children[par, 1])
            for q in range(nparts):
                pops.append([pr.pre(v), -1, -1, pr.pre(par), q * pr.B + v, sib, q * pr.B + sib,
                             q, -1])
        inst.updatePrePartialsByPartition(np.array(pops, dtype=np.int32))
    return np.asarray(byp), tot


def edge_by_partition(inst, problem, nparts, v, derivs, parent=None):
    """calculateEdgeLogLikelihoodsByPartition after run_partitioned: for each
    partition q the edge between node v's parent's pre-order partials (or the
    buffer `parent`) and v (post-order partials or a tip), with partition q's
    matrix of branch v; with
    `derivs`, its first and second derivative matrices are formed first in the
    spare matrices nparts * B + 1 + (0 .. 2 nparts).  Returns the call's tuple
    and the site log-likelihoods."""
    pr = problem
    d1 = d2 = None
    if derivs:
        base = nparts * pr.B + 1
        d1 = [base + q for q in range(nparts)]
        d2 = [base + nparts + q for q in range(nparts)]
        for q in range(nparts):
            inst.updateTransitionMatrices(0, [q * pr.B + v], [d1[q]], [d2[q]],
                                          [pr.lengths[v] * (1 + 0.3 * q)])
    par = pr.pre(int(pr.parent[v])) if parent is None else parent
    cum0 = nparts * (pr.N - 1)
    res = inst.calculateEdgeLogLikelihoodsByPartition(
        [par] * nparts, [v] * nparts, [q * pr.B + v for q in range(nparts)], d1, d2,
        [0] * nparts, [0] * nparts, [cum0 + q for q in range(nparts)], list(range(nparts)))
    return res, inst.getSiteLogLikelihoods()


def model_variant_args(problem):
    """create_args with 3 eigen systems (and rate sets) and 4 spare matrices
    after the problem's own (derivatives of branches 0 and 1)."""
    args = list(problem.create_args())
    args[5] = 3
    args[6] = max(args[6], problem.B + 5)
    return args


def run_model_variants(inst, problem, kind):
    """The problem's tree (no rescaling) evaluated with matrices from
    updateTransitionMatricesWithMultipleModels (kind "multiple": branch u from
    eigen system u % 3 and rate set (u // 3) % 2) or
    updateTransitionMatricesWithModelCategories ("categories": category c
    from eigen system c % 3, no category rate), plus the first and second
    derivative matrices of branches 0 and 1 (matrices B+1 .. B+4).  Eigen
    systems 1, 2 and rate set 1 come from a fixed seed.  Returns (lnL, the
    matrices 0, 1, 2, 3, B+1 .. B+4)."""
    from importlib import import_module
    syn = import_module("beagle-lib_b200").synthetic
    pr = problem
    rng = np.random.Generator(np.random.PCG64(4242))
    for e in (1, 2):
        Q, pi = syn.gtr_model(rng) if pr.S == 4 else syn.amino_model(rng, pr.S)
        V, Vi, lam = syn.eigen_reversible(Q, pi)
        inst.setEigenDecomposition(e, V.reshape(-1), Vi.reshape(-1), lam)
    inst.setCategoryRatesWithIndex(1, np.linspace(0.3, 2.0, pr.C))
    B = pr.B
    probs = np.arange(B, dtype=np.int32)
    d1, d2 = [B + 1, B + 2], [B + 3, B + 4]
    if kind == "multiple":
        eig = [u % 3 for u in range(B)]
        rix = [(u // 3) % 2 for u in range(B)]
        inst.updateTransitionMatricesWithMultipleModels(eig, rix, probs, None, None, pr.lengths)
        inst.updateTransitionMatricesWithMultipleModels(eig[:2], rix[:2], [0, 1], d1, d2,
                                                        pr.lengths[:2])
    else:
        eig = [c % 3 for c in range(pr.C)]
        inst.updateTransitionMatricesWithModelCategories(eig, probs, None, None, pr.lengths)
        inst.updateTransitionMatricesWithModelCategories(eig, [0, 1], d1, d2, pr.lengths[:2])
    inst.updatePartials(pr.post_ops())
    lnl = inst.calculateRootLogLikelihoods([pr.root], [0], [0], [-1])
    mats = [inst.getTransitionMatrix(m) for m in (0, 1, 2, 3, B + 1, B + 2, B + 3, B + 4)]
    return lnl, mats
