"""Parity of the B200 resource against the oracle, through the C ABI.

Every test runs the same seeded inputs through libbeagle_b200.so (on the GPU)
and through the float64 numpy oracle (``oracle/oracle.py``, itself pinned to
the compiled reference by test_oracle.py), and compares with the tolerance
written in tests/helpers.py: FP64 path relative lnL <= 1e-10, mixed FP32 path
relative lnL <= 1e-6 and gradient error <= 1e-4.
"""
import numpy as np
import pytest

from helpers import SCALERS_LOG, SCALERS_RAW, TOL, grad_err, rel, run_b200, run_oracle, gpu_flags

pytestmark = pytest.mark.gpu

SMALL = [
    ("gtr4_n16_p1000", {}),
    ("gtr4_n128_p100k", dict(N=32, P=3000)),
    ("aa20_n64_p20k", dict(N=16, P=1000)),
    ("codon61_n32_p10k", dict(N=8, P=600)),
]


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("name,over", SMALL, ids=[c[0] for c in SMALL])
def test_lnl_and_gradient_small(b200, syn, oracle, name, over, precision):
    pr = syn.config_problem(name, **over)
    inst, lnl, g = run_b200(b200, pr, precision)
    oi, lnl_o, g_o = run_oracle(oracle, pr)
    tol = TOL[precision]
    assert rel(lnl, lnl_o) <= tol["lnl"], (lnl, lnl_o)
    assert grad_err(g, g_o) <= tol["grad"], grad_err(g, g_o)
    site = inst.getSiteLogLikelihoods()
    site_o = oi.getSiteLogLikelihoods()
    assert np.max(np.abs(site - site_o) / np.abs(site_o)) <= 100 * tol["lnl"]
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_auto_transpose_matches_manual(b200, syn, oracle, precision):
    pr = syn.config_problem("aa20_n64_p20k", N=12, P=700)
    _, l1, g1 = run_b200(b200, pr, precision, auto_transpose=True)
    _, l2, g2 = run_b200(b200, pr, precision, auto_transpose=False)
    _, lo, go = run_oracle(oracle, pr)
    tol = TOL[precision]
    assert rel(l1, lo) <= tol["lnl"] and rel(l2, lo) <= tol["lnl"]
    assert grad_err(g1, go) <= tol["grad"] and grad_err(g2, go) <= tol["grad"]


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S", [4, 5, 20, 61])
def test_partials_matrices_and_scalers(b200, syn, oracle, precision, S):
    """Intermediate buffers: P(t), post-order partials, scale factors,
    pre-order partials and per-site derivatives against the oracle."""
    pr = syn.make_problem(S=S, N=10, P=333, C=3, seed=77 + S, rescale=True)
    inst, _, _ = run_b200(b200, pr, precision)
    oi, _, _ = run_oracle(oracle, pr)
    tight = precision == "double"
    # FP64 intermediate buffers: eigen-sum rounding of P(t) (sums of S terms of
    # both signs) differs between summation orders; 1e-9 of the buffer maximum
    # covers the 61-state codon model's conditioning.
    # transition matrices
    for m in [0, 3, pr.B]:
        a, b = inst.getTransitionMatrix(m), oi.getTransitionMatrix(m)
        assert np.max(np.abs(a - b)) <= (1e-13 if tight else 1e-6)
    # post-order root partials and scale buffers
    a, b = inst.getPartials(pr.root), oi.getPartials(pr.root)
    assert np.max(np.abs(a - b)) <= (1e-9 if tight else 1e-5) * np.max(np.abs(b))
    for s in range(pr.N - 1):
        a, b = inst.getScaleFactors(s), oi.getScaleFactors(s)
        assert np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))) <= (1e-9 if tight else 1e-5)
    # pre-order partials of a few nodes (both sides rescale per pattern)
    for v in [0, pr.N, pr.B - 1]:
        a, b = inst.getPartials(pr.pre(v)), oi.getPartials(pr.pre(v))
        assert np.max(np.abs(a - b)) <= (1e-9 if tight else 1e-4) * np.max(np.abs(b))
    # per-site derivatives and sums of squares
    nonroot = np.arange(pr.B, dtype=np.int32)
    dm = np.full(pr.B, pr.B, dtype=np.int32)
    d, s1, s2 = inst.calculateEdgeDerivatives(nonroot, nonroot + pr.pre(0), dm, [0])
    do, s1o, s2o = oi.calculateEdgeDerivatives(nonroot, nonroot + pr.pre(0), dm, [0])
    scale = np.max(np.abs(do))
    assert np.max(np.abs(d - do)) <= (1e-8 if tight else 1e-4) * scale
    assert grad_err(s1, s1o) <= (1e-8 if tight else 1e-4)
    assert grad_err(s2, s2o) <= (1e-8 if tight else 1e-4)
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_raw_scalers_and_cumulative_in_update(b200, syn, oracle, precision):
    """RAW scalers, with the cumulative buffer filled by updatePartials itself."""
    pr = syn.make_problem(S=4, N=24, P=513, C=4, seed=5, rescale=True)
    pref, req = gpu_flags(precision, log_scalers=False)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*pr.create_args(), flags=0)
    out = []
    for x in (inst, oi):
        pr.load(x)
        x.updateTransitionMatrices(0, np.arange(pr.B), None, None, pr.lengths)
        x.resetScaleFactors(pr.cumulative)
        x.updatePartials(pr.post_ops(), pr.cumulative)
        out.append(x.calculateRootLogLikelihoods([pr.root], [0], [0], [pr.cumulative]))
        out.append(x.getScaleFactors(3))
    assert rel(out[0], out[2]) <= TOL[precision]["lnl"]
    assert np.max(np.abs(out[1] - out[3]) / out[3]) <= (1e-12 if precision == "double" else 1e-6)


@pytest.mark.parametrize("precision", ["double", "single"])
def test_edge_loglikelihood_and_derivatives(b200, syn, oracle, precision):
    pr = syn.make_problem(S=4, N=12, P=400, C=4, seed=9)
    pref, req = gpu_flags(precision)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*pr.create_args(), flags=1 << 10)
    res = []
    # edge between node v's pre-order partials and its post-order partials
    v = pr.N + 1
    w = pr.B + 1 + (v + 1) % pr.B          # a spare matrix for d2P/dt2 of branch v
    for x in (inst, oi):
        pr.load(x)
        idx = np.arange(pr.B)
        x.updateTransitionMatrices(0, idx, idx + pr.B + 1, None, pr.lengths)
        # matrix indices B+1.. hold dP/dt here; branch v's d2P/dt2 goes to w
        x.updateTransitionMatrices(0, [v], [v + pr.B + 1], [w], [pr.lengths[v]])
        x.updatePartials(pr.post_ops())
        x.calculateRootLogLikelihoods([pr.root], [0], [0], [-1])
        pr.set_root_pre(x)
        x.updatePrePartials(pr.pre_ops(False))
        res.append(x.calculateEdgeLogLikelihoods(pr.pre(int(pr.parent[v])), v, v,
                                                 v + pr.B + 1, None, 0, 0, -1))
        res.append(x.calculateEdgeLogLikelihoods(pr.pre(int(pr.parent[v])), v, v,
                                                 v + pr.B + 1, w, 0, 0, -1))
    (_, l0, d0, _), (_, l0b, d0b, e0), (_, l1, d1, _), (_, l1b, d1b, e1) = res
    tol = TOL[precision]
    assert rel(l0, l1) <= tol["lnl"] and rel(l0b, l1b) <= tol["lnl"]
    assert abs(d0 - d1) <= tol["grad"] * max(1.0, abs(d1))
    assert abs(d0b - d1b) <= tol["grad"] * max(1.0, abs(d1b))
    # the second derivative (edge lnL with d1 and d2 in one call)
    assert abs(e0 - e1) <= tol["grad"] * max(1.0, abs(e1)), (e0, e1)


def test_missing_states_and_ragged_patterns(b200, syn, oracle):
    """States >= S are missing (all-ones); pattern counts off the 128 tile."""
    for P in (1, 127, 129, 1000):
        pr = syn.make_problem(S=4, N=9, P=P, C=2, seed=P)
        rng = np.random.default_rng(P)
        pr.tip_states[rng.random(pr.tip_states.shape) < 0.1] = 4 + rng.integers(0, 3)
        _, l, _ = run_b200(b200, pr, "double", gradient=False)
        _, lo, _ = run_oracle(oracle, pr, gradient=False)
        assert rel(l, lo) <= 1e-10


def test_error_codes(b200, syn):
    pr = syn.make_problem(S=4, N=6, P=50, C=2, seed=1)
    pref, req = gpu_flags("double")
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(inst)
    bad = np.array([[pr.root, -1, -1, 9999, 0, 1, 1]], dtype=np.int32)
    assert inst.updatePartials(bad, check=False) == -5
    assert inst.transposeTransitionMatrices([0], [0], check=False) == -5
    code, _ = inst.calculateRootLogLikelihoods([pr.n_buffers + 5], [0], [0], [-1], check=False)
    assert code == -5
    # NaN partials -> BEAGLE_ERROR_FLOATING_POINT, value still written
    nanp = np.full(pr.C * pr.P * pr.S, np.nan)
    inst.setPartials(pr.root, nanp)
    code, v = inst.calculateRootLogLikelihoods([pr.root], [0], [0], [-1], check=False)
    assert code == -8 and np.isnan(v)
    inst.finalize()
    assert b200.fn["SetPatternWeights"](inst.h if inst.h is not None else 12345, None) == -4


@pytest.mark.slow
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("name", ["gtr4_n128_p100k", "aa20_n64_p20k", "codon61_n32_p10k"])
def test_full_size_configs(b200, syn, oracle, name, precision):
    pr = syn.config_problem(name)
    inst, lnl, g = run_b200(b200, pr, precision)
    inst.finalize()
    _, lo, go = run_oracle(oracle, pr)
    tol = TOL[precision]
    assert rel(lnl, lo) <= tol["lnl"], (lnl, lo, rel(lnl, lo))
    assert grad_err(g, go) <= tol["grad"], grad_err(g, go)


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("variant", list(range(15)))
def test_s4_kernel_variants(b200, syn, oracle, monkeypatch, precision, variant):
    """Every S = 4 op-walk and derivative kernel shape the autotuner can pick
    (forced through BEAGLE_B200_FORCE_VARIANT) against the oracle, with C = 4
    (lane-group shapes; tips as states and as partials) and C = 3
    (thread-per-pattern walk)."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    for C, amb in ((4, 0.0), (4, 0.02), (3, 0.0)):
        pr = syn.make_problem(S=4, N=20, P=2900, C=C, seed=40 + variant, rescale=True,
                              ambiguous=amb)
        _, lnl, g = run_b200(b200, pr, precision)
        _, lo, go = run_oracle(oracle, pr)
        tol = TOL[precision]
        assert rel(lnl, lo) <= tol["lnl"], (C, lnl, lo)
        assert grad_err(g, go) <= tol["grad"], (C, grad_err(g, go))


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("variant", [7, 8, 14])
def test_s4_parameter_walks_longer_than_one_launch(b200, syn, oracle, monkeypatch, precision,
                                                   variant):
    """The parameter-list walks (7, 8, and 14 with staged matrices) take 256
    ops a launch: a 300-taxon tree (299 post-order, 598 pre-order ops) runs
    as consecutive launches."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=4, N=300, P=700, C=4, seed=77 + variant, rescale=True)
    inst, lnl, g = run_b200(b200, pr, precision)
    tv = inst.tunedVariants()
    assert tv["post"] == variant and tv["pre"] == variant, tv
    _, lo, go = run_oracle(oracle, pr)
    tol = TOL[precision]
    assert rel(lnl, lo) <= tol["lnl"], (lnl, lo)
    assert grad_err(g, go) <= tol["grad"], grad_err(g, go)
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("variant", [9, 10, 12])
def test_s4_slot_walks_more_live_values_than_slots(b200, syn, oracle, monkeypatch, precision,
                                                   variant):
    """The slot walks on a post-order list in height order (every cherry
    first, then their parents, ...): far more results are live at once than
    there are slots, so most operands come back from device memory; and with
    the pre-order list reversed per level likewise."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=4, N=96, P=1100, C=4, seed=321, rescale=True)
    ops = pr.post_ops()
    height = {}
    for op in ops:                      # post order: children first
        height[op[0]] = 1 + max(height.get(op[3], 0), height.get(op[5], 0))
    by_height = ops[np.argsort([height[o[0]] for o in ops], kind="stable")]
    pref, req = gpu_flags(precision)
    res = []
    for x in (b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req),
              oracle.OracleInstance(*pr.create_args(), flags=SCALERS_LOG)):
        pr.load(x)
        x.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, pr.lengths)
        x.updatePartials(by_height, -1)
        x.resetScaleFactors(pr.cumulative)
        x.accumulateScaleFactors(np.arange(pr.N - 1, dtype=np.int32), pr.cumulative)
        res.append(x.calculateRootLogLikelihoods([pr.root], [0], [0], [pr.cumulative]))
    assert rel(res[0], res[1]) <= TOL[precision]["lnl"], res


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,C,variant", [(4, 4, 1), (4, 4, 4), (4, 4, 14), (4, 3, 0), (20, 4, 0),
                                         (20, 4, 1)])
def test_partitions(b200, syn, oracle, monkeypatch, precision, S, C, variant):
    """updatePartialsByPartition / updatePrePartialsByPartition (one launch
    each over every partition's ops) and calculateRootLogLikelihoodsByPartition
    against the oracle, for each kernel family the partitions run on."""
    from helpers import PRE_AUTO, SCALERS_LOG, partitioned_args, run_partitioned
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=S, N=10, P=777, C=C, seed=90 + S + C, rescale=True)
    args = partitioned_args(pr, 3)
    pref, req = gpu_flags(precision, auto_transpose=True)
    inst = b200.create(*args, preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*args, flags=SCALERS_LOG)
    res = []
    for x in (inst, oi):
        pr.load(x)
        res.append(run_partitioned(x, pr, 3))
    (b1, t1), (b2, t2) = res
    tol = TOL[precision]["lnl"]
    assert np.max(np.abs(b1 - b2) / np.abs(b2)) <= tol and rel(t1, t2) <= tol
    big = 1e-9 if precision == "double" else 2e-4
    for v in [pr.root, pr.pre(0), pr.pre(pr.N), pr.pre(pr.B - 1)]:
        a, b = inst.getPartials(v), oi.getPartials(v)
        assert np.max(np.abs(a - b)) <= big * np.max(np.abs(b)), v
    cum0 = 3 * (pr.N - 1)
    for s in [0, pr.N - 2, (pr.N - 1) + 3, cum0, cum0 + 2]:
        a, b = inst.getScaleFactors(s), oi.getScaleFactors(s)
        assert np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))) <= big, s
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,derivs", [(4, False), (4, True), (20, True)])
def test_edge_by_partition(b200, syn, oracle, precision, S, derivs):
    """calculateEdgeLogLikelihoodsByPartition (per-partition launches over
    pattern ranges) against the oracle: lnL and derivative sums per partition,
    totals, site values; internal and tip children; d1 alone -> -7."""
    from helpers import PRE_AUTO, SCALERS_LOG, edge_by_partition, partitioned_args, \
        run_partitioned
    pr = syn.make_problem(S=S, N=10, P=777, C=4, seed=110 + S, rescale=True)
    args = partitioned_args(pr, 3)
    pref, req = gpu_flags(precision, auto_transpose=True)
    inst = b200.create(*args, preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*args, flags=SCALERS_LOG)
    got = []
    for x in (inst, oi):
        pr.load(x)
        run_partitioned(x, pr, 3)
        got.append([edge_by_partition(x, pr, 3, v, derivs) for v in (pr.N + 2, 1)])
    tol = TOL[precision]
    for (g, site_g), (o, site_o) in zip(*got):
        assert g[0] == o[0] == 0
        assert np.max(np.abs(g[1] - o[1]) / np.abs(o[1])) <= tol["lnl"]
        assert rel(g[2], o[2]) <= tol["lnl"]
        assert np.max(np.abs(site_g - site_o) / np.abs(site_o)) <= 100 * tol["lnl"]
        if derivs:
            for a, b in ((g[3], o[3]), (g[5], o[5])):
                assert np.max(np.abs(a - b)) <= tol["grad"] * max(1.0, np.max(np.abs(b)))
            assert abs(g[4] - o[4]) <= tol["grad"] * max(1.0, abs(o[4]))
            assert abs(g[6] - o[6]) <= tol["grad"] * max(1.0, abs(o[6]))
    code = inst.calculateEdgeLogLikelihoodsByPartition([pr.root], [1], [1], [3 * pr.B + 1],
                                                       None, [0], [0], [-1], [0],
                                                       check=False)[0]
    assert code == -7
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,kind", [(4, "multiple"), (4, "categories"), (20, "multiple"),
                                    (20, "categories"), (61, "categories")])
def test_model_variant_matrices(b200, syn, oracle, precision, S, kind):
    """updateTransitionMatricesWithMultipleModels / ...WithModelCategories on
    the device (P, dP, d2P from the FP64 cubes of three eigen systems) and the
    lnL of a tree built on them, against the oracle."""
    from helpers import model_variant_args, run_model_variants
    pr = syn.make_problem(S=S, N=8, P=300, C=4, seed=140 + S)
    args = model_variant_args(pr)
    pref, req = gpu_flags(precision)
    inst = b200.create(*args, preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*args, flags=SCALERS_LOG)
    got = []
    for x in (inst, oi):
        pr.load(x)
        got.append(run_model_variants(x, pr, kind))
    (l1, m1), (l2, m2) = got
    assert rel(l1, l2) <= TOL[precision]["lnl"]
    mt = 1e-12 if precision == "double" else 1e-6
    for a, b in zip(m1, m2):
        assert np.max(np.abs(a - b)) <= mt * max(1.0, np.max(np.abs(b)))
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S", [4, 20])
def test_fixed_scaling_transpose_convolve_and_set_matrices(b200, syn, oracle, precision, S):
    """Read-only (fixed) scale factors, matrix transposition and convolution,
    matrices set by the caller (setTransitionMatrices, setDifferentialMatrix),
    and a post-order op on a convolved matrix (an epoch boundary), against
    the oracle."""
    pr = syn.make_problem(S=S, N=10, P=190, C=2, seed=150 + S, rescale=True)
    pref, req = gpu_flags(precision, log_scalers=False)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*pr.create_args(), flags=SCALERS_RAW)
    rng = np.random.default_rng(S)
    given = rng.random((2, pr.C * S * S))
    res = []
    for x in (inst, oi):
        pr.load(x)
        x.updateTransitionMatrices(0, np.arange(pr.B), None, None, pr.lengths)
        x.updatePartials(pr.post_ops())
        ops = pr.post_ops()
        ops[:, 2] = ops[:, 1]      # read the factors just written ...
        ops[:, 1] = -1             # ... without writing new ones
        x.updatePartials(ops)
        x.transposeTransitionMatrices([0, 1], [pr.B + 1, pr.B + 2])
        x.convolveTransitionMatrices([0], [1], [pr.B + 3])
        if x is inst:
            x.setTransitionMatrices([pr.B + 4, pr.B + 5], given.reshape(-1), [1.0, 0.5])
            x.setDifferentialMatrix(pr.B + 6, given[0])
        else:
            x.setTransitionMatrix(pr.B + 4, given[0], 1.0)
            x.setTransitionMatrix(pr.B + 5, given[1], 0.5)
            x.setTransitionMatrix(pr.B + 6, given[0], 0.0)
        # one more op with a convolved matrix and a caller-set one
        c1, c2 = (int(v) for v in pr.children[pr.root])
        x.updatePartials(np.array([[pr.root, -1, -1, c1, pr.B + 3, c2, pr.B + 5]],
                                  dtype=np.int32))
        res.append([x.getPartials(pr.root)] +
                   [x.getTransitionMatrix(m) for m in (pr.B + 1, pr.B + 3, pr.B + 5, pr.B + 6)])
    tol = 1e-12 if precision == "double" else 2e-5
    for a, b in zip(*res):
        assert np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("log_scalers", [True, False])
def test_scale_factor_calls_and_getters(b200, syn, oracle, precision, log_scalers):
    """Accumulate / remove / copy / reset of scale factors, whole and by
    partition, read back through root log-likelihoods and getScaleFactors;
    setRootPrePartials; an edge lnL's getDerivatives and getSiteDerivatives;
    waitForPartials -- against the oracle (RAW and LOG scalers)."""
    pr = syn.make_problem(S=4, N=12, P=500, C=3, seed=170, rescale=True)
    pref, req = gpu_flags(precision, log_scalers=log_scalers)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    oi = oracle.OracleInstance(*pr.create_args(),
                               flags=SCALERS_LOG if log_scalers else SCALERS_RAW)
    nodes = list(range(pr.N - 1))
    cum, cum2 = pr.cumulative, pr.N - 1          # N - 1: a free scale buffer here
    parts = (np.arange(pr.P) >= 200).astype(np.int32)
    res = []
    for x in (inst, oi):
        pr.load(x)
        idx = np.arange(pr.B)
        x.updateTransitionMatrices(0, idx, idx + pr.B + 1, None, pr.lengths)
        x.updatePartials(pr.post_ops())
        x.resetScaleFactors(cum)
        x.accumulateScaleFactors(nodes, cum)
        x.removeScaleFactors(nodes[:3], cum)
        x.copyScaleFactors(cum2, cum)
        x.accumulateScaleFactors(nodes[:3], cum)
        out = [x.calculateRootLogLikelihoods([pr.root], [0], [0], [cum]),
               x.calculateRootLogLikelihoods([pr.root], [0], [0], [cum2]),
               x.getScaleFactors(cum2)]
        x.setPatternPartitions(2, parts)
        for q in (0, 1):
            x.resetScaleFactorsByPartition(cum2, q)
            x.accumulateScaleFactorsByPartition(nodes, cum2, q)
        x.removeScaleFactorsByPartition(nodes[:4], cum2, 1)
        byp, tot = x.calculateRootLogLikelihoodsByPartition([pr.root] * 2, [0, 0], [0, 0],
                                                            [cum2, cum2], [0, 1])
        out += [np.asarray(byp), tot, x.getScaleFactors(cum2)]
        x.setRootPrePartials([pr.pre(pr.root)], [0])
        out.append(x.getPartials(pr.pre(pr.root)))
        v = pr.N + 1
        x.updatePrePartials(pr.pre_ops())
        code, lnl, d1, d2 = x.calculateEdgeLogLikelihoods(pr.pre(int(pr.parent[v])), v, v,
                                                          v + pr.B + 1, None, 0, 0, -1)
        out += [lnl, d1]
        if x is inst:
            assert x.waitForPartials([pr.root]) == 0
            g1, _ = x.getDerivatives()
            assert g1 == d1
            site_d1, _ = x.getSiteDerivatives()
        else:
            site_d1 = x.site_d1
        out.append(site_d1)
        res.append(out)
    tol = TOL[precision]
    g, o = res
    for k in (0, 1, 4, 7):
        assert rel(g[k], o[k]) <= tol["lnl"], k
    assert np.max(np.abs(g[3] - o[3]) / np.abs(o[3])) <= tol["lnl"]
    for k in (2, 5):
        assert np.max(np.abs(g[k] - o[k]) / np.maximum(1.0, np.abs(o[k]))) <= \
            (1e-12 if precision == "double" else 1e-5), k
    assert np.max(np.abs(g[6] - o[6])) <= 1e-15 * np.max(np.abs(o[6])) + 1e-7 * (precision != "double")
    assert abs(g[8] - o[8]) <= tol["grad"] * max(1.0, abs(o[8]))
    assert np.max(np.abs(g[9] - o[9])) <= tol["grad"] * max(1.0, np.max(np.abs(o[9])))
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S", [4, 20])
def test_repeat_determinism_and_site_derivative_sums(b200, syn, precision, S):
    """Repeated evaluations give the same lnL and gradient bits (fixed-order
    reductions, the autotuner's pick cached after the first call), as the
    reference's rep-to-rep check expects (synthetictest.cpp:2436-2447); and
    the per-site derivatives, weighted and summed, give the reduced sums
    (hmctest.cpp:716-722), as do the sums of squares."""
    pr = syn.make_problem(S=S, N=18, P=1500, C=4, seed=180 + S, rescale=True)
    inst, l0, g0 = run_b200(b200, pr, precision)
    for _ in range(3):
        l1, g1 = pr.evaluate(inst, transposed_pre=S > 4)
        assert l1 == l0
        assert np.array_equal(g1, g0)
    nonroot = np.arange(pr.B, dtype=np.int32)
    site, sums, sumsq = inst.calculateEdgeDerivatives(
        nonroot, nonroot + pr.pre(0), np.full(pr.B, pr.B, dtype=np.int32), [0])
    # the per-site output may come from another derivative kernel shape than
    # the sums-only call: equal to FP64 reduction rounding
    assert np.max(np.abs(sums - g0)) <= 1e-12 * np.max(np.abs(g0))
    w = pr.patw
    assert np.max(np.abs(site @ w - sums)) <= 1e-10 * np.max(np.abs(sums))
    assert np.max(np.abs((site * site) @ w - sumsq)) <= 1e-9 * np.max(np.abs(sumsq))
    inst.finalize()
