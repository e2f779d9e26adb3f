"""The FP32 path for 4 < S <= 64 has kernel families that compute the same
results: CUDA-core cluster kernels (variant 0), tensor-core tcgen05 kernels
with 3 x tf32 split products (variant 1, k_tc.cu), and for the walks the same
tensor-core kernels fed by TMA (variant 2; the derivative runs variant 1 then).
Each is forced in turn
(BEAGLE_B200_FORCE_VARIANT) and checked against the oracle: lnL and gradient
at the mixed-path tolerances, and the intermediate buffers (partials, scale
factors, pre-order partials, per-site derivatives) at 2e-4 of the buffer
maximum: the FP32 worst case of a 64-term sum is 64 x 2^-24 = 3.8e-6 relative
per matrix-vector product, compounded over two children and ~9 tree levels.  The state counts cover every padded width the tensor-core
kernels have (N = 16, 32, 48, 64) and both K layouts (one chunk, two chunks)."""
import numpy as np
import pytest

from helpers import TOL, grad_err, rel, run_b200, run_oracle

pytestmark = pytest.mark.gpu

CASES = [(5, 3), (13, 2), (20, 4), (33, 2), (48, 8), (61, 4), (61, 1)]


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("S,C", CASES, ids=[f"S{s}C{c}" for s, c in CASES])
def test_fp32_generic_kernels(b200, syn, oracle, monkeypatch, variant, S, C):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=S, N=10, P=700, C=C, seed=500 + S + C, rescale=True,
                          ambiguous=0.01)
    inst, lnl, g = run_b200(b200, pr, "single")
    if variant == 2:   # the TMA-fed walks ran (no fallback to the CUDA-core kernels)
        tv = inst.tunedVariants()
        assert tv["post"] == 2 and tv["pre"] == 2, tv
    oi, lo, go = run_oracle(oracle, pr)
    tol = TOL["single"]
    assert rel(lnl, lo) <= tol["lnl"], (lnl, lo)
    assert grad_err(g, go) <= tol["grad"], grad_err(g, go)
    a, b = inst.getPartials(pr.root), oi.getPartials(pr.root)
    assert np.max(np.abs(a - b)) <= 2e-4 * np.max(np.abs(b))
    for s in range(pr.N - 1):
        a, b = inst.getScaleFactors(s), oi.getScaleFactors(s)
        assert np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))) <= 2e-4
    for v in [0, pr.N, pr.B - 1]:
        a, b = inst.getPartials(pr.pre(v)), oi.getPartials(pr.pre(v))
        assert np.max(np.abs(a - b)) <= 2e-4 * np.max(np.abs(b))
    nonroot = np.arange(pr.B, dtype=np.int32)
    dm = np.full(pr.B, pr.B, dtype=np.int32)
    d, _, _ = inst.calculateEdgeDerivatives(nonroot, nonroot + pr.pre(0), dm, [0])
    do, _, _ = oi.calculateEdgeDerivatives(nonroot, nonroot + pr.pre(0), dm, [0])
    assert np.max(np.abs(d - do)) <= 2e-4 * np.max(np.abs(do))
    inst.finalize()


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_fp32_generic_auto_transpose_and_raw_scalers(b200, syn, oracle, monkeypatch, variant):
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=61, N=8, P=300, C=2, seed=77, rescale=True)
    _, l1, g1 = run_b200(b200, pr, "single", auto_transpose=True)
    _, l2, g2 = run_b200(b200, pr, "single", log_scalers=False)
    _, lo, go = run_oracle(oracle, pr)
    assert rel(l1, lo) <= 1e-6 and rel(l2, lo) <= 1e-6
    assert grad_err(g1, go) <= 1e-4 and grad_err(g2, go) <= 1e-4


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("S", [20, 61])
def test_fp32_generic_missing_compact_states(b200, syn, oracle, monkeypatch, variant, S):
    """Compact tips with missing states (state S, an all-ones partial): the
    walks read the matrix's pad value for them (post-order child and
    pre-order sibling), and the derivative an all-ones row; every kernel
    family against the oracle, whose missing state is an all-ones partial
    on every path."""
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", str(variant))
    pr = syn.make_problem(S=S, N=12, P=650, C=4, seed=600 + S, rescale=True)
    rng = np.random.default_rng(S)
    pr.tip_states[rng.random(pr.tip_states.shape) < 0.08] = S
    inst, lnl, g = run_b200(b200, pr, "single")
    oi, lo, go = run_oracle(oracle, pr)
    assert rel(lnl, lo) <= TOL["single"]["lnl"], (lnl, lo)
    assert grad_err(g, go) <= TOL["single"]["grad"], grad_err(g, go)
    for v in [pr.root, pr.pre(0), pr.pre(pr.N)]:
        a, b = inst.getPartials(v), oi.getPartials(v)
        assert np.max(np.abs(a - b)) <= 2e-4 * np.max(np.abs(b)), v
    inst.finalize()
