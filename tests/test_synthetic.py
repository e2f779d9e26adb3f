"""Host-side logic on the CPU: workload generators and the operation lists."""
import numpy as np
import pytest


def test_random_tree_is_binary_and_rooted(syn):
    rng = np.random.default_rng(0)
    for N in (2, 3, 16, 128):
        par, ch = syn.random_tree(N, rng)
        root = 2 * N - 2
        assert par[root] == -1 and (par[:root] >= 0).all()
        kids = ch[N:]
        assert (kids >= 0).all() and len(set(kids.reshape(-1))) == 2 * N - 2


def test_post_and_pre_orders(syn):
    pr = syn.make_problem(S=4, N=30, P=10, C=1, seed=2, rescale=True)
    done = set(range(pr.N))
    for op in pr.post_ops():
        assert op[3] in done and op[5] in done
        done.add(op[0])
    assert pr.root in done
    seen = {pr.pre(pr.root)}
    for op in pr.pre_ops():
        assert op[3] in seen
        seen.add(op[0])
    assert len(pr.pre_ops()) == pr.B


@pytest.mark.parametrize("S", [4, 20, 61])
def test_models_are_reversible_and_normalised(syn, S):
    pr = syn.make_problem(S=S, N=4, P=5, C=4, seed=S)
    Q, pi = pr.Q, pr.pi
    assert np.allclose(Q.sum(axis=1), 0, atol=1e-12)
    assert np.isclose(-np.dot(pi, np.diag(Q)), 1.0)
    assert np.allclose(pi[:, None] * Q, (pi[:, None] * Q).T, atol=1e-12)
    assert np.allclose(pr.V @ np.diag(pr.lam) @ pr.Vi, Q, atol=1e-10)
    assert np.isclose(np.dot(pr.rates, pr.catw), 1.0)


def test_codon_model_has_61_sense_codons(syn):
    Q, pi = syn.codon_model(np.random.default_rng(1))
    assert Q.shape == (61, 61)
    # single-nucleotide neighbours only: each codon has at most 9 neighbours
    assert ((Q > 0).sum(axis=1) <= 9).all()


def test_batched_problem_mix(syn):
    probs = syn.batched_problems(count=40, seed=7, max_patterns=2000)
    assert {p.S for p in probs} <= {4, 20}
    assert {p.C for p in probs} <= {1, 4, 8}
    assert all(16 <= p.N <= 256 and 100 <= p.P <= 2000 for p in probs)


def test_finite_difference_gradient_on_oracle(syn, oracle):
    """The edge-derivative gradient equals central finite differences of lnL
    (the check hmctest.R:216-236 makes), on the oracle."""
    pr = syn.make_problem(S=4, N=8, P=60, C=4, seed=11, rescale=True)
    inst = oracle.OracleInstance(*pr.create_args(), flags=1 << 10)
    pr.load(inst)
    lnl, g = pr.evaluate(inst)
    h = 1e-6
    for b in (0, 3, pr.B - 1):
        t = pr.lengths.copy()
        t[b] += h
        lp, _ = pr.evaluate(inst, gradient=False, lengths=t)
        t[b] -= 2 * h
        lm, _ = pr.evaluate(inst, gradient=False, lengths=t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[b]) <= 1e-5 * max(1.0, abs(g[b]))
