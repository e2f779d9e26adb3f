"""beagleB200UpdatePartialsWithRootLogLikelihood: updatePartials, the list's
cumulative scale factors (reset, then accumulated) and the root lnL in one
call, against the separate calls on the same instance and against the
oracle: lnL, site lnL, the cumulative buffer and the scale buffers.  S = 4
with C = 1, 2, 4, 8 runs the fused walk; C = 3, S = 20, a root that is not the
last op's destination and lists of more than 256 ops run as the separate
calls.  LOG and RAW scalers, no cumulative buffer, ASYNCH delivery."""
import numpy as np
import pytest

from helpers import TOL, gpu_flags, rel, run_oracle

pytestmark = pytest.mark.gpu

ASYNCH = 1 << 3


def _separate(inst, pr, cum):
    inst.updatePartials(pr.post_ops(), -1)
    if cum >= 0:
        inst.resetScaleFactors(cum)
        inst.accumulateScaleFactors(np.arange(pr.N - 1, dtype=np.int32), cum)
    return inst.calculateRootLogLikelihoods([pr.root], [0], [0], [cum])


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("log_scalers", [True, False])
@pytest.mark.parametrize("S,C,N", [(4, 1, 40), (4, 2, 40), (4, 4, 40), (4, 8, 40), (4, 3, 40),
                                   (20, 4, 12), (4, 4, 300)])
def test_post_root_matches_separate_calls(b200, syn, oracle, precision, log_scalers, S, C, N):
    pr = syn.make_problem(S=S, N=N, P=2100, C=C, seed=700 + S + C + N, rescale=True)
    pref, req = gpu_flags(precision, log_scalers=log_scalers, auto_transpose=True)
    inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(inst)
    inst.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, pr.lengths)
    cum = pr.cumulative
    l0 = _separate(inst, pr, cum)
    site0, cum0 = inst.getSiteLogLikelihoods(), inst.getScaleFactors(cum)
    sc0 = [inst.getScaleFactors(s) for s in range(pr.N - 1)]
    inst.accumulateScaleFactors([0, 1], cum)          # the call must reset the buffer
    l1 = inst.updatePartialsWithRootLogLikelihood(pr.post_ops(), cum, pr.root, 0, 0)
    site1, cum1 = inst.getSiteLogLikelihoods(), inst.getScaleFactors(cum)
    dbl = precision == "double"
    assert rel(l1, l0) <= (1e-13 if dbl else 1e-6), (l1, l0)
    assert np.max(np.abs(site1 - site0) / np.abs(site0)) <= (1e-13 if dbl else 1e-6)
    # RAW FP32 factors: the fused walk adds the FP32 exponent-split log of
    # each factor, the accumulate call the FP64 log of the stored factor
    ctol = 1e-12 if (dbl or log_scalers) else 1e-5
    assert np.max(np.abs(cum1 - cum0)) <= ctol * max(1.0, np.max(np.abs(cum0)))
    for s in range(pr.N - 1):
        a = inst.getScaleFactors(s)
        assert np.max(np.abs(a - sc0[s]) / np.maximum(1.0, np.abs(sc0[s]))) <= \
            (1e-13 if dbl else 1e-6), s
    _, lo, _ = run_oracle(oracle, pr, gradient=False, log_scalers=log_scalers)
    assert rel(l1, lo) <= TOL[precision]["lnl"]
    # no cumulative buffer: lnL of the rescaled root alone, as the reference
    inst.updatePartials(pr.post_ops(), -1)
    l2 = inst.calculateRootLogLikelihoods([pr.root], [0], [0], [-1])
    l3 = inst.updatePartialsWithRootLogLikelihood(pr.post_ops(), -1, pr.root, 0, 0)
    assert rel(l3, l2) <= (1e-13 if dbl else 1e-6)
    inst.finalize()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_post_root_other_root_and_asynch(b200, syn, precision):
    """A root that is not the last op's destination (the separate calls, on
    that root), and an ASYNCH instance: nothing written at the call, the
    value delivered by getLogLikelihood."""
    pr = syn.make_problem(S=4, N=30, P=1500, C=4, seed=733, rescale=False)
    pref, req = gpu_flags(precision)
    for flags in (0, ASYNCH):
        inst = b200.create(*pr.create_args(), preferenceFlags=pref | flags, requirementFlags=req)
        pr.load(inst)
        inst.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, pr.lengths)
        ops = pr.post_ops()
        other = int(ops[-2][0])                       # an internal node below the root
        inst.updatePartials(ops, -1)
        lo = inst.calculateRootLogLikelihoods([other], [0], [0], [-1])
        if flags:
            lo = inst.getLogLikelihood()
        l1 = inst.updatePartialsWithRootLogLikelihood(ops, -1, other, 0, 0)
        if flags:
            l1 = inst.getLogLikelihood()
        assert rel(l1, lo) <= 1e-13
        inst.updatePartials(ops, -1)
        lr = inst.calculateRootLogLikelihoods([pr.root], [0], [0], [-1])
        if flags:
            lr = inst.getLogLikelihood()
        l2 = inst.updatePartialsWithRootLogLikelihood(ops, -1, pr.root, 0, 0)
        if flags:
            l2 = inst.getLogLikelihood()
        assert rel(l2, lr) <= (1e-13 if precision == "double" else 1e-6)
        inst.finalize()
