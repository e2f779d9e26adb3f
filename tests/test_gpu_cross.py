"""beagleCalculateCrossProductDerivative on the GPU against the oracle: the
S x S sums over all branches of an evaluated tree (compact tips with missing
states, ambiguous tips as partials, rescaled partials), added to the caller's
array as the reference does."""
import numpy as np
import pytest

from helpers import SCALERS_LOG, TOL, gpu_flags

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S,C,amb", [(4, 4, 0.03), (4, 1, 0.0), (20, 2, 0.0), (61, 4, 0.0)])
def test_cross_products_match_oracle(b200, syn, oracle, precision, S, C, amb):
    pr = syn.make_problem(S=S, N=12, P=700, C=C, seed=70 + S + C, rescale=True, ambiguous=amb)
    for t in (0, 1):
        if t not in pr.tip_partials:
            pr.tip_states[t][::9] = S
    nodes = np.arange(pr.B, dtype=np.int32)
    pref, req = gpu_flags(precision)
    g = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    o = oracle.OracleInstance(*pr.create_args(), flags=SCALERS_LOG)
    outs = []
    for inst, tr in ((g, S > 4), (o, False)):
        pr.load(inst)
        pr.evaluate(inst, transposed_pre=tr)
        out = np.full(S * S, 1.0)
        inst.calculateCrossProductDerivative(nodes, nodes + pr.pre(0), [0], [0], pr.lengths, out)
        outs.append(out)
    err = np.max(np.abs(outs[0] - outs[1])) / np.max(np.abs(outs[1]))
    assert err <= (1e-10 if precision == "double" else TOL["single"]["grad"]), err
    g.finalize()
