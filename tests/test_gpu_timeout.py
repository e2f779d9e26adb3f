"""Bounded kernel waits and their error path.

Every wait in this library's kernels is bounded.  A wait that runs out sets a
device flag; the kernel ends without its result (after waiting, with the full
bound, for its own copies still in flight), and the next result call returns
BEAGLE_ERROR_GENERAL (-1) instead of numbers.  The reference's CUDA path exits
the process instead (GPU/GPUInterfaceCUDA.cpp:98-104).

* test_bulk_derivative_wait_runs_out makes a real wait run out: the bulk-copy
  derivative (autotuner variant 6 of the 4-state derivative) with its stage
  waits bounded at one clock cycle (BEAGLE_B200_WAIT_CYCLES), so they give up
  before any copy can land.  Every access of that kernel stays in bounds
  whatever the wait returns; only the values are wrong, and they are not
  delivered.
* test_injected_timeout_is_reported raises the same flag from the host
  (beagleB200InjectKernelTimeout) for both kernel families.

In both, the following evaluation on the same instance must succeed and match
the oracle."""
import numpy as np
import pytest

from helpers import TOL, gpu_flags, grad_err, rel, run_oracle

pytestmark = pytest.mark.gpu


def _instance(b200, pr, precision):
    pref, req = gpu_flags(precision)
    inst = b200.create(*pr.create_args(), resources=[0], preferenceFlags=pref,
                       requirementFlags=req)
    pr.load(inst)
    return inst


def _derivatives(inst, pr):
    nonroot = np.arange(pr.B, dtype=np.int32)
    _, sums, _ = inst.calculateEdgeDerivatives(
        nonroot, nonroot + pr.pre(0), np.full(pr.B, pr.B, dtype=np.int32), [0],
        per_site=False, sums=True, sumsq=False)
    return sums


@pytest.mark.parametrize("precision", ["single", "double"])
def test_bulk_derivative_wait_runs_out(b200, syn, oracle, monkeypatch, precision):
    pr = syn.make_problem(S=4, N=16, P=20000, C=4, seed=61, rescale=True)
    _, lo, go = run_oracle(oracle, pr)
    monkeypatch.setenv("BEAGLE_B200_FORCE_VARIANT", "-1,-1,6")     # bulk-copy derivative
    inst = _instance(b200, pr, precision)
    lnl, g = pr.evaluate(inst)                       # full bound: a normal evaluation
    assert rel(lnl, lo) <= TOL[precision]["lnl"]
    assert grad_err(g, go) <= TOL[precision]["grad"]
    monkeypatch.setenv("BEAGLE_B200_WAIT_CYCLES", "1")
    with pytest.raises(b200_error(b200)) as e:
        _derivatives(inst, pr)
    assert e.value.code == -1
    monkeypatch.delenv("BEAGLE_B200_WAIT_CYCLES")
    # the same instance evaluates again, and right
    lnl2, g2 = pr.evaluate(inst)
    assert rel(lnl2, lo) <= TOL[precision]["lnl"]
    assert grad_err(g2, go) <= TOL[precision]["grad"]
    inst.finalize()


def b200_error(lib):
    import importlib
    return importlib.import_module("beagle-lib_b200").binding.BeagleError


@pytest.mark.parametrize("which", [0, 1])
def test_injected_timeout_is_reported(b200, syn, oracle, which):
    pr = syn.make_problem(S=20, N=10, P=700, C=2, seed=62 + which, rescale=True)
    _, lo, go = run_oracle(oracle, pr)
    inst = _instance(b200, pr, "single")
    tr = True                                        # S > 4: transposed pre-order matrices
    lnl, g = pr.evaluate(inst, transposed_pre=tr)
    assert rel(lnl, lo) <= TOL["single"]["lnl"]
    inst.updateTransitionMatrices(0, np.arange(pr.B, dtype=np.int32), None, None, pr.lengths)
    inst.updatePartials(pr.post_ops())
    inst.injectKernelTimeout(which)
    with pytest.raises(b200_error(b200)) as e:
        inst.calculateRootLogLikelihoods([pr.root], [0], [0], [-1])
    assert e.value.code == -1
    lnl2, g2 = pr.evaluate(inst, transposed_pre=tr)
    assert rel(lnl2, lo) <= TOL["single"]["lnl"]
    assert grad_err(g2, go) <= TOL["single"]["grad"]
    inst.finalize()


def test_inject_rejects_unknown_family(b200, syn):
    pr = syn.make_problem(S=4, N=6, P=100, C=1, seed=63)
    inst = _instance(b200, pr, "single")
    with pytest.raises(b200_error(b200)) as e:
        inst.injectKernelTimeout(2)
    assert e.value.code == -5
    inst.finalize()
