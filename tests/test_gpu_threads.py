"""Several client threads, each driving its own instance at the same time, as
a BEAGLE client with one thread per partition or chain does (the reference's
synthetictest --clientthreads).  The instance table, the autotuner's cache
and the per-thread launch-parameter buffers are shared by the threads; each
thread's lnL and gradient must match the same evaluation run alone and the
oracle.  ctypes releases the GIL for the duration of every C call, so the
threads' calls do overlap.

The instances here run the 4-state walks and the FP64 CUDA-core kernels; the
FP32 tensor-core kernels of S > 4 are not mixed in (their cross-stream TMEM
sharing is made safe by construction, see k_tc.cu's tc_smem)."""
import threading

import numpy as np
import pytest

from helpers import TOL, grad_err, rel, run_b200, run_oracle, gpu_flags

pytestmark = pytest.mark.gpu

CASES = [(4, "single", 4), (4, "double", 4), (20, "double", 4), (4, "single", 1),
         (61, "double", 2), (4, "single", 8), (4, "double", 2), (20, "double", 1)]


def test_client_threads(b200, syn, oracle):
    probs = [syn.make_problem(S=S, N=14 + 3 * i, P=900 + 70 * i, C=C, seed=300 + i,
                              rescale=True)
             for i, (S, _, C) in enumerate(CASES)]
    alone = []
    for pr, (S, prec, _) in zip(probs, CASES):
        inst, lnl, g = run_b200(b200, pr, prec)
        inst.finalize()
        alone.append((lnl, g))
    results = [None] * len(CASES)
    errors = []
    start = threading.Barrier(len(CASES))

    def work(i):
        try:
            pr = probs[i]
            S, prec, _ = CASES[i]
            pref, req = gpu_flags(prec)
            inst = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
            pr.load(inst)
            start.wait(timeout=60)
            out = []
            for _ in range(4):
                out.append(pr.evaluate(inst, transposed_pre=S > 4))
            inst.finalize()
            results[i] = out
        except Exception as e:          # reported below, in the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(CASES))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    for i, (pr, (S, prec, _)) in enumerate(zip(probs, CASES)):
        tol = TOL[prec]
        lnl0, g0 = alone[i]
        for lnl, g in results[i]:
            assert rel(lnl, lnl0) <= tol["lnl"], (i, lnl, lnl0)
            assert grad_err(g, g0) <= tol["grad"], i
        # The 61-state case is ill-conditioned at this seed: the compiled
        # reference itself differs from the oracle by 5e-8 in the gradient
        # (one branch's derivative is 1.4e6) and 8e-11 in lnL.
        lt, gt = (1e-9, 1e-6) if S == 61 else (tol["lnl"], tol["grad"])
        _, lo, go = run_oracle(oracle, pr)
        assert rel(results[i][-1][0], lo) <= lt, i
        assert grad_err(results[i][-1][1], go) <= gt, i
