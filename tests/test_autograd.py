"""Gradient checks through the torch.autograd.Function of tests/torch_lnl.py:
backward (the pre-order adjoint) against central finite differences of the
forward lnL.  CPU: on the oracle.  GPU: on libbeagle_b200.so through the C
ABI, FP64 against its own differences and the mixed path against the FP64
differences (gradient relative error <= 1e-4)."""
import numpy as np
import pytest
import torch

from helpers import gpu_flags
from torch_lnl import central_differences, lnl


def _check(inst, pr, tol, transposed=False, fd_inst=None, h=1e-6):
    t = torch.tensor(pr.lengths, dtype=torch.float64, requires_grad=True)
    out = lnl(t, inst, pr, transposed)
    out.backward()
    g = t.grad.numpy()
    branches = [0, 1, pr.N // 2, pr.B - 2, pr.B - 1]
    fd = central_differences(fd_inst or inst, pr, pr.lengths.copy(), branches, h=h,
                             transposed_pre=transposed)
    err = np.max(np.abs(g[branches] - fd)) / np.max(np.abs(fd))
    assert err <= tol, (err, g[branches], fd)
    return out.item()


@pytest.mark.parametrize("S", [4, 20])
def test_oracle_gradient_matches_finite_differences(syn, oracle, S):
    pr = syn.make_problem(S=S, N=8, P=120, C=2, seed=11 + S, rescale=True)
    oi = oracle.OracleInstance(*pr.create_args(), flags=1 << 10)
    pr.load(oi)
    _check(oi, pr, 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("S", [4, 20, 61])
def test_b200_gradient_matches_finite_differences(b200, syn, S):
    pr = syn.make_problem(S=S, N=12, P=900, C=4, seed=21 + S, rescale=True)
    pref, req = gpu_flags("double")
    i64 = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(i64)
    tr = S > 4
    # FP64 on the GPU: the differences' own error (lnL rounding / step, step^2
    # truncation) is about 1e-6 here, so the bar is 1e-5.
    _check(i64, pr, 1e-5, transposed=tr, h=1e-5)
    pref, req = gpu_flags("single")
    i32 = b200.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
    pr.load(i32)
    # mixed-path gradient against finite differences of the FP64 lnL
    _check(i32, pr, 1e-4, transposed=tr, fd_inst=i64, h=1e-5)
    i64.finalize()
    i32.finalize()
