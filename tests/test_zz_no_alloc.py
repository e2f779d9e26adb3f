"""The allocation-free root log-likelihood entry point
(beagleB200RootLogLikelihoodsNoAlloc), for callers that cannot let a library
call cudaMalloc because they own all device memory or must not trigger its
implicit synchronisation.

The test hands it device buffers that the test itself owns (torch tensors),
holding a root partials buffer read back from an instance.  Two calls in a row
must agree with the instance path (beagleB200CalculateRootLogLikelihoods) on
the same data within the tolerances of tests/helpers.py.  The second call
checks that leftovers in the shared scratch array do not leak into the
result.  This file is collected last so that a failing run has already run
every other test."""
import ctypes

import numpy as np
import pytest

from helpers import TOL, gpu_flags, rel

pytestmark = pytest.mark.gpu


def _device_layout(host_cps, C, P, S):
    """[C][P][S] -> [P][C][Sg] with Sg = S rounded up to 4."""
    Sg = (S + 3) // 4 * 4
    x = np.zeros((P, C, Sg))
    x[:, :, :S] = np.transpose(host_cps.reshape(C, P, S), (1, 0, 2))
    return x


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S", [4, 20])
def test_no_alloc_matches_instance_path(b200, syn, precision, S):
    import torch
    pr = syn.make_problem(S=S, N=20, P=3001, C=4, seed=41 + S, rescale=True)
    pref, req = gpu_flags(precision)
    inst = b200.create(*pr.create_args(), resources=[0], preferenceFlags=pref,
                       requirementFlags=req)
    pr.load(inst)
    lnl, _ = pr.evaluate(inst, gradient=False)
    site = inst.getSiteLogLikelihoods()
    root = inst.getPartials(pr.root)
    cum = inst.getScaleFactors(pr.cumulative)
    inst.finalize()

    dt = torch.float64 if precision == "double" else torch.float32
    dev = torch.device("cuda:0")
    rootd = torch.tensor(_device_layout(root, pr.C, pr.P, pr.S), dtype=dt, device=dev)
    catw = torch.tensor(pr.catw, dtype=torch.float64, device=dev)
    freqs = torch.tensor(pr.pi, dtype=torch.float64, device=dev)
    cumd = torch.tensor(cum, dtype=torch.float64, device=dev)
    patw = torch.tensor(pr.patw, dtype=torch.float64, device=dev)
    fn = b200.lib.beagleB200RootLogLikelihoodsNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        site_out = torch.full((pr.P,), float("nan"), dtype=torch.float64, device=dev)
        sum_out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        code = fn(0, ctypes.c_void_p(stream.cuda_stream), ctypes.c_void_p(rootd.data_ptr()),
                  1 if precision == "double" else 0, pr.S, pr.P, pr.C,
                  ctypes.c_void_p(catw.data_ptr()), ctypes.c_void_p(freqs.data_ptr()),
                  ctypes.c_void_p(cumd.data_ptr()), ctypes.c_void_p(patw.data_ptr()),
                  ctypes.c_void_p(site_out.data_ptr()), ctypes.c_void_p(sum_out.data_ptr()))
        assert code == 0, f"call {call} returned {code}"
        torch.cuda.synchronize(dev)
        got = float(sum_out.item())
        assert rel(got, lnl) <= TOL[precision]["lnl"], (call, got, lnl)
        s = site_out.cpu().numpy()
        assert np.max(np.abs(s - site) / np.abs(site)) <= 100 * TOL[precision]["lnl"]


def test_no_alloc_rejects_misaligned_partials(b200):
    """An offset view of the root partials (8 bytes into an allocation) is
    refused before any launch: the rows are read as 16-byte vectors."""
    import torch
    dev = torch.device("cuda:0")
    P, C, S = 256, 2, 4
    rootd = torch.ones(P * C * S + 2, dtype=torch.float64, device=dev)
    w = torch.full((max(P, S, C),), 0.25, dtype=torch.float64, device=dev)
    out = torch.zeros(P + 1, dtype=torch.float64, device=dev)
    fn = b200.lib.beagleB200RootLogLikelihoodsNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6
    p = ctypes.c_void_p
    code = fn(0, None, p(rootd.data_ptr() + 8), 1, S, P, C, p(w.data_ptr()), p(w.data_ptr()),
              None, p(w.data_ptr()), p(out.data_ptr()), p(out.data_ptr() + 8 * P))
    assert code == -5
    torch.cuda.synchronize(dev)
    assert float(out.abs().sum().item()) == 0.0      # nothing was written


def test_no_alloc_rejects_too_many_patterns(b200):
    fn = b200.lib.beagleB200RootLogLikelihoodsNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 6
    dummy = ctypes.c_void_p(16)
    # 8192 blocks of 128 patterns is the limit; one more pattern is refused
    # before anything is touched or queued.
    code = fn(0, None, dummy, 1, 4, 8192 * 128 + 1, 4, dummy, dummy, None, dummy, dummy, dummy)
    assert code == -5
