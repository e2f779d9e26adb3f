"""A thin torch.autograd.Function over a BEAGLE instance: lnL as a function of
the branch lengths, with the pre-order adjoint gradient (updatePrePartials +
calculateEdgeDerivatives) as its backward pass.

Works with any object that has the beagle.h call set of the bindings: an
instance of libbeagle_b200.so through the C ABI, the compiled reference
library, or the oracle.  The forward pass computes the gradient alongside the
likelihood (one traversal pair) and keeps it for backward.
"""
import numpy as np
import torch


class BeagleLnL(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lengths, inst, problem, transposed_pre):
        t = lengths.detach().to(torch.float64).cpu().numpy().copy()
        lnl, grad = problem.evaluate(inst, gradient=True, transposed_pre=transposed_pre,
                                     lengths=t)
        ctx.save_for_backward(torch.as_tensor(np.asarray(grad, dtype=np.float64)))
        return torch.tensor(float(lnl), dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None


def lnl(lengths, inst, problem, transposed_pre=False):
    return BeagleLnL.apply(lengths, inst, problem, transposed_pre)


def central_differences(inst, problem, lengths, branches, h=1e-6, transposed_pre=False):
    """(lnL(t + h e_b) - lnL(t - h e_b)) / 2h for each listed branch b, with a
    relative step h * t_b."""
    out = []
    for b in branches:
        step = h * max(lengths[b], 1e-3)
        tp, tm = lengths.copy(), lengths.copy()
        tp[b] += step
        tm[b] -= step
        lp, _ = problem.evaluate(inst, gradient=False, transposed_pre=transposed_pre, lengths=tp)
        lm, _ = problem.evaluate(inst, gradient=False, transposed_pre=transposed_pre, lengths=tm)
        out.append((lp - lm) / (2 * step))
    return np.array(out)
