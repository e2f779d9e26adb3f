"""Pattern sharding of one lnL + gradient evaluation over several ranks.

Patterns are independent given the tree and the model, so a tree's patterns
can be split into contiguous ranges, one per rank (one process per GPU).
Each rank holds every buffer for its own range only, and runs the whole call
sequence on it. The only exchange is one sum over ranks of 1 + B doubles: the
lnL and the branch gradient. The per-rank sums are pattern-weighted sums over
disjoint pattern sets, so they add up to the unsharded evaluation.

``torch.distributed`` carries that all-reduce: NCCL between GPUs, gloo in the
CPU tests. A tree too small to fill one GPU is better evaluated whole, with
whole trees spread over ranks (``bench.py --gpus N`` does that: weak scaling,
no collective on the data path).
"""

import copy

import numpy as np


def shard_bounds(P, world):
    """Contiguous pattern ranges [lo, hi) of `world` ranks, sizes differing by
    at most one."""
    edges = np.linspace(0, P, world + 1).round().astype(int)
    return [(int(edges[r]), int(edges[r + 1])) for r in range(world)]


def pattern_shard(problem, rank, world):
    """The Problem restricted to rank `rank`'s patterns (same tree, model and
    branch lengths)."""
    lo, hi = shard_bounds(problem.P, world)[rank]
    sh = copy.copy(problem)
    sh.__dict__ = dict(problem.__dict__)
    for cached in ("_post_ops", "_pre_ops"):
        sh.__dict__.pop(cached, None)
    sh.P = hi - lo
    sh.patw = problem.patw[lo:hi].copy()
    sh.tip_states = problem.tip_states[:, lo:hi].copy()
    S = problem.S
    sh.tip_partials = {t: np.asarray(v).reshape(problem.P, S)[lo:hi].reshape(-1).copy()
                       for t, v in problem.tip_partials.items()}
    return sh


def sharded_evaluate(shard, inst, group=None, fused=False, transposed_pre=False, device=None):
    """Evaluate this rank's shard on `inst` and sum lnL and the gradient over
    the ranks of `group` (torch.distributed all-reduce).  Returns (lnL,
    gradient[B]) of the whole tree on every rank."""
    import torch
    import torch.distributed as dist

    lnl, grad = shard.evaluate(inst, transposed_pre=transposed_pre, fused=fused)
    if fused:
        grad = shard.branch_gradient(grad)
    t = torch.tensor(np.concatenate([[lnl], np.asarray(grad)]), dtype=torch.float64,
                     device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    return float(t[0]), t[1:]
