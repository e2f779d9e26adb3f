"""Pattern-sharded evaluation on the product library: two ranks (spawned
processes, gloo all-reduce on the host), each with a libbeagle_b200.so
instance on cuda:0 for its contiguous pattern range, call
shard.sharded_evaluate.  The summed lnL and gradient must equal the
unsharded evaluation on the GPU: 1e-12 on the FP64 path, and the mixed
path's tolerance on FP32.

The ranks share one GPU only as two independent processes: no kernel of
one waits on the other, and the one exchange is a host all-reduce after
both have finished their evaluation."""
import importlib
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import TOL, gpu_flags, grad_err, rel

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = {
    "gtr4": dict(S=4, N=24, P=20001, C=4, seed=71, rescale=True),
    "aa20": dict(S=20, N=12, P=3001, C=4, seed=72, rescale=True),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out, case, precision):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]
    import datetime
    import torch.distributed as dist
    from helpers import gpu_flags as flags
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    pkg = importlib.import_module("beagle-lib_b200")
    pr = pkg.synthetic.make_problem(**CASES[case])
    sh = pkg.shard.pattern_shard(pr, rank, world)
    pref, req = flags(precision)
    inst = pkg.load().create(*sh.create_args(), resources=[0], preferenceFlags=pref,
                             requirementFlags=req)
    sh.load(inst)
    lnl, grad = pkg.shard.sharded_evaluate(sh, inst, transposed_pre=sh.S > 4)
    inst.finalize()
    np.save(os.path.join(out, f"r{rank}.npy"), np.concatenate([[lnl], grad]))
    dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_sharded_product_library_matches_whole_tree(b200, syn, case, precision):
    world = 2
    out = tempfile.mkdtemp()
    mp.start_processes(_rank, args=(world, _free_port(), out, case, precision), nprocs=world,
                       join=True, start_method="spawn")
    pr = syn.make_problem(**CASES[case])
    pref, req = gpu_flags(precision)
    inst = b200.create(*pr.create_args(), resources=[0], preferenceFlags=pref,
                       requirementFlags=req)
    pr.load(inst)
    l0, g0 = pr.evaluate(inst, transposed_pre=pr.S > 4)
    inst.finalize()
    tol = dict(lnl=1e-12, grad=1e-12) if precision == "double" else TOL["single"]
    for r in range(world):
        v = np.load(os.path.join(out, f"r{r}.npy"))
        assert rel(v[0], l0) <= tol["lnl"], (r, v[0], l0)
        assert grad_err(v[1:], g0) <= tol["grad"], (r, grad_err(v[1:], g0))
