"""Pattern-sharded evaluation (beagle-lib_b200/shard.py) on two gloo ranks
(CPU, the oracle as each rank's instance): the all-reduced lnL and gradient
equal the unsharded evaluation, with rescaling, ambiguous tips and uneven
shards."""
import importlib
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import SCALERS_LOG, grad_err, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
    import datetime
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    pkg = importlib.import_module("beagle-lib_b200")
    pr = pkg.synthetic.make_problem(S=4, N=14, P=301, C=4, seed=5, rescale=True, ambiguous=0.03)
    sh = pkg.shard.pattern_shard(pr, rank, world)
    inst = oracle.OracleInstance(*sh.create_args(), flags=SCALERS_LOG)
    sh.load(inst)
    lnl, grad = pkg.shard.sharded_evaluate(sh, inst)
    np.save(os.path.join(out, f"r{rank}.npy"), np.concatenate([[lnl], grad]))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_evaluation_matches_whole_tree(pkg, syn, oracle, world):
    out = tempfile.mkdtemp()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    pr = syn.make_problem(S=4, N=14, P=301, C=4, seed=5, rescale=True, ambiguous=0.03)
    inst = oracle.OracleInstance(*pr.create_args(), flags=SCALERS_LOG)
    pr.load(inst)
    l0, g0 = pr.evaluate(inst)
    for r in range(world):
        v = np.load(os.path.join(out, f"r{r}.npy"))
        assert rel(v[0], l0) <= 1e-12, (r, v[0], l0)
        assert grad_err(v[1:], g0) <= 1e-12, r


def test_shard_bounds_cover_patterns(pkg):
    for P, world in [(10, 3), (7, 7), (100000, 8)]:
        b = pkg.shard.shard_bounds(P, world)
        assert b[0][0] == 0 and b[-1][1] == P
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        sizes = [hi - lo for lo, hi in b]
        assert max(sizes) - min(sizes) <= 1
