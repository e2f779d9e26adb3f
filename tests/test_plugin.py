"""The drop-in boundary: libhmsbeagle-cuda.so.40.0.0 loaded by the stock BEAGLE
dispatcher (libhmsbeagle.so compiled from the reference sources by
oracle/Makefile), driven through beagle.h calls in a child process
(tests/plugin_driver.py) with the plugin's folder on LD_LIBRARY_PATH.

CPU: the dispatcher loads the plugin and, with no usable device, still offers
its CPU resources.  GPU: an instance created with the CUDA framework required
lands on this library and matches the oracle."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import TOL, grad_err, rel, run_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "beagle-lib_b200", "lib")
PLUGIN = os.path.join(LIBDIR, "libhmsbeagle-cuda.so.40.0.0")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libhmsbeagle.so")
FRAMEWORK_CUDA = 1 << 22


def _need():
    if not os.path.exists(PLUGIN):
        pytest.skip("plugin not built (needs the BEAGLE headers at build time)")
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built (make -C oracle)")


def _drive(mode, args=None):
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = LIBDIR + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    cmd = [sys.executable, os.path.join(ROOT, "tests", "plugin_driver.py"), mode]
    if args is not None:
        cmd.append(json.dumps(args))
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_plugin_exports_plugin_init():
    _need()
    import ctypes
    lib = ctypes.CDLL(PLUGIN)
    assert hasattr(lib, "plugin_init")


def test_dispatcher_loads_plugin():
    _need()
    out = _drive("resources")
    assert out["plugin_loaded"]
    names = [r[0] for r in out["resources"]]
    assert any(n.startswith("CPU") for n in names), names
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        assert any(sf & FRAMEWORK_CUDA for _, sf, _ in out["resources"]), out["resources"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("S", [4, 20])
def test_dispatcher_runs_b200(syn, oracle, precision, S):
    _need()
    spec = dict(S=S, N=12, P=777, C=4, seed=300 + S, rescale=True)
    out = _drive("evaluate", {"problem": spec, "precision": precision})
    assert out["impl"].startswith("B200-sm100a"), out["impl"]
    assert out["flags"] & FRAMEWORK_CUDA
    pr = syn.make_problem(**spec)
    oi, lo, go = run_oracle(oracle, pr)
    tol = TOL[precision]
    assert rel(out["lnl"], lo) <= tol["lnl"], (out["lnl"], lo)
    assert grad_err(out["grad"], go) <= tol["grad"]
    site_o = oi.getSiteLogLikelihoods()
    assert np.max(np.abs(np.array(out["site"]) - site_o) / np.abs(site_o)) <= 100 * tol["lnl"]
