"""Child process of test_plugin.py: drives the stock BEAGLE dispatcher
(oracle/_ref/libhmsbeagle.so, compiled from the reference sources) with
libhmsbeagle-cuda.so.40.0.0 from this repository on its library path, the way
an application linked against libhmsbeagle would run.

    LD_LIBRARY_PATH=<repo>/beagle-lib_b200/lib python tests/plugin_driver.py MODE [ARGS_JSON]

MODE "resources": print the dispatcher's resource list and whether the
plugin was loaded.  MODE "evaluate": build the Problem described by ARGS_JSON,
create an instance through the dispatcher with the CUDA framework required,
run one lnL + gradient evaluation and print the results.  Output: one JSON
line on stdout.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import importlib  # noqa: E402

from helpers import gpu_flags  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libhmsbeagle.so")
PLUGIN = "libhmsbeagle-cuda.so.40.0.0"


def plugin_loaded():
    with open("/proc/self/maps") as f:
        return any(PLUGIN in line for line in f)


def main():
    mode = sys.argv[1]
    args = json.loads(sys.argv[2]) if len(sys.argv) > 2 else {}
    pkg = importlib.import_module("beagle-lib_b200")
    lib = pkg.binding.BeagleLib(REF_LIB, "beagle")
    res = lib.resources()
    out = {"resources": res, "plugin_loaded": plugin_loaded()}
    if mode == "evaluate":
        pr = pkg.synthetic.make_problem(**args["problem"])
        pref, req = gpu_flags(args["precision"], auto_transpose=args.get("auto", False))
        inst = lib.create(*pr.create_args(), preferenceFlags=pref, requirementFlags=req)
        pr.load(inst)
        transposed = pr.S > 4 and not args.get("auto", False)
        lnl, grad = pr.evaluate(inst, transposed_pre=transposed)
        out.update(impl=inst.impl_name, resource=inst.info.resourceNumber, flags=inst.flags,
                   lnl=lnl, grad=[float(g) for g in grad],
                   site=[float(v) for v in inst.getSiteLogLikelihoods()])
        inst.finalize()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
