"""Generate tests/golden/golden.npz by running the compiled reference BEAGLE
CPU library (oracle/_ref, built by oracle/Makefile) on seeded workloads.

    python tests/golden/make_golden.py

Each case is a seeded Problem from beagle-lib_b200/synthetic.py; the fixture
stores the reference's outputs (root lnL, site lnL, per-branch gradient sums
and, for one branch, per-site derivatives) together with the generator
parameters, so the inputs are rebuilt from the seed when the fixture is read.
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
pkg = importlib.import_module("beagle-lib_b200")
syn = pkg.synthetic

# (case name, make_problem kwargs, scalers)
CASES = [
    ("gtr4_n16_p1000", dict(S=4, N=16, P=1000, C=4, seed=1000, mean_length=0.1,
                            ambiguous=0.05, rescale=False), "log"),
    ("gtr4_n32_p3000_rescaled", dict(S=4, N=32, P=3000, C=4, seed=1001, mean_length=0.05,
                                     rescale=True), "log"),
    ("gtr4_n20_p700_raw", dict(S=4, N=20, P=700, C=2, seed=1101, rescale=True), "raw"),
    ("aa20_n16_p1000", dict(S=20, N=16, P=1000, C=4, seed=1002, rescale=True), "log"),
    ("codon61_n8_p600", dict(S=61, N=8, P=600, C=4, seed=1003, rescale=True), "log"),
    ("s5_n10_p333_c3", dict(S=5, N=10, P=333, C=3, seed=1004, rescale=True), "log"),
]

DOUBLE, LOG, RAW, CPU = 1 << 1, 1 << 10, 1 << 9, 1 << 15


def main():
    lib = pkg.binding.BeagleLib(os.path.join(ROOT, "oracle", "_ref", "libhmsbeagle.so"), "beagle")
    out = {}
    meta = {}
    for name, kw, sc in CASES:
        pr = syn.make_problem(name=name, **kw)
        flags = DOUBLE | CPU | (LOG if sc == "log" else RAW)
        inst = lib.create(*pr.create_args(), preferenceFlags=flags, requirementFlags=DOUBLE)
        pr.load(inst)
        lnl, grad = pr.evaluate(inst)
        site = inst.getSiteLogLikelihoods()
        nonroot = np.arange(pr.B, dtype=np.int32)
        d, _, sq = inst.calculateEdgeDerivatives(nonroot, nonroot + pr.pre(0),
                                                 np.full(pr.B, pr.B, dtype=np.int32), [0])
        out[name + "/lnl"] = np.array([lnl])
        out[name + "/grad"] = grad
        out[name + "/site_lnl"] = site
        out[name + "/site_d_branch0"] = d[0]
        out[name + "/sumsq"] = sq
        meta[name] = dict(kw=kw, scalers=sc, impl=inst.impl_name)
        inst.finalize()
        print(name, inst.impl_name, lnl)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)


if __name__ == "__main__":
    main()
