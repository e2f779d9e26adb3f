#!/usr/bin/env python
"""Benchmark: lnL + branch-gradient evaluations per second on B200.

One step is one evaluation of the BEAGLE hot path on the 4-state GTR+Gamma4
workload with 128 taxa and 100,000 site patterns (FP32 partials, per-node
rescaling, FP64 P(t) and reductions):

    updateTransitionMatrices (254 branches) -> updatePartials (127 ops)
    -> scale accumulation -> root lnL -> root pre-partials
    -> updatePrePartials (254 ops) -> calculateEdgeDerivatives (254 branches)

through libbeagle_b200.so's C ABI: the post-order walk, scale accumulation and
root lnL as one beagleB200UpdatePartialsWithRootLogLikelihood call, and the
last two as one beagleB200UpdatePrePartialsWithDerivatives call.  ``value``
queues K evaluations on the
instance's stream (ASYNCH instance, inputs resident) and times them with CUDA
events on that stream; ``e2e`` runs K evaluations that each copy new branch
lengths in and read lnL and the gradient back (host round trip per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank evaluates its own tree (weak scaling, no
collective on the data path); rank 0 prints the JSON line with the maximum
device time over ranks.  ``--impl reference`` times the reference's own CPU
implementation (the compiled beagle-lib CPU plugins under oracle/_ref) on the
host cores instead, rank 0 only.
"""
import argparse
import importlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
WORKLOAD = "gtr4_n128_p100k"
METRIC = "lnL+gradient evals/s, mixed-batched vs plain FP64 on B200 at rel lnL err ≤1e-6"

SINGLE, DOUBLE, ASYNCH = 1 << 0, 1 << 1, 1 << 3
SCALERS_LOG = 1 << 10
THREADING_CPP = 1 << 30
PROC_CPU, PROC_GPU = 1 << 15, 1 << 16
FW_CUDA, FW_CPU = 1 << 22, 1 << 27
PRE_MANUAL, PRE_AUTO = 1 << 30, 1 << 31
BATCH_WORKLOAD = "batch256"

# Our kernels launched per evaluation: P(t) 1, post-order 1, scale accumulate 1,
# root lnL 2 (sites + final sum), root pre-partials fill 1, pre-order 1,
# edge derivatives 2 (branches x pattern blocks + final sum); one fewer when
# the fused pre-order + derivative walk runs (walk + final sum), and two fewer
# when the fused post-order + root lnL walk runs (walk + final sum).
LAUNCHES_PER_EVAL = 9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="small case for ncu: mixed path only, no JSON")
    ap.add_argument("--profile-patterns", type=int, default=20000,
                    help="patterns of the --profile case")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[4:]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, r in rows:
            for n, v in zip(names, r[1:5]):
                if v.lower() == "active":
                    reasons.add(n)
        sm = [r[0] for r in rows]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": rows[0][1],
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------- CPU side
def reference_lib():
    pkg = importlib.import_module("beagle-lib_b200")
    path = os.path.join(ROOT, "oracle", "_ref", "libhmsbeagle.so")
    if not os.path.exists(path):
        return None
    return pkg.binding.BeagleLib(path, "beagle")


def cpu_reference_rate(workload, seconds=10.0, sample_patterns=4000, max_evals=50):
    """The reference CPU implementation (compiled beagle-lib, SSE plugin with
    C++ threads on every host core) on a pattern sample of the workload.
    Returns (evals/s of the full workload, info)."""
    pkg = importlib.import_module("beagle-lib_b200")
    lib = reference_lib()
    if lib is None:
        return None, {"unavailable": "oracle/_ref not built"}
    full = pkg.synthetic.CONFIGS[workload]
    sample = min(sample_patterns, full["P"])
    pr = pkg.synthetic.config_problem(workload, P=sample)
    cores = os.cpu_count() or 1
    inst = lib.create(*pr.create_args(),
                      preferenceFlags=DOUBLE | PROC_CPU | SCALERS_LOG | THREADING_CPP,
                      requirementFlags=DOUBLE | FW_CPU)
    inst.setCPUThreadCount(cores)
    pr.load(inst)
    pr.evaluate(inst)
    n, t0 = 0, time.perf_counter()
    while n < max_evals and (time.perf_counter() - t0) < seconds:
        pr.evaluate(inst)
        n += 1
    dt = time.perf_counter() - t0
    rate = n / dt * sample / full["P"]
    info = {"impl": inst.impl_name, "cores": cores, "evals": n, "seconds": dt,
            "sample": f"{sample} of {full['P']} patterns, same tree and model, {n} evals "
                      f"in {dt:.1f}s; evals/s scaled by {sample}/{full['P']}"}
    inst.finalize()
    return rate, info


def run_reference_arm(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    if reference_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    pkg = importlib.import_module("beagle-lib_b200")
    full = pkg.synthetic.CONFIGS[args.workload]
    # warm-up, then K steps; each step a bounded pattern sample of the workload
    sample = min(2000, full["P"])
    lib = reference_lib()
    pr = pkg.synthetic.config_problem(args.workload, P=sample)
    cores = os.cpu_count() or 1
    inst = lib.create(*pr.create_args(),
                      preferenceFlags=DOUBLE | PROC_CPU | SCALERS_LOG | THREADING_CPP,
                      requirementFlags=DOUBLE | FW_CPU)
    inst.setCPUThreadCount(cores)
    pr.load(inst)
    for _ in range(args.warmup):
        pr.evaluate(inst)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pr.evaluate(inst)
    dt = time.perf_counter() - t0
    rate = args.steps / dt * sample / full["P"]
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "implementation": inst.impl_name,
                   "threads": cores},
        "cpu_baseline": {"value": rate, "unit": "evals/s", "cores": cores, "kind": "reference",
                         "sample": f"{sample} of {full['P']} patterns per step, evals/s scaled "
                                   f"by {sample}/{full['P']}"},
        "e2e": {"value": rate, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------- GPU side
def make_instance(lib, pr, precision, device, asynch=True, auto_transpose=False):
    pref = (SINGLE if precision == "single" else DOUBLE) | SCALERS_LOG | PROC_GPU
    pref |= PRE_AUTO if auto_transpose else PRE_MANUAL
    if asynch:
        pref |= ASYNCH
    req = (SINGLE if precision == "single" else DOUBLE) | FW_CUDA
    inst = lib.create(*pr.create_args(), resources=[device], preferenceFlags=pref,
                      requirementFlags=req)
    pr.load(inst)
    return inst


def timed_value(torch, inst, pr, steps, warmup, phases=False, fused=True):
    """Queue `steps` evaluations (ASYNCH) and time them on the instance's stream.
    With phases=True also time every phase of every step.  ``fused``: the
    pre-order walk and the edge derivatives as one
    beagleB200UpdatePrePartialsWithDerivatives call (the library runs its fused
    walk or the two calls' kernels, whichever its autotuner timed faster)."""
    stream = torch.cuda.ExternalStream(inst.cudaStream())
    tr = pr.S > 4
    for _ in range(warmup):
        pr.evaluate(inst, transposed_pre=tr, fused=fused)
        inst.getLogLikelihood()
    ev_marks = []

    def mark(name):
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        ev_marks.append((name, e))

    torch.cuda.synchronize()
    inst.waitForPartials([])
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        pr.evaluate(inst, transposed_pre=tr, mark=mark if phases else None, fused=fused)
    end.record(stream)
    end.synchronize()
    lnl = inst.getLogLikelihood()
    total = start.elapsed_time(end)
    per_phase = {}
    if phases:
        for (n0, e0), (n1, e1) in zip(ev_marks, ev_marks[1:]):
            if n1 == "start":
                continue
            per_phase.setdefault(n1, []).append(e0.elapsed_time(e1))
    return total, lnl, per_phase


def timed_e2e(torch, inst, pr, steps):
    """Steps with new branch lengths copied in from pinned host memory and lnL +
    gradient read back every step (the host round trip a caller sees)."""
    stream = torch.cuda.ExternalStream(inst.cudaStream())
    rng = np.random.default_rng(7)
    lengths = torch.empty(pr.B, dtype=torch.float64).pin_memory()
    host = lengths.numpy()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    inst.waitForPartials([])
    start.record(stream)
    for k in range(steps):
        host[:] = pr.lengths * (1.0 + 1e-3 * rng.standard_normal(pr.B))
        _, sums = pr.evaluate(inst, transposed_pre=pr.S > 4, lengths=host, fused=True)
        inst.getLogLikelihood()          # waits for lnL and the gradient sums
        pr.branch_gradient(sums)
    end.record(stream)
    end.synchronize()
    # bytes per step: the P(t) job table (branch lengths inside) in, lnL + gradient out
    h2d = pr.B * 56
    d2h = 8 + 2 * pr.B * 8
    return start.elapsed_time(end), h2d, d2h


def timed_e2e_graph(torch, inst, pr, steps):
    """As timed_e2e, with the whole step -- transition matrices included --
    replayed from a CUDA graph captured once: per step the new branch lengths
    and the graph go in one beagleB200LaunchGraphWithLengths call, then one
    wait for lnL and the gradient."""
    stream = torch.cuda.ExternalStream(inst.cudaStream())
    graph, grad = pr.capture_step(inst, transposed_pre=pr.S > 4, fused=True)
    rng = np.random.default_rng(7)
    lengths = torch.empty(pr.B, dtype=torch.float64).pin_memory()
    host = lengths.numpy()
    for _ in range(2):
        pr.evaluate_graph_step(inst, graph, grad)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    inst.waitForPartials([])
    start.record(stream)
    for _ in range(steps):
        host[:] = pr.lengths * (1.0 + 1e-3 * rng.standard_normal(pr.B))
        pr.evaluate_graph_step(inst, graph, grad, lengths=host)
        pr.branch_gradient(grad)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def timed_checkpointed(torch, lib, pr, device, steps, ref_lnl, ref_grad):
    """lnL + gradient with subtree checkpointing of the post-order partials
    (beagle-lib_b200/checkpoint.py, the plan with the fewest buffers), captured
    as one CUDA graph and timed as timed_e2e_graph times the full schedule.
    Returns the summary object of the JSON line."""
    pkg = importlib.import_module("beagle-lib_b200")
    plan = pkg.checkpoint.smallest_plan(pr, transposed_pre=pr.S > 4)
    pref = SINGLE | SCALERS_LOG | PROC_GPU | PRE_MANUAL | ASYNCH
    inst = lib.create(*plan.create_args(), resources=[device], preferenceFlags=pref,
                      requirementFlags=SINGLE | FW_CUDA)
    pr.load(inst)
    stream = torch.cuda.ExternalStream(inst.cudaStream())
    graph, gradient = plan.capture(inst)
    idx = np.arange(pr.B, dtype=np.int32)

    def step(t):
        inst.updateTransitionMatrices(0, idx, None, None, t)
        inst.launchGraph(graph)
        return inst.getLogLikelihood()

    lnl = step(pr.lengths)
    g = gradient()
    lnl_err = abs(lnl - ref_lnl) / abs(ref_lnl)
    grad_err = float(np.max(np.abs(g - ref_grad)) / np.max(np.abs(ref_grad)))
    rng = np.random.default_rng(7)
    lengths = torch.empty(pr.B, dtype=torch.float64).pin_memory()
    host = lengths.numpy()
    step(pr.lengths)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    inst.waitForPartials([])
    start.record(stream)
    for _ in range(steps):
        host[:] = pr.lengths * (1.0 + 1e-3 * rng.standard_normal(pr.B))
        step(host)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end)
    inst.finalize()
    per_buffer = pr.P * pr.C * pr.S * 4
    return {"value": steps / (ms / 1000.0), "unit": "evals/s",
            "how": "new lengths in, lnL + gradient out; post-matrix work from a CUDA graph",
            "block": plan.block, "blocks": plan.n_blocks, "calls_per_eval": plan.calls,
            "partials_buffers": plan.pool, "partials_buffers_full": pr.B + pr.N - 1,
            "partials_gb": plan.pool * per_buffer / 1e9,
            "partials_gb_full": (pr.B + pr.N - 1) * per_buffer / 1e9,
            "rel_lnl_vs_full": lnl_err, "grad_err_vs_full": grad_err}


def run_profile_case(args):
    """The workload's tree and model on --profile-patterns patterns (default
    20,000: partials larger than L2, a few hundred MB on the device), mixed
    path only: warm-up then `steps` queued evaluations.  For ncu captures."""
    import torch
    pkg = importlib.import_module("beagle-lib_b200")
    pr = pkg.synthetic.config_problem(args.workload, P=min(args.profile_patterns,
                                                           pkg.synthetic.CONFIGS[
                                                               args.workload]["P"]))
    inst = make_instance(pkg.load(), pr, "single", 0)
    timed_value(torch, inst, pr, args.steps, args.warmup)
    inst.finalize()


def run_b200_arm(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pkg = importlib.import_module("beagle-lib_b200")
    syn = pkg.synthetic
    lib = pkg.load()
    # weak scaling: rank r evaluates its own tree and data (seed offset r)
    base = syn.CONFIGS[args.workload]
    pr = syn.config_problem(args.workload, seed=base["seed"] + 7919 * rank)

    clocks = Clocks(local)
    inst = make_instance(lib, pr, "single", local)
    clocks.start()
    barrier(ws)
    ms_total, lnl, _ = timed_value(torch, inst, pr, args.steps, args.warmup)
    clocks_info = clocks.stop()
    ms_total = max_over_ranks(ms_total, ws)
    ms_step = ms_total / args.steps
    value = ws * args.steps / (ms_total / 1000.0)

    # per-phase device times (separate pass) for the roofline of the top kernel.
    # With the fused walk picked, the "deriv" phase is that one kernel (plus
    # its final sum); otherwise the phases of the two calls are timed apart.
    tuned = inst.tunedVariants()
    fused_walk = tuned["fused"] == 1
    nph = max(5, min(50, args.steps // 4))
    _, _, phases = timed_value(torch, inst, pr, nph, 1, phases=True, fused=fused_walk)
    ph_ms = {k: float(np.mean(v)) for k, v in phases.items()}
    if fused_walk:
        ph_ms["fused"] = ph_ms.pop("deriv")
    alg = pr.algorithmic_bytes(4)
    # API-level algorithmic bytes: each call's operations read each input once
    # and write each output once.  The fused walk does the work of the
    # pre-order and derivative calls and is credited with their bytes; its
    # own compulsory traffic (a sibling pair reads its parent and both
    # post-order rows once) is reported beside them.
    credited = dict(alg, fused=alg["pre"] + alg["deriv"])
    # The fused post-order + root call (4 states, 1/2/4/8 categories, at most
    # 256 ops) also does the scale accumulation and root lnL calls' work.
    # (The phase pass above used the fused calls when the fused walk won.)
    post_root = pr.S == 4 and pr.C in (1, 2, 4, 8) and pr.N - 1 <= 256
    if post_root and fused_walk:
        credited["post"] = alg["post"] + alg["scale"] + alg["root"]
    kern = max(["post", "pre", "deriv", "fused"], key=lambda k: ph_ms.get(k, 0))
    peak, peak_kind = peaks()
    achieved = credited[kern] / (ph_ms[kern] * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(args.workload, {}).get(kern)

    # end-to-end through the C ABI with host round trips
    ms_e2e, h2d, d2h = timed_e2e(torch, inst, pr, max(5, args.steps // 5))
    e2e_steps = max(5, args.steps // 5)
    e2e_value = ws * e2e_steps / (max_over_ranks(ms_e2e, ws) / 1000.0)
    ms_graph = timed_e2e_graph(torch, inst, pr, e2e_steps)
    e2e_graph_value = ws * e2e_steps / (max_over_ranks(ms_graph, ws) / 1000.0)
    _, ref_grad = pr.evaluate(inst, transposed_pre=pr.S > 4)
    ref_lnl = inst.getLogLikelihood()        # ASYNCH: delivers lnL and the gradient
    inst.finalize()
    ckpt = timed_checkpointed(torch, lib, pr, local, e2e_steps, ref_lnl, ref_grad)

    # the plain FP64 path (one instance, same workload) for the mixed/FP64 ratio
    inst64 = make_instance(lib, pr, "double", local)
    k64 = max(5, args.steps // 3)
    ms64, lnl64, _ = timed_value(torch, inst64, pr, k64, min(args.warmup, 3))
    ms64 = max_over_ranks(ms64, ws)
    value64 = ws * k64 / (ms64 / 1000.0)
    inst64.finalize()
    rel_err = abs(lnl - lnl64) / abs(lnl64)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        rate, info = cpu_reference_rate(args.workload)
        if rate is not None:
            cpu = {"value": rate, "unit": "evals/s", "cores": info["cores"],
                   "kind": "reference", "sample": info["sample"] + f"; {info['impl']}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "states": pr.S, "taxa": pr.N,
                       "patterns": pr.P, "categories": pr.C, "branches": pr.B,
                       "precision": "FP32 partials, FP64 P(t), scalers and reductions",
                       "rescaling": "every internal node, post- and pre-order",
                       "l2": "inputs larger than L2 (%.1f GB of partials)" % (
                           pr.n_buffers * pr.P * pr.C * pr.S * 4 / 1e9),
                       "parallelism": f"replicas x{ws}", "seed": int(pr.seed)},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes": credited[kern],
                         "algorithmic": "API-level bytes of the calls the kernel runs "
                                        "(pre-order + derivatives for the fused walk; "
                                        "post-order + scale accumulation + root lnL for "
                                        "the fused post-order walk)",
                         "compulsory_bytes": alg[kern],
                         "ms_per_launch": ph_ms[kern], "phase_ms": ph_ms,
                         "phase_frac": {k: credited[k] / (ph_ms[k] * 1e-3) / 1e9 / peak
                                        for k in ("post", "pre", "deriv", "fused")
                                        if k in ph_ms}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "e2e_graph": {"value": e2e_graph_value, "unit": "evals/s",
                          "how": "same steps, each one graph launch with the new branch "
                                 "lengths (P(t) included) and one wait"},
            "checkpointed": ckpt,
            "plain_fp64": {"value": value64, "unit": "evals/s", "ms_per_step": ms64 / k64,
                           "mixed_over_fp64": value / value64,
                           "mixed_vs_fp64_rel_lnl_err": rel_err},
            "lnl": lnl,
            "gpu_launches": (LAUNCHES_PER_EVAL - (1 if fused_walk else 0)
                             - (2 if post_root else 0)) * args.steps,
            "tuned_variants": tuned,
            "clocks": clocks_info,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_batch_arm(args):
    """--workload batch256: 256 independent trees as the batched multi-instance
    configuration draws them (16-256 taxa, 4 or 20 states, 1/4/8 categories),
    with patterns log-uniform in 100-10,000 instead of 100-50,000 so that the
    FP64 instances (101 GB of partials) fit one GPU.  One step evaluates lnL and
    the full gradient of every tree.  value: tree-evals/s of the mixed path
    through the batched calls (one launch per kernel family and category
    count), captured once as a CUDA graph of the batch and replayed per step
    (batched_calls: the same calls issued every step); per_instance_mixed /
    plain_fp64: the same trees evaluated one instance at a time (each
    instance's own launches) on one shared stream.
    All device-timed with CUDA events on that stream."""
    import torch
    pkg = importlib.import_module("beagle-lib_b200")
    syn = pkg.synthetic
    lib = pkg.load()
    probs = syn.batched_problems(count=256, seed=2000, max_patterns=10000)
    n = len(probs)

    def instances(precision):
        return [make_instance(lib, pr, precision, 0, asynch=True, auto_transpose=pr.S > 4)
                for pr in probs]

    def timed(stream, body, steps, warmup):
        for _ in range(warmup):
            body()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            body()
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end)

    def per_instance(insts):
        for pr, inst in zip(probs, insts):
            pr.evaluate(inst, transposed_pre=False)

    steps = max(3, min(args.steps, 20))
    warmup = max(3, args.warmup)
    insts = instances("single")
    batch = pkg.binding.Batch(lib, insts)
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    state = {}

    def batched():
        state["lnl"], _ = syn.batch_evaluate(batch, probs)

    ms_b = timed(stream, batched, steps, warmup)
    lnl32 = np.array(state["lnl"])
    # the same step with everything after the matrices replayed from a CUDA
    # graph of the batch
    graph, lnl_g, _ = syn.batch_capture(batch, probs)
    ms_g = timed(stream, lambda: syn.batch_evaluate_graph(batch, probs, graph), steps, warmup)
    graph_err = float(np.max(np.abs(np.asarray(lnl_g) - lnl32) / np.abs(lnl32)))
    ms_i = timed(stream, lambda: per_instance(insts), max(2, steps // 2), 1)
    batch.finalize()
    for x in insts:
        x.finalize()
    del insts, batch
    insts = instances("double")
    batch = pkg.binding.Batch(lib, insts)        # only to share one stream
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    ms_64 = timed(stream, lambda: per_instance(insts), max(2, steps // 2), 1)
    lnl64 = np.array([x.getLogLikelihood() for x in insts])
    batch.finalize()
    for x in insts:
        x.finalize()
    value_calls = n * steps / (ms_b / 1000.0)
    value = n * steps / (ms_g / 1000.0)
    v_i = n * max(2, steps // 2) / (ms_i / 1000.0)
    v_64 = n * max(2, steps // 2) / (ms_64 / 1000.0)
    rel_err = float(np.max(np.abs(lnl32 - lnl64) / np.abs(lnl64)))
    line = {
        "metric": "tree lnL+gradient evals/s, 256-tree batch, mixed batched vs per-instance",
        "value": value, "unit": "tree-evals/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": ms_g / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "trees": n,
                   "patterns_total": int(sum(p.P for p in probs)),
                   "states": {"4": sum(p.S == 4 for p in probs),
                              "20": sum(p.S == 20 for p in probs)},
                   "patterns": "log-uniform 100-10,000 (configuration: 100-50,000)"},
        "how": "batched calls captured once as a CUDA graph of the batch; per step new "
               "transition matrices (one batched call), one graph launch, one wait",
        "batched_calls": {"value": value_calls, "unit": "tree-evals/s",
                          "ms_per_step": ms_b / steps,
                          "graph_vs_calls_max_rel_lnl_diff": graph_err},
        "per_instance_mixed": {"value": v_i, "unit": "tree-evals/s"},
        "plain_fp64": {"value": v_64, "unit": "tree-evals/s", "batched_mixed_over_fp64": value / v_64,
                       "mixed_vs_fp64_max_rel_lnl_err": rel_err},
        "gpu_launches": None,
    }
    print(json.dumps(line))


def run_batch_full_arm(args):
    """--workload batch256_p50k: the batched multi-instance configuration at
    its own pattern range (log-uniform 100-50,000; 178 GB of FP32 partials
    with every buffer alive).  Every tree runs a subtree checkpoint plan
    (checkpoint.quick_plan: pooled buffers, per-block recomputation); the
    mixed path runs the 256 plans side by side through batched calls
    (checkpoint.batch_checkpointed_evaluate); plain_fp64 runs the same plans
    one instance at a time.  Device-timed with CUDA events on the shared
    stream."""
    import torch
    pkg = importlib.import_module("beagle-lib_b200")
    syn, ck = pkg.synthetic, pkg.checkpoint
    lib = pkg.load()
    probs = syn.batched_problems(count=256, seed=2000, max_patterns=50000)
    plans = [ck.quick_plan(pr) for pr in probs]
    n = len(probs)

    def bytes_of(pr, bufs, w):
        return bufs * pr.P * pr.C * pr.S * w

    full_gb = sum(bytes_of(pr, pl.full_buffers() - pr.N, 4) for pr, pl in zip(probs, plans)) / 1e9
    pool_gb = sum(bytes_of(pr, pl.pool, 4) for pr, pl in zip(probs, plans)) / 1e9

    def instances(precision):
        pref = (SINGLE if precision == "single" else DOUBLE) | SCALERS_LOG | PROC_GPU | ASYNCH
        req = (SINGLE if precision == "single" else DOUBLE) | FW_CUDA
        out = []
        for pr, pl in zip(probs, plans):
            inst = lib.create(*pl.create_args(), resources=[0],
                              preferenceFlags=pref | (PRE_AUTO if pr.S > 4 else PRE_MANUAL),
                              requirementFlags=req)
            pr.load(inst)
            out.append(inst)
        return out

    def timed(stream, body, steps, warmup):
        for _ in range(warmup):
            body()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            body()
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end)

    steps = max(2, min(args.steps, 5))
    insts = instances("single")
    batch = pkg.binding.Batch(lib, insts)
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    state = {}

    def batched():
        state["lnl"], _ = ck.batch_checkpointed_evaluate(batch, plans)

    ms_b = timed(stream, batched, steps, 2)
    lnl32 = np.array(state["lnl"])
    batch.finalize()
    for x in insts:
        x.finalize()
    del insts, batch
    insts = instances("double")
    batch = pkg.binding.Batch(lib, insts)        # only to share one stream
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    lnl64 = np.zeros(n)

    def per_instance():
        for pl, inst in zip(plans, insts):
            pl.evaluate(inst)

    ms_64 = timed(stream, per_instance, 1, 1)
    for i, inst in enumerate(insts):
        lnl64[i] = inst.getLogLikelihood()       # ASYNCH: the last evaluation's lnL
    batch.finalize()
    for x in insts:
        x.finalize()
    value = n * steps / (ms_b / 1000.0)
    v_64 = n / (ms_64 / 1000.0)
    line = {
        "metric": "tree lnL+gradient evals/s, 256-tree batch at 100-50,000 patterns, "
                  "checkpointed, mixed batched vs FP64 per-instance",
        "value": value, "unit": "tree-evals/s", "n_gpus": 1, "steps": steps, "warmup": 2,
        "ms_per_step": ms_b / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "trees": n,
                   "patterns_total": int(sum(p.P for p in probs)),
                   "states": {"4": sum(p.S == 4 for p in probs),
                              "20": sum(p.S == 20 for p in probs)},
                   "patterns": "log-uniform 100-50,000",
                   "checkpointing": "quick_plan per tree (blocks of about sqrt(N/2) internal nodes)",
                   "fp32_partials_gb_full": full_gb, "fp32_partials_gb_pooled": pool_gb},
        "plain_fp64": {"value": v_64, "unit": "tree-evals/s",
                       "how": "the same plans, one instance at a time, FP64",
                       "batched_mixed_over_fp64": value / v_64,
                       "mixed_vs_fp64_max_rel_lnl_err":
                           float(np.max(np.abs(lnl32 - lnl64) / np.abs(lnl64)))},
        "gpu_launches": None,
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.profile:
        run_profile_case(args)
    elif args.workload == BATCH_WORKLOAD:
        run_batch_arm(args)
    elif args.workload == BATCH_WORKLOAD + "_p50k":
        run_batch_full_arm(args)
    else:
        run_b200_arm(args)


if __name__ == "__main__":
    main()
