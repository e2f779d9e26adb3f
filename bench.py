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
device time over ranks.  ``--shard`` splits one tree by patterns over the
ranks instead, with one all-reduce of lnL and the gradient per evaluation
(strong scaling).  ``--impl reference`` times the reference's own CPU
implementation (the compiled beagle-lib CPU plugins under oracle/_ref) on the
host cores instead, rank 0 only, on the whole workload.

At N = 1 the line also carries, under ``workloads``, the 61-state codon and
20-state amino-acid configurations (mixed and plain FP64 paths, one instance
each and a batch of 8 trees, with lnL and per-branch gradient errors against
the reference CPU implementation on the same inputs) and the 256-tree batch
(batched mixed against per-instance FP64); ``target_61_state`` summarises
the codon configuration against the bars of the benchmark metric.
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
    ap.add_argument("--shard", action="store_true",
                    help="one tree split by patterns over the ranks (strong scaling)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 20-state, 61-state and batch256 sub-records")
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


def workload_config(pr, ws):
    """The ``config`` object of both arms' JSON lines (the same dict, so that
    the two lines name the same workload)."""
    return {"workload": pr.name, "states": pr.S, "taxa": pr.N, "patterns": pr.P,
            "categories": pr.C, "branches": pr.B,
            "rescaling": "every internal node, post- and pre-order" if pr.rescale else "none",
            "l2": "inputs larger than L2 (%.1f GB of FP32 partials)" % (
                pr.n_buffers * pr.P * pr.C * pr.S * 4 / 1e9),
            "parallelism": f"replicas x{ws}", "seed": int(pr.seed)}


def reference_instance(pr):
    """The reference CPU implementation (compiled beagle-lib, FP64, SSE plugin
    with C++ threads on every host core) loaded with a workload."""
    lib = reference_lib()
    cores = os.cpu_count() or 1
    inst = lib.create(*pr.create_args(),
                      preferenceFlags=DOUBLE | PROC_CPU | SCALERS_LOG | THREADING_CPP,
                      requirementFlags=DOUBLE | FW_CPU)
    inst.setCPUThreadCount(cores)
    pr.load(inst)
    return inst, cores


def reference_run(pr, evals=1):
    """The reference CPU implementation on the whole workload: one evaluation
    whose lnL and gradient are the FP64 reference values for the error
    figures, then ``evals`` timed ones.  Returns (lnL, gradient, cpu_baseline
    object)."""
    inst, cores = reference_instance(pr)
    lnl, g = pr.evaluate(inst)
    t0 = time.perf_counter()
    for _ in range(evals):
        pr.evaluate(inst)
    dt = time.perf_counter() - t0
    base = {"value": evals / dt, "unit": "evals/s", "cores": cores, "kind": "reference",
            "sample": f"the whole workload ({pr.P} patterns), {evals} evals in {dt:.2f}s "
                      f"after one untimed; {inst.impl_name}"}
    inst.finalize()
    return lnl, g, base


def errors_vs(lnl, g, ref_lnl, ref_g):
    """lnL and per-branch gradient errors against reference values
    (synthetic.gradient_errors)."""
    pkg = importlib.import_module("beagle-lib_b200")
    e = pkg.synthetic.gradient_errors(g, ref_g)
    return {"rel_lnl": abs(lnl - ref_lnl) / abs(ref_lnl), "grad_branch": e["branch"],
            "grad_branch_unfloored": e["branch_unfloored"], "grad_max_norm": e["max_norm"]}


def run_reference_arm(args):
    """The reference's own CPU implementation on the whole workload (no
    pattern sample): W untimed evaluations, then K timed ones.  When K + W
    evaluations of the whole workload would take more than about two and a
    half minutes, every step runs a contiguous pattern sample sized to fit,
    and the rate is scaled to the whole workload (``sample`` says so)."""
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    if reference_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    pkg = importlib.import_module("beagle-lib_b200")
    full = pkg.synthetic.config_problem(args.workload)
    inst, cores = reference_instance(full)
    t0 = time.perf_counter()
    pr, sample = full, full.P
    pr.evaluate(inst)
    est = time.perf_counter() - t0
    budget = 150.0
    if (args.steps + args.warmup) * est > budget:
        sample = max(100, int(full.P * budget / ((args.steps + args.warmup) * est)))
        inst.finalize()
        pr = pkg.synthetic.config_problem(args.workload, P=sample)
        inst, cores = reference_instance(pr)
        pr.evaluate(inst)
    for _ in range(max(0, args.warmup - 1)):
        pr.evaluate(inst)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pr.evaluate(inst)
    dt = time.perf_counter() - t0
    rate = args.steps / dt * sample / full.P
    how = (f"the whole workload ({full.P} patterns) every step" if sample == full.P else
           f"{sample} of {full.P} patterns per step, evals/s scaled by {sample}/{full.P}")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / rate, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(full, ws),
        "implementation": inst.impl_name, "threads": cores,
        "precision": "FP64 throughout (the reference CPU implementation)",
        "cpu_baseline": {"value": rate, "unit": "evals/s", "cores": cores, "kind": "reference",
                         "sample": how},
        "e2e": {"value": rate, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    inst.finalize()
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
    graph, gradient = plan.capture(inst, fused=True)
    idx = np.arange(pr.B, dtype=np.int32)

    def step(t):
        inst.updateTransitionMatrices(0, idx, None, None, t)
        inst.launchGraph(graph)
        return inst.getLogLikelihood()

    lnl = step(pr.lengths)
    g = gradient()
    err = errors_vs(lnl, g, ref_lnl, ref_grad)
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
            "vs_full_schedule": err}


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


def evaluate_once(inst, pr, fused=True):
    """One evaluation's lnL and branch-order gradient (ASYNCH instance: the
    wait delivers both)."""
    _, sums = pr.evaluate(inst, transposed_pre=pr.S > 4, fused=fused)
    lnl = inst.getLogLikelihood()
    return lnl, (pr.branch_gradient(sums) if fused else sums)


def roofline_of(pr, ph_ms, fused_walk, peak, peak_kind, traffic_table):
    """Roofline of the dominant kernel of one evaluation from per-phase device
    times: algorithmic bytes (synthetic.Problem.algorithmic_bytes, FP32) over
    the phase's time.  The fused walks are credited with the API-level bytes
    of the calls they run."""
    alg = pr.algorithmic_bytes(4)
    credited = dict(alg, fused=alg["pre"] + alg["deriv"])
    post_root = pr.S == 4 and pr.C in (1, 2, 4, 8) and pr.N - 1 <= 256
    if post_root and fused_walk:
        credited["post"] = alg["post"] + alg["scale"] + alg["root"]
    kern = max(["post", "pre", "deriv", "fused"], key=lambda k: ph_ms.get(k, 0))
    achieved = credited[kern] / (ph_ms[kern] * 1e-3) / 1e9
    traffic = (traffic_table or {}).get(pr.name, {}).get(kern)
    return {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "algorithmic_bytes": credited[kern],
            "algorithmic": "API-level bytes of the calls the kernel runs "
                           "(pre-order + derivatives for the fused walk; "
                           "post-order + scale accumulation + root lnL for "
                           "the fused post-order walk)",
            "compulsory_bytes": alg[kern], "ms_per_launch": ph_ms[kern], "phase_ms": ph_ms,
            "phase_frac": {k: credited[k] / (ph_ms[k] * 1e-3) / 1e9 / peak
                           for k in ("post", "pre", "deriv", "fused") if k in ph_ms}}


def phase_times(torch, inst, pr, steps, fused_walk):
    _, _, phases = timed_value(torch, inst, pr, steps, 1, phases=True, fused=fused_walk)
    ph_ms = {k: float(np.mean(v)) for k, v in phases.items()}
    if fused_walk:
        ph_ms["fused"] = ph_ms.pop("deriv")
    return ph_ms


def traffic_table():
    tf = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.json")
    return json.load(open(tf)) if os.path.exists(tf) else {}


def timed_batch(torch, stream, body, steps, warmup):
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


def batched_trees(torch, lib, probs, steps, warmup, device=0, reference_members=()):
    """The trees of ``probs`` evaluated together through the batched calls
    (one launch per kernel family and (states, categories) group), captured
    once as a CUDA graph of the batch and replayed per step (new transition
    matrices, one graph launch, one wait), against the plain FP64 path one
    instance at a time on one shared stream.  Errors: every tree's mixed lnL
    and per-branch gradient against its FP64 evaluation, and for the members
    listed in ``reference_members`` against the reference CPU
    implementation.  All device-timed with CUDA events on the shared stream."""
    pkg = importlib.import_module("beagle-lib_b200")
    syn = pkg.synthetic
    n = len(probs)

    def instances(precision):
        return [make_instance(lib, pr, precision, device, asynch=True, auto_transpose=pr.S > 4)
                for pr in probs]

    def per_instance(insts, out=None):
        for i, (pr, inst) in enumerate(zip(probs, insts)):
            r = pr.evaluate(inst, transposed_pre=False)
            if out is not None:
                out[i] = r[1]

    insts = instances("single")
    batch = pkg.binding.Batch(lib, insts)
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    state = {}

    def batched(fused):
        state["lnl"], state["grad"] = syn.batch_evaluate(batch, probs, fused=fused)

    ms_u = timed_batch(torch, stream, lambda: batched(False), steps, warmup)
    ms_b = timed_batch(torch, stream, lambda: batched(True), steps, warmup)
    # the whole step (matrices included) as one graph of the batch, launched
    # with each step's new branch lengths
    graph, lnl_g, grad_g = syn.batch_capture_step(batch, probs, fused=True)
    rng = np.random.default_rng(11)
    steps_t = [[p.lengths * (1.0 + 1e-3 * rng.standard_normal(p.B)) for p in probs]
               for _ in range(2)]
    cnt = {"k": 0}

    def graph_step():
        cnt["k"] += 1
        syn.batch_evaluate_graph_step(batch, probs, graph, steps_t[cnt["k"] % 2])

    ms_g = timed_batch(torch, stream, graph_step, steps, warmup)
    syn.batch_evaluate_graph_step(batch, probs, graph)            # the problems' own lengths
    lnl32 = np.array(lnl_g, dtype=np.float64)
    grad32 = [np.array(g, dtype=np.float64)
              for g in syn.batch_gradients(probs, grad_g, fused=True)]
    graph_err = float(np.max(np.abs(lnl32 - np.asarray(state["lnl"])) / np.abs(lnl32)))
    k_i = max(2, steps // 2)
    ms_i = timed_batch(torch, stream, lambda: per_instance(insts), k_i, 1)
    batch.finalize()
    for x in insts:
        x.finalize()
    del insts, batch
    insts = instances("double")
    batch = pkg.binding.Batch(lib, insts)        # only to share one stream
    stream = torch.cuda.ExternalStream(insts[0].cudaStream())
    grad64 = [None] * n
    ms_64 = timed_batch(torch, stream, lambda: per_instance(insts, grad64), k_i, 1)
    lnl64 = np.array([x.getLogLikelihood() for x in insts])
    grad64 = [np.array(g, dtype=np.float64) for g in grad64]
    batch.finalize()
    for x in insts:
        x.finalize()
    value = n * steps / (ms_g / 1000.0)
    v_64 = n * k_i / (ms_64 / 1000.0)
    e32 = [errors_vs(lnl32[i], grad32[i], lnl64[i], grad64[i]) for i in range(n)]
    rec = {"value": value, "unit": "tree-evals/s", "trees": n, "steps": steps,
           "ms_per_step": ms_g / steps,
           "how": "the whole batched step (matrices, post-order walks, scaling, root lnL, "
                  "fused pre-order walks with derivatives) captured once as a CUDA graph of "
                  "the batch; per step one launch with every tree's new branch lengths, one "
                  "wait",
           "batched_calls": {"value": n * steps / (ms_b / 1000.0), "unit": "tree-evals/s",
                             "how": "the same batched calls issued every step",
                             "graph_vs_calls_max_rel_lnl_diff": graph_err},
           "batched_calls_unfused": {"value": n * steps / (ms_u / 1000.0),
                                     "unit": "tree-evals/s",
                                     "how": "pre-order walk and derivatives as two batched "
                                            "calls"},
           "per_instance_mixed": {"value": n * k_i / (ms_i / 1000.0), "unit": "tree-evals/s"},
           "plain_fp64": {"value": v_64, "unit": "tree-evals/s",
                          "how": "one instance per tree, each its own launches, one stream"},
           "batched_mixed_over_fp64": value / v_64,
           "mixed_vs_fp64": {"max_rel_lnl": max(e["rel_lnl"] for e in e32),
                             "max_grad_branch": max(e["grad_branch"] for e in e32),
                             "max_grad_max_norm": max(e["grad_max_norm"] for e in e32)}}
    if reference_members and reference_lib() is not None:
        worst = {"mixed": {}, "fp64": {}}
        for i in reference_members:
            rl, rg, _ = reference_run(probs[i], evals=0)
            for key, (l, g) in (("mixed", (lnl32[i], grad32[i])),
                                ("fp64", (lnl64[i], grad64[i]))):
                e = errors_vs(l, g, rl, rg)
                for k, v in e.items():
                    worst[key][k] = max(worst[key].get(k, 0.0), v)
        rec["vs_reference"] = dict(worst, members=[int(i) for i in reference_members],
                                   how="reference CPU implementation (FP64) on these members")
    return rec


def workload_record(torch, lib, name, args, device):
    """lnL + gradient of one benchmark configuration on the mixed path and
    the plain FP64 path, one instance each, with errors against the reference
    CPU implementation on the same inputs; then a batch of 8 trees drawn as
    the configuration draws them, batched mixed against FP64 per instance."""
    pkg = importlib.import_module("beagle-lib_b200")
    syn = pkg.synthetic
    pr = syn.config_problem(name)
    steps = max(5, min(args.steps, 30))
    warm = max(3, min(args.warmup, 5))
    inst = make_instance(lib, pr, "single", device)
    ms, _, _ = timed_value(torch, inst, pr, steps, warm)
    mixed = steps / (ms / 1000.0)
    tuned = inst.tunedVariants()
    # the fused pre-order + derivative walk (S = 4 kernels, or the tensor-core
    # ones for S > 4) when the autotuner picked any of its forms
    fused_walk = tuned.get("fused", 0) > 0
    ph_ms = phase_times(torch, inst, pr, 5, fused_walk)
    peak, peak_kind = peaks()
    roof = roofline_of(pr, ph_ms, fused_walk, peak, peak_kind, traffic_table())
    k_e2e = max(10, steps // 2)
    ms_e, h2d, d2h = timed_e2e(torch, inst, pr, k_e2e)
    ms_eg = timed_e2e_graph(torch, inst, pr, k_e2e)
    lnl32, g32 = evaluate_once(inst, pr)
    inst.finalize()
    inst64 = make_instance(lib, pr, "double", device)
    ms64, _, _ = timed_value(torch, inst64, pr, steps, min(warm, 3))
    fp64 = steps / (ms64 / 1000.0)
    ms64_e, _, _ = timed_e2e(torch, inst64, pr, k_e2e)
    lnl64, g64 = evaluate_once(inst64, pr)
    inst64.finalize()
    rec = {"workload": name, "config": workload_config(pr, 1),
           "mixed": {"value": mixed, "unit": "evals/s", "ms_per_step": ms / steps,
                     "how": f"{steps} evaluations queued on one ASYNCH instance"},
           "e2e": {"value": k_e2e / (ms_eg / 1000.0), "unit": "evals/s",
                   "h2d_bytes_per_step": pr.B * 8, "d2h_bytes_per_step": d2h,
                   "how": "new lengths in, the whole-step graph, lnL + gradient out"},
           "e2e_calls": {"value": k_e2e / (ms_e / 1000.0), "unit": "evals/s",
                         "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "plain_fp64": {"value": fp64, "unit": "evals/s", "ms_per_step": ms64 / steps,
                          "e2e": {"value": k_e2e / (ms64_e / 1000.0), "unit": "evals/s"}},
           "mixed_over_fp64": mixed / fp64,
           "e2e_calls_mixed_over_fp64": (k_e2e / ms_e) / (k_e2e / ms64_e),
           "mixed_vs_fp64": errors_vs(lnl32, g32, lnl64, g64),
           "roofline": roof, "tuned_variants": tuned}
    if reference_lib() is not None:
        rl, rg, base = reference_run(pr, evals=1)
        rec["vs_reference"] = {"mixed": errors_vs(lnl32, g32, rl, rg),
                               "fp64": errors_vs(lnl64, g64, rl, rg),
                               "reference_lnl": rl}
        rec["cpu_baseline"] = base
    base = syn.CONFIGS[name]
    trees = [syn.config_problem(name, seed=base["seed"] + 100 + k) for k in range(8)]
    rec["batched_x8"] = batched_trees(torch, lib, trees, steps, warm, device,
                                      reference_members=(0,))
    return rec


def batch256_record(torch, lib, args, device=0):
    """The batched multi-instance configuration: 256 independent trees
    (16-256 taxa, 4 or 20 states, 1/4/8 categories) with patterns log-uniform
    in 100-10,000 instead of 100-50,000, so that the FP64 instances (101 GB
    of partials) fit one GPU with every buffer alive.  One step evaluates lnL
    and the full gradient of every tree."""
    pkg = importlib.import_module("beagle-lib_b200")
    probs = pkg.synthetic.batched_problems(count=256, seed=2000, max_patterns=10000)
    steps = max(3, min(args.steps, 20))
    warm = max(3, args.warmup)
    s4 = [i for i, p in enumerate(probs) if p.S == 4][:3]
    s20 = [i for i, p in enumerate(probs) if p.S == 20][:3]
    rec = batched_trees(torch, lib, probs, steps, warm, device, reference_members=s4 + s20)
    rec["config"] = {"workload": BATCH_WORKLOAD, "trees": len(probs),
                     "patterns_total": int(sum(p.P for p in probs)),
                     "states": {"4": sum(p.S == 4 for p in probs),
                                "20": sum(p.S == 20 for p in probs)},
                     "patterns": "log-uniform 100-10,000 (configuration: 100-50,000; "
                                 "--workload batch256_p50k runs that range checkpointed)"}
    return rec


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
    fused_walk = tuned["fused"] > 0          # any fused-walk form (variants 1-3)
    nph = max(5, min(50, args.steps // 4))
    ph_ms = phase_times(torch, inst, pr, nph, fused_walk)
    peak, peak_kind = peaks()
    roof = roofline_of(pr, ph_ms, fused_walk, peak, peak_kind, traffic_table())
    post_root = pr.S == 4 and pr.C in (1, 2, 4, 8) and pr.N - 1 <= 256

    # end to end through the C ABI with host round trips: the whole-step graph
    # call (new lengths in, one launch, one wait for lnL and the gradient),
    # and the per-call sequence
    e2e_steps = max(10, args.steps // 2)
    ms_calls, h2d_calls, d2h = timed_e2e(torch, inst, pr, e2e_steps)
    e2e_calls_value = ws * e2e_steps / (max_over_ranks(ms_calls, ws) / 1000.0)
    ms_graph = timed_e2e_graph(torch, inst, pr, e2e_steps)
    e2e_value = ws * e2e_steps / (max_over_ranks(ms_graph, ws) / 1000.0)
    h2d = pr.B * 8        # the step's branch lengths
    ref_lnl, ref_grad = evaluate_once(inst, pr)
    inst.finalize()
    ckpt = timed_checkpointed(torch, lib, pr, local, e2e_steps, ref_lnl, ref_grad)

    # the plain FP64 path (one instance, same workload) for the mixed/FP64 ratio
    inst64 = make_instance(lib, pr, "double", local)
    k64 = max(5, args.steps // 3)
    ms64, _, _ = timed_value(torch, inst64, pr, k64, min(args.warmup, 3))
    ms64 = max_over_ranks(ms64, ws)
    value64 = ws * k64 / (ms64 / 1000.0)
    lnl64, g64 = evaluate_once(inst64, pr)
    inst64.finalize()

    cpu = errors = None
    extra = {}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and reference_lib() is not None:
        rl, rg, cpu = reference_run(pr, evals=3)
        errors = {"mixed": errors_vs(ref_lnl, ref_grad, rl, rg),
                  "fp64": errors_vs(lnl64, g64, rl, rg), "reference_lnl": rl,
                  "how": "against the reference CPU implementation (FP64) on the same inputs; "
                         "grad_branch = max_b |g_b - r_b| / (|r_b| + 0.1 rms(r))"}
    if rank == 0 and ws == 1 and args.workload == WORKLOAD and not args.no_extra:
        for name in ("codon61_n32_p10k", "aa20_n64_p20k"):
            extra[name] = workload_record(torch, lib, name, args, local)
        extra[BATCH_WORKLOAD] = batch256_record(torch, lib, args, local)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config(pr, ws),
            "precision": "FP32 partials, FP64 P(t), scalers and reductions",
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "how": "per step the new branch lengths from pinned host memory and the "
                           "whole-step graph in one beagleB200LaunchGraphWithLengths call, "
                           "then one wait for lnL and the gradient"},
            "e2e_calls": {"value": e2e_calls_value, "unit": "evals/s",
                          "h2d_bytes_per_step": h2d_calls, "d2h_bytes_per_step": d2h,
                          "how": "the same steps as the beagle.h call sequence (matrix "
                                 "update, the two fused calls, the wait)"},
            "checkpointed": ckpt,
            "plain_fp64": {"value": value64, "unit": "evals/s", "ms_per_step": ms64 / k64,
                           "mixed_over_fp64": value / value64,
                           "mixed_vs_fp64": errors_vs(ref_lnl, ref_grad, lnl64, g64)},
            "errors": errors,
            "lnl": lnl,
            "gpu_launches": (LAUNCHES_PER_EVAL - (1 if fused_walk else 0)
                             - (2 if post_root else 0)) * args.steps,
            "tuned_variants": tuned,
            "clocks": clocks_info,
        }
        if extra:
            line["workloads"] = extra
            cod = extra["codon61_n32_p10k"]
            ref = cod.get("vs_reference", {}).get("mixed", cod["mixed_vs_fp64"])
            line["target_61_state"] = {
                "workload": "codon61_n32_p10k",
                "mixed_over_fp64": cod["mixed_over_fp64"],
                "batched_x8_mixed_over_fp64": cod["batched_x8"]["batched_mixed_over_fp64"],
                "rel_lnl_err": ref["rel_lnl"], "grad_branch_err": ref["grad_branch"],
                "bars": {"ratio": 3.0, "rel_lnl": 1e-6, "grad_branch": 1e-4},
                "met": bool(cod["mixed_over_fp64"] >= 3.0 and ref["rel_lnl"] <= 1e-6
                            and ref["grad_branch"] <= 1e-4)}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_shard_arm(args):
    """--shard: ONE tree of the workload split by patterns over the ranks
    (beagle-lib_b200/shard.py), each rank evaluating its contiguous pattern
    range on its own GPU, with one all-reduce of 1 + B doubles (lnL and the
    gradient) per evaluation: NCCL over NVLink between GPUs.  Strong scaling:
    the total work is fixed as N grows.  Each step: new branch lengths in,
    the shard's evaluation, the all-reduce, lnL and the gradient out on every
    rank.  Device-timed from an event on the instance's stream before the
    first step to one on torch's stream after the last all-reduce; max over
    ranks."""
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pkg = importlib.import_module("beagle-lib_b200")
    syn, shard = pkg.synthetic, pkg.shard
    lib = pkg.load()
    pr = syn.config_problem(args.workload)
    sh = shard.pattern_shard(pr, rank, ws)
    inst = make_instance(lib, sh, "single", local)
    stream = torch.cuda.ExternalStream(inst.cudaStream())
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", local)

    def step(t):
        lnl, sums = sh.evaluate(inst, transposed_pre=sh.S > 4, lengths=t, fused=True)
        lnl = inst.getLogLikelihood()
        g = sh.branch_gradient(sums)
        if ws == 1:
            return lnl, g
        x = torch.tensor(np.concatenate([[lnl], g]), dtype=torch.float64, device=dev)
        import torch.distributed as dist
        dist.all_reduce(x, op=dist.ReduceOp.SUM)
        x = x.cpu().numpy()
        return float(x[0]), x[1:]

    for _ in range(args.warmup):
        step(pr.lengths)
    barrier(ws)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        lnl, g = step(pr.lengths * (1.0 + 1e-3 * rng.standard_normal(pr.B)))
    end.record(torch.cuda.current_stream(dev))
    end.synchronize()
    ms = max_over_ranks(start.elapsed_time(end), ws)
    lnl, g = step(pr.lengths)
    inst.finalize()
    if rank == 0:
        line = {
            "metric": METRIC, "value": args.steps / (ms / 1000.0), "unit": "evals/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(pr, ws), parallelism=f"pattern shards x{ws}"),
            "how": "one tree, contiguous pattern range per rank, one all-reduce of 1 + B "
                   "doubles per evaluation; new lengths in, lnL + gradient out per step",
            "lnl": lnl, "gpu_launches": None}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_batch_arm(args):
    """--workload batch256 as a line of its own (batch256_record)."""
    import torch
    pkg = importlib.import_module("beagle-lib_b200")
    rec = batch256_record(torch, pkg.load(), args)
    line = {
        "metric": "tree lnL+gradient evals/s, 256-tree batch, mixed batched vs per-instance",
        "value": rec["value"], "unit": "tree-evals/s", "n_gpus": 1, "steps": rec["steps"],
        "warmup": max(3, args.warmup), "ms_per_step": rec["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": rec.pop("config"), "gpu_launches": None}
    line.update(rec)
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
        state["lnl"], _ = ck.batch_checkpointed_evaluate(batch, plans, fused=True)

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
            pl.evaluate(inst, fused=True)

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
    elif args.shard:
        run_shard_arm(args)
    elif args.workload == BATCH_WORKLOAD:
        run_batch_arm(args)
    elif args.workload == BATCH_WORKLOAD + "_p50k":
        run_batch_full_arm(args)
    else:
        run_b200_arm(args)


if __name__ == "__main__":
    main()
