#!/usr/bin/env python
"""Benchmark of the blocks_3d drop-in hot path on B200: blocks_3d tasks per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload cfg2] [--schedule batched|plain]
    python bench.py --impl reference ...        the reference's CPU path (the oracle port) on the host cores

A step is one blocks_3d task of the workload (default cfg2: external spins (2,2,2,2), 2 j12 = 2 j43 = 8,
internal spins 0-22, Lambda 11, order 40, kept pole order 20, 1024 bits, xt; its six lambda orders are the
task's right-hand sides): radial recursion with derivative moments, numerators with pole shifting, the xt
map.  Inputs are synthetic (random M matrices and h_infinity: the cost does not depend on the values).
The operator's constants (plan, M tables, derivative and write_output maps) are built once before timing,
as they are once per group of tasks.  `value` times the step with h_inf already on the device; `e2e` times
the same step through the drop-in runner's host interface: h_inf copied from pinned host memory and the
write_output limbs copied back to the host inside the timed region, every step (pipelined: a copy stream
moves one step's results out and the next step's inputs in while a step runs).

With N > 1 (torchrun), every rank runs the same workload on its own GPU (independent replicas: the path has no
exchange step); the timing is the max over ranks and `value` counts the tasks of all ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--schedule", default="batched", choices=("batched", "plain"))
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sample", type=int, default=0, help="set644: time only this many task groups (0: all)")
    ap.add_argument("--no-graph", action="store_true", help="launch every kernel from Python instead of a CUDA graph")
    ap.add_argument("--rate", type=float, default=200.0, help="cfg4: Poisson arrival rate (tasks/s)")
    ap.add_argument("--requests", type=int, default=32, help="cfg4: requests in the stream")
    ap.add_argument("--cauchy", default=None, help="Cauchy kernel form (Recursion's cauchy argument)")
    ap.add_argument("--pole", default=None, choices=(None, "auto", "mma", "cuda"), help="pole-step kernel form")
    ap.add_argument("--moments", default=None, choices=(None, "staged", "per_level"), help="moments form")
    ap.add_argument("--no-set644", action="store_true", help="default run: skip the full 644-task set")
    ap.add_argument("--no-cfg4", action="store_true", help="default run: skip the serving stream at its stated rate")
    ap.add_argument("--one-step", action="store_true",
                    help="run one launched step and one JSON render of the workload, untimed, and exit (the case "
                         "that kernel profiles capture; with --schedule plain each recursion has one right-hand side)")
    return ap.parse_args()


def config_dict(workload, c, schedule="batched", world=1):
    """the workload's configuration, one dict for both arms (the residue slot buffer from the plan alone)"""
    from blocksvibe_b200 import mpf
    from blocksvibe_b200.plan import Plan
    L = mpf.limbs_for_precision(c["precision"])
    nrhs = len(range((1 - c["sign"]) // 2, c["Lam"] + 1, 2)) if "xt" in c["coords"] else 1
    pl = Plan(c["tj12"], c["tj43"], c["tjmax"], c["order"], c["pp"], reuse=True)
    slots = (4 * L + 8) * pl.Smax ** 2 * nrhs * (pl.nphys + 1)
    d = {"workload": workload, "schedule": schedule, "two_js": list(c["two_js"]), "two_j12": c["tj12"],
         "two_j43": c["tj43"], "two_j_max": c["tjmax"], "Lambda": c["Lam"], "order": c["order"],
         "kept_pole_order": c["kept"], "precision": c["precision"], "limbs": mpf.limbs_for_precision(c["precision"]),
         "coordinates": list(c["coords"]), "parallelism": f"replicas{world}", "rhs_per_task": nrhs,
         "l2": "inputs larger than L2 (residue slot buffer %.2f GB)" % (slots / 1e9)}
    return d


# ---------------------------------------------------------------- distributed plumbing
def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        # replicas only: the process group carries the barrier and the max over ranks of the timings (NCCL on
        # GPUs; gloo on CPU, as the multi-process tests run it)
        if torch.cuda.is_available() and os.environ.get("B3D_DIST_BACKEND", "nccl") == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- clocks during the timed region
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self, gpu_index=0):
        if self.proc is None:
            return None
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != str(gpu_index):
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- kernel probe (launch count, per-kernel events)
KERNELS_PER_CALL = {"b3d_pole_level": 2, "b3d_pole_level_mma": 2, "b3d_cauchy_align": 2, "b3d_cauchy_align_sm": 2}


class Probe:
    """wraps the C ABI dispatcher: counts kernel launches and records CUDA events around the calls of one
    entry point on the launching (current) stream"""

    def __init__(self):
        from blocksvibe_b200 import _lib
        self.lib = _lib
        self.orig = _lib.call
        self.launches = 0
        self.watch = None
        self.events = []
        self.by_name = None
        _lib.call = self._call

    def _call(self, name, *args):
        import torch
        self.launches += KERNELS_PER_CALL.get(name, 1)
        timed = name == self.watch or self.by_name is not None
        if timed:
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
        rc = self.orig(name, *args)
        if timed:
            e.record()
            if name == self.watch:
                self.events.append((s, e))
            if self.by_name is not None:
                self.by_name.setdefault(name, []).append((s, e))
        return rc


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


_INT8_PEAK = {}


def int8_peak_tops(device):
    if str(device) not in _INT8_PEAK:
        _INT8_PEAK[str(device)] = _int8_peak_tops(device)
    return _INT8_PEAK[str(device)]


def _int8_peak_tops(device):
    """dense INT8 tensor throughput of this GPU, measured with a plain library GEMM (torch._int_mm on 8192^3,
    best of 5): the denominator of the RNS GEMM's tensor roofline (no INT8 figure is in MEASURED_PEAKS.json)"""
    import torch
    n = 8192
    a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
    b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=device)
    best = None
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3
        best = t if best is None else min(best, t)
    return 2 * n ** 3 / best / 1e12


def profile_traffic(kernel, workload):
    """dram bytes per launch of `kernel` from the committed ncu summary of this workload, if any"""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


# ---------------------------------------------------------------- CPU baseline (oracle port on the host cores)
def cpu_baseline(c, budget, cores, anchor=True):
    """the oracle (the reference's CPU algorithm restated) on the host cores: its multiprecision MAC rate, sampled
    on the workload's own recursion for `budget` seconds on every core, divided by the MACs of EVERY stage of a
    task (recursion, moments, c, a, G, polynomial part, numerators, write_output: oracle.sample.task_macs).  The
    anchor times one complete config-1 task through the whole oracle chain on one core beside the same model's
    prediction for it, so the model's distance from a measured complete task is stated."""
    from oracle import sample as OS
    from blocksvibe_b200 import mpf
    from blocksvibe_b200.workloads import CONFIGS
    L = mpf.limbs_for_precision(c["precision"])
    per_task = OS.task_macs(c)
    macs, secs = OS.parallel_sample(c["tj12"], c["tj43"], c["tjmax"], c["order"], c["pp"], 32 * L + 64, budget, cores)
    rate = macs / secs                                     # MP MACs per second over all workers
    out = {"value": rate / per_task, "unit": "tasks/s", "cores": cores, "kind": "port",
           "sample": (f"oracle fill_residues (mpmath, {32 * L + 64}-bit) on {cores} spawned processes for "
                      f"{budget:.0f} s each, {macs:.3g} MP MACs done ({rate:.3g} MAC/s); tasks/s = MAC rate / "
                      f"{per_task:.3g} MACs of every stage of one task")}
    if anchor:
        c1 = CONFIGS["cfg1"]
        bits1 = 32 * mpf.limbs_for_precision(c1["precision"]) + 64
        measured = OS.chain_task_seconds(c1, bits1)
        m1, s1 = OS.sample(c1["tj12"], c1["tj43"], c1["tjmax"], c1["order"], c1["pp"], bits1, 3.0)
        predicted = OS.task_macs(c1) / (m1 / s1)
        out["anchor"] = {"workload": "cfg1", "measured_s": measured, "model_s": predicted,
                         "measured_over_model": measured / predicted,
                         "what": "one complete config-1 task through the oracle chain on one core, beside the MAC "
                                 "model at the same core's MAC rate"}
    return out


def json_measure(op, G, t, outs, dev, steps, cpu):
    """blocks_3d's per-spin JSON files of one task from the step's device outputs (the writer after the
    drop-in boundary, GPU-formatted): device time of its three kernels (CUDA events), end-to-end time with the
    device-to-host copy of the text, and (cpu) the oracle's formatter timed on a sample of the same numbers"""
    import torch
    from blocksvibe_b200 import jsonout as JO
    opts = JO.task_options(G, t)
    outputs = {c: list(o.outputs) for (c, d), o in op.outs.items() if d == t.delta_1_plus_2}
    x0 = next(iter(outs.values()))
    w = JO.SpinWriter(opts, sorted(t.two_js_internal), t.pp, outputs, op.plan.Smax, 1, x0.shape[-1], dev)
    t0 = time.perf_counter()
    files = w.render(outs)                                 # builds the tables and caches the skeleton
    first_s = time.perf_counter() - t0
    text_bytes = sum(len(f) for f in files.values())
    n = w.last_numbers
    per = {}
    e2e = []
    for _ in range(steps):
        ev = []
        w.render_device(outs, 0, events=ev)
        torch.cuda.synchronize()
        for name, a, b in ev:
            per.setdefault(name, []).append(a.elapsed_time(b))
        s0 = time.perf_counter()
        w.render(outs)
        torch.cuda.synchronize()
        e2e.append(time.perf_counter() - s0)
    dev_ms = sum(statistics.mean(v) for v in per.values())
    alg = n * (4 * x0.L + 8) + text_bytes                 # numbers read once, text written once
    hbm, kind = peaks()
    res = {"files": len(files), "numbers": n, "text_bytes": text_bytes, "digits": w.p,
           "kernel_ms": {k: round(statistics.mean(v), 4) for k, v in per.items()}, "device_ms": dev_ms,
           "e2e_ms": statistics.mean(e2e) * 1e3, "e2e_what": "device kernels + copy of the text to pinned host memory",
           "first_render_s": first_s,
           "roofline": {"kernels": "b3d_format_decimal + b3d_poly_sizes + b3d_emit_text", "bound": "hbm",
                        "achieved": alg / (dev_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                        "frac": alg / (dev_ms / 1e3) / 1e9 / hbm, "peak_source": kind,
                        "algorithmic_bytes": alg}}
    if cpu:
        import numpy as np
        from oracle import jsonfmt as OJ
        m = x0.m.reshape(x0.L, -1)[:, :400].cpu().numpy().astype(np.int64) & 0xFFFFFFFF
        e = x0.e.reshape(-1)[:400].cpu().numpy()
        vals = []
        for i in range(m.shape[1]):
            v = int.from_bytes(m[:, i].astype("<u4").tobytes(), "little", signed=True)
            vals.append((v, int(e[i]) if v else 0))
        s0 = time.perf_counter()
        for v, ex in vals:
            OJ.fmt(v, ex, w.p)
        per_num = (time.perf_counter() - s0) / len(vals)
        res["cpu_baseline"] = {"value": per_num * n, "unit": "s per task (number formatting)", "cores": 1,
                               "kind": "port", "sample": f"oracle jsonfmt.fmt on {len(vals)} of the task's {n} numbers, "
                                                         "extrapolated (the reference's production writer uses MPFR "
                                                         "through gmpy2, not installed here)"}
    return res


def run_reference(args):
    """--impl reference: the reference's CPU path (the oracle port of recursion_ref) on the host cores"""
    from blocksvibe_b200.workloads import CONFIGS
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    c = CONFIGS[args.workload]
    cores = os.cpu_count() or 1
    budget = max(2.0, min(args.cpu_budget, 150.0 / max(1, args.steps + args.warmup)))
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(c, budget, cores, anchor=i == args.warmup + args.steps - 1)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.mean(vals)
    r["value"] = v
    line = {"impl": "reference", "metric": "blocks_3d tasks/s", "value": v, "unit": "tasks/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "mpf (mpmath)", "data": "synthetic",
            "config": config_dict(args.workload, c, args.schedule, args.gpus),
            "cpu_baseline": r, "e2e": {"value": v, "unit": "tasks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    from blocksvibe_b200 import dropin as DI, mpf, roofline as RL
    from blocksvibe_b200.mpf import MPF
    from blocksvibe_b200.workloads import CONFIGS, make_tasks

    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = CONFIGS[args.workload]
    G, tasks = make_tasks(c, nq=1, seed=rank)
    t = tasks[0]
    parity = t.parity
    ns = t.lambda_orders(G.Lambda)
    t_setup = time.perf_counter()
    op = DI.Operator(G, t.pp, parity, None, t.two_js_internal, list(t.coordinates), [t.delta_1_plus_2], dev)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    dtask = DI.Task(t.q4, t.sign, t.pp, t.two_js_internal, t.coordinates, t.delta_1_plus_2,
                    {n: MPF(h.m.to(dev), h.e.to(dev)) for n, h in t.h_inf.items()})
    run = op.run_batched if args.schedule == "batched" else op.run_plain
    if args.one_step:
        from blocksvibe_b200 import jsonout as JO
        probe = Probe()
        outs = op.apply_outputs(run([dtask], ns), t.delta_1_plus_2)
        outputs = {cc: list(o.outputs) for (cc, d), o in op.outs.items() if d == t.delta_1_plus_2}
        x0 = next(iter(outs.values()))
        w = JO.SpinWriter(JO.task_options(G, t), sorted(t.two_js_internal), t.pp, outputs, op.plan.Smax, 1,
                          x0.shape[-1], dev)
        w.render_device(outs, 0)
        torch.cuda.synchronize()
        print(json.dumps({"one_step": args.workload, "schedule": args.schedule, "launches": probe.launches,
                          "peak_device_bytes": torch.cuda.max_memory_allocated(dev)}), flush=True)
        return
    graph = None
    if args.schedule == "batched" and not args.no_graph:
        graph = DI.GraphStep(op, 1, ns, t.delta_1_plus_2)
        graph.load([dtask])

    def step_device():
        if graph is not None:
            return graph.run()
        nums = run([dtask], ns)
        return op.apply_outputs(nums, t.delta_1_plus_2)

    h2d = sum(h.m.numel() * 4 + h.e.numel() * 8 for h in t.h_inf.values())
    d2h = [0]

    def step_e2e():
        if graph is not None:
            out = graph.run([t])
        else:
            out = op.apply_outputs(run([t], ns), t.delta_1_plus_2)
        host = op.to_host(out)
        d2h[0] = sum(m.numel() * 4 + e.numel() * 8 for m, e in host.values())
        return host

    probe = Probe()
    # per-kernel split (one untimed step launched from Python, the moments not overlapped with the next level's
    # Cauchy step so that every entry point is timed alone) to pick the dominant kernel; kernels per step
    probe.by_name = {}
    n0 = probe.launches
    op.rec.overlap_hook = False
    op.apply_outputs(run([dtask], ns), t.delta_1_plus_2)
    torch.cuda.synchronize()
    op.rec.overlap_hook = True
    launches = probe.launches - n0
    split = {k: sum(s.elapsed_time(e) for s, e in v) for k, v in probe.by_name.items()}
    probe.by_name = None
    dominant = max(split, key=split.get)

    for _ in range(args.warmup):
        step_device()
    clocks = Clocks()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    if rank == 0:
        clocks.start()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        step_device()
    end.record()
    torch.cuda.synchronize()
    barrier(world)
    ms = start.elapsed_time(end) / args.steps
    # the dominant kernel's launches timed with events (steps launched from Python: a graph replay has no
    # per-launch events), on the launching stream
    probe.watch, probe.events = dominant, []
    op.rec.overlap_hook = False
    for _ in range(min(2, args.steps)):
        op.apply_outputs(run([dtask], ns), t.delta_1_plus_2)
    torch.cuda.synchronize()
    op.rec.overlap_hook = True
    kernel_ms = [s.elapsed_time(e) for s, e in probe.events]
    probe.watch = None
    ksteps = min(2, args.steps)
    clk = clocks.stop(local) if rank == 0 else None
    ms = max_over_ranks(ms, world, dev)

    # the other schedule, same timing, for the batched-vs-plain comparison
    other = op.run_plain if args.schedule == "batched" else op.run_batched
    for _ in range(2):
        op.apply_outputs(other([dtask], ns), t.delta_1_plus_2)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(args.steps):
        op.apply_outputs(other([dtask], ns), t.delta_1_plus_2)
    s1.record()
    torch.cuda.synchronize()
    other_ms = max_over_ranks(s0.elapsed_time(s1) / args.steps, world, dev)

    # end to end through the host interface.  Throughput: with the graph, the pipelined runner (every step's
    # h_inf copied in from pinned host memory and its results copied out to pinned host memory, on a copy
    # stream that overlaps the neighbouring steps); without it, one task at a time.  Latency (p50 / p99): one
    # task at a time, copy in, step, copy out.
    for _ in range(args.warmup):
        step_e2e()
    torch.cuda.synchronize()
    barrier(world)
    lat = []
    e0 = time.perf_counter()
    for _ in range(args.steps):
        s = time.perf_counter()
        step_e2e()
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - s)
    e2e_s = (time.perf_counter() - e0) / args.steps
    e2e_mode = "one task at a time"
    if graph is not None:
        for _ in graph.run_stream([[t]] * args.warmup):
            pass
        torch.cuda.synchronize()
        barrier(world)
        e0 = time.perf_counter()
        for host in graph.run_stream([[t]] * args.steps):
            d2h[0] = sum(m.numel() * 4 + e.numel() * 8 for m, e in host.values())
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - e0) / args.steps
        e2e_mode = "pipelined (GraphStep.run_stream)"
    barrier(world)
    e2e_s = max_over_ranks(e2e_s, world, dev)

    # blocks_3d's JSON files of the task (GPU formatter), after the boundary
    jout = json_measure(op, G, t, op.apply_outputs(run([dtask], ns), t.delta_1_plus_2), dev, args.steps,
                        rank == 0 and world == 1 and not args.no_cpu_baseline)

    # roofline of the dominant kernel: algorithmic bytes per launch / mean launch time
    L, N, S = op.L, op.plan.Smax ** 2 * (len(ns) if args.schedule == "batched" else 1), op.plan.Smax
    levs = [lv for lv in op.plan.levels if lv]
    if dominant in ("b3d_cauchy_level", "b3d_cauchy_level2", "b3d_cauchy_level3", "b3d_cauchy_level4"):
        per_step_bytes = sum(RL.cauchy_level_bytes(lv, N, L) for lv in levs if lv["m"] > 0 or dominant == "b3d_cauchy_level") \
            * (1 if args.schedule == "batched" else len(ns))
    elif dominant in ("b3d_pole_level", "b3d_pole_level_mma"):
        per_step_bytes = sum(RL.pole_level_bytes(lv, N, S, L) for lv in levs) * (1 if args.schedule == "batched" else len(ns))
    else:
        per_step_bytes = None
    hbm, peak_kind = peaks()
    roof = None
    if per_step_bytes and kernel_ms:
        nl = len(kernel_ms) / ksteps
        achieved = (per_step_bytes / nl) / (statistics.mean(kernel_ms) / 1e3) / 1e9
        traffic = profile_traffic(dominant, args.workload)
        roof = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": per_step_bytes / nl, "mean_launch_ms": statistics.mean(kernel_ms)}
    # tensor roofline of the residue GEMM kernel (k_rns_mma): algorithmic int8 MACs / its event-timed launches
    from blocksvibe_b200 import rns as RNS
    RNS.MMA_TIMER, RNS.MMA_STATS["alg_macs"], RNS.MMA_STATS["macs"] = [], 0, 0
    op.apply_outputs(run([dtask], ns), t.delta_1_plus_2)
    torch.cuda.synchronize()
    tensor_roof = None
    if RNS.MMA_TIMER:
        mma_s = sum(s.elapsed_time(e) for s, e in RNS.MMA_TIMER) / 1e3
        peak8 = int8_peak_tops(dev)
        ach = 2 * RNS.MMA_STATS["alg_macs"] / mma_s / 1e12
        tensor_roof = {"kernel": "k_rns_mma (tcgen05.mma.kind::i8)", "bound": "tensor", "achieved": ach, "peak": peak8,
                       "unit": "TOPS", "frac": ach / peak8, "peak_source": "measured here: torch._int_mm 8192^3",
                       "issued_over_algorithmic": RNS.MMA_STATS["macs"] / RNS.MMA_STATS["alg_macs"],
                       "launches_per_step": len(RNS.MMA_TIMER), "ms_per_step": mma_s * 1e3}
    RNS.MMA_TIMER = None
    # tensor roofline of the pole step when it runs on the tensor cores: int8 MACs issued by its MMAs per step
    # over its CUDA-event time per step (split), with the share of those MACs the exact sums need
    pole_roof = None
    if "b3d_pole_level_mma" in split:
        issued = useful = 0
        for lv in levs:
            i_, u_ = RL.pole_mma_macs(lv, N, S, L)
            issued, useful = issued + i_, useful + u_
        reps = 1 if args.schedule == "batched" else len(ns)
        pole_s = split["b3d_pole_level_mma"] / 1e3
        peak8 = int8_peak_tops(dev)
        ach = 2 * issued * reps / pole_s / 1e12
        pole_roof = {"kernel": "k_pole_mma (tcgen05.mma.kind::i8)", "bound": "tensor", "achieved": ach, "peak": peak8,
                     "unit": "TOPS", "frac": ach / peak8, "peak_source": "measured here: torch._int_mm 8192^3",
                     "issued_over_algorithmic": issued / useful, "ms_per_step": pole_s * 1e3}
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(c, args.cpu_budget, os.cpu_count() or 1)
    set644 = cfg4 = None
    if world == 1 and not args.no_set644:
        from blocksvibe_b200.workloads import task_set_644
        set644 = measure_set(dev, task_set_644(), 1, 1, world)
    if world == 1 and not args.no_cfg4:
        cfg4 = measure_stream(dev, 200.0, 48, world)
    lat.sort()
    pct = lambda q: lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))] * 1e3
    value = world / (ms / 1e3)
    line = {"metric": "blocks_3d tasks/s", "value": value, "unit": "tasks/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mpf int32 limbs", "data": "synthetic (random M and h_inf of the config's shape)",
            "config": config_dict(args.workload, c, args.schedule, world), "cuda_graph": graph is not None,
            "e2e": {"value": world / e2e_s, "unit": "tasks/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h[0],
                    "mode": e2e_mode},
            "latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "source": "e2e steps, one task at a time"},
            "gpu_launches": launches, "setup_s": t_setup,
            "other_schedule": {"schedule": "plain" if args.schedule == "batched" else "batched",
                               "value": world / (other_ms / 1e3), "ms_per_step": other_ms},
            "kernel_split_ms": {k: round(v, 3) for k, v in sorted(split.items(), key=lambda x: -x[1])},
            "e2e_with_json": {"value": world / (e2e_s + jout["e2e_ms"] / 1e3), "unit": "tasks/s",
                              "what": "e2e plus the task's blocks_3d JSON files formatted on the GPU and copied to "
                                      "pinned host memory (the files blocks_3d writes)"},
            "roofline": roof, "tensor_roofline": tensor_roof, "pole_tensor_roofline": pole_roof, "json_output": jout, "cpu_baseline": cpu, "clocks": clk,
            "set644": set644, "cfg4": cfg4}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def measure_set(dev, groups, steps, warmup, world, budget_frac=0.35):
    """the tasks of `groups` ((config, task count) pairs of the seeded 644-task set): every group as batched passes
    (all its tasks and lambda orders per pass, split into chunks whose device footprint fits budget_frac of the
    free memory), task by task with one recursion per lambda order (the plain per-task path), and through the
    serving loop (all submitted at once).  Operators are built before timing; h_inf is resident on the device."""
    import torch
    from blocksvibe_b200 import dropin as DI, serve
    from blocksvibe_b200.workloads import make_device_tasks
    ntask = sum(n for _, n in groups)
    t0 = time.perf_counter()
    prepared = []
    free, _ = torch.cuda.mem_get_info(dev)
    for gi, (c, n) in enumerate(groups):
        G, tasks = make_device_tasks(c, n, dev, seed=gi)
        t = tasks[0]
        op = DI.Operator(G, t.pp, t.parity, None, t.two_js_internal, list(t.coordinates), [t.delta_1_plus_2], dev)
        ns = t.lambda_orders(G.Lambda)
        per_task = max(1, op.footprint_bytes(len(ns)))
        chunk = max(1, min(len(tasks), int(budget_frac * free // (2 * per_task))))
        prepared.append((op, tasks, ns, t.delta_1_plus_2, chunk))
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0

    def batched():
        for op, tasks, ns, d12, chunk in prepared:
            for i in range(0, len(tasks), chunk):
                op.apply_outputs(op.run_batched(tasks[i:i + chunk], ns), d12)

    def plain():
        for op, tasks, ns, d12, chunk in prepared:
            for task in tasks:
                op.apply_outputs(op.run_plain([task], ns), d12)

    out = {}
    for name, fn in (("batched", batched), ("plain", plain)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier(world)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(steps):
            fn()
        s1.record()
        torch.cuda.synchronize()
        out[name] = max_over_ranks(s0.elapsed_time(s1) / steps, world, dev)
    # batched passes replayed as CUDA graphs (the production form of a batched step, as in the cfg2 line): one
    # group at a time, its graph per chunk size captured untimed, one warm-up replay, then `steps` timed replays
    # with CUDA events; the graph and its memory pool are released before the next group (all 58 would not fit).
    # The timed work per group equals the launched batched pass: every chunk of every task, h_inf loaded from
    # the resident device tensors into the graph's static input.
    graph_ms = 0.0
    torch.cuda.empty_cache()                               # the launched arms' cached blocks: graphs use own pools
    for op, tasks, ns, d12, chunk in prepared:
        parts = [tasks[i:i + chunk] for i in range(0, len(tasks), chunk)]
        steps_of = {n: DI.GraphStep(op, n, ns, d12) for n in sorted({len(q) for q in parts})}
        for q in parts:
            steps_of[len(q)].run(q)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(steps):
            for q in parts:
                steps_of[len(q)].run(q)
        g1.record()
        torch.cuda.synchronize()
        graph_ms += g0.elapsed_time(g1) / steps
        del steps_of
        torch.cuda.empty_cache()
    out["batched_graph"] = max_over_ranks(graph_ms, world, dev)
    # the serving loop: all tasks submitted at once, continuous batching per operator, two workers on their own
    # streams, admission by footprint, results left on the device for the GPU JSON writer (wall clock from the
    # first submit to the last result)
    srv = serve.Server(dev, workers=2, max_batch=32, host_results=False)
    for op, tasks, ns, d12, chunk in prepared:
        srv.add_operator(op, op.group, tasks[0])
    try:
        warm = [srv.submit(op.group, tasks[0], None) for op, tasks, ns, d12, chunk in prepared]
        for r in warm:
            srv.wait(r, timeout=900)
        n0, nb0 = len(srv.finished), len(srv.batches)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        reqs = [srv.submit(op.group, t, None) for op, tasks, ns, d12, chunk in prepared for t in tasks]
        for r in reqs:
            srv.wait(r, timeout=1800)
        serve_s = time.perf_counter() - t1
        lat = sorted(r.done - r.arrival for r in srv.finished[n0:])
    finally:
        srv.close()
    plain_rate = world * ntask / (out["plain"] / 1e3)
    return {"groups": len(groups), "tasks": ntask, "setup_s": setup_s,
            "batched": {"value": world * ntask / (out["batched"] / 1e3), "unit": "tasks/s", "ms": out["batched"]},
            "plain": {"value": plain_rate, "unit": "tasks/s", "ms": out["plain"],
                      "what": "one task at a time, one recursion per lambda order (the reference's schedule)"},
            "batched_over_plain": out["plain"] / out["batched"],
            "batched_graph": {"value": world * ntask / (out["batched_graph"] / 1e3), "unit": "tasks/s",
                              "ms": out["batched_graph"],
                              "what": "the batched passes replayed as one CUDA graph per group and chunk size"},
            "batched_graph_over_plain": out["plain"] / out["batched_graph"],
            "serving_loop": {"value": world * ntask / serve_s, "unit": "tasks/s", "wall_s": serve_s,
                             "requests": len(reqs), "batches": len(srv.batches) - nb0,
                             "latency_ms": {"p50": serve.percentile(lat, 0.5) * 1e3,
                                            "p99": serve.percentile(lat, 0.99) * 1e3},
                             "over_plain": (world * ntask / serve_s) / plain_rate,
                             "includes": "results left on the device for the GPU JSON writer (wall clock)"},
            "timing": f"{steps} timed pass(es) after {warmup} warm-up pass(es) of every task"}


def run_set(args):
    """--workload set644: the seeded 644-task set (all of it, or --sample groups), batched vs plain vs serving"""
    import torch
    from blocksvibe_b200.workloads import task_set_644
    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    groups = task_set_644()
    if args.sample and args.sample < len(groups):
        step = max(1, len(groups) // args.sample)
        groups = groups[::step][:args.sample]
    r = measure_set(dev, groups, args.steps, max(1, args.warmup), world)
    if rank == 0:
        line = {"metric": "blocks_3d tasks/s", "value": r["batched"]["value"], "unit": "tasks/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["batched"]["ms"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "mpf int32 limbs",
                "data": "synthetic (seeded 644-task set, random M and h_inf)",
                "config": {"workload": "set644", "groups": r["groups"], "tasks": r["tasks"]}, "set644": r}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def measure_stream(dev, rate, requests, world=1):
    """a Poisson stream of config-2-shaped tasks (512 / 768 / 1024 / 1280 bits, pole shifting on for half of
    them: kept pole order 20, or 40 = order: none) through the serving loop at `rate` tasks/s offered, results
    copied to the host; then the same requests submitted all at once (the loop's saturation throughput).
    Operators are built before the stream starts."""
    import random
    import torch
    from blocksvibe_b200 import dropin as DI, serve
    from blocksvibe_b200.workloads import CONFIGS, make_device_tasks
    kinds = [dict(CONFIGS["cfg2"], precision=p, kept=k) for p in (512, 768, 1024, 1280) for k in (20, 40)]
    per = max(1, (requests + len(kinds) - 1) // len(kinds))
    pools, ops = [], []
    t0 = time.perf_counter()
    for ki, c in enumerate(kinds):
        G, tasks = make_device_tasks(c, per, dev, seed=100 + ki)
        t = tasks[0]
        op = DI.Operator(G, t.pp, t.parity, None, t.two_js_internal, list(t.coordinates), [t.delta_1_plus_2], dev)
        op.apply_outputs(op.run_batched(tasks[:1], t.lambda_orders(G.Lambda)), t.delta_1_plus_2)   # warm
        ops.append((op, G, t))
        pools.append((G, tasks))
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    rng = random.Random(4)
    items = []
    for i in range(requests):
        G, tasks = pools[rng.randrange(len(pools))]
        items.append((G, tasks[i % len(tasks)], None))

    def server():
        srv = serve.Server(dev, workers=2, max_batch=16)
        for op, G, t in ops:
            srv.add_operator(op, G, t)
        return srv

    srv = server()
    depth = []
    stop = [False]

    def sample_depth():
        while not stop[0]:
            with srv.lock:
                depth.append(len(srv.pending))
            time.sleep(0.005)
    import threading
    th = threading.Thread(target=sample_depth, daemon=True)
    th.start()
    try:
        reqs, wall = serve.replay(srv, items, rate, seed=5)
    finally:
        stop[0] = True
        th.join()
        srv.close()
    lat = sorted(r.done - r.arrival for r in reqs)
    arrivals = serve.poisson_arrivals(rate, requests, seed=5)
    srv2 = server()
    try:
        s0 = time.perf_counter()
        burst = [srv2.submit(G, t, M) for G, t, M in items]
        for r in burst:
            srv2.wait(r, timeout=1800)
        sat_s = time.perf_counter() - s0
    finally:
        srv2.close()
    achieved = world * len(reqs) / wall
    return {"offered_rate": rate, "requests": len(reqs), "arrival_span_s": arrivals[-1],
            "achieved": {"value": achieved, "unit": "tasks/s", "wall_s": wall},
            "latency_ms": {"p50": serve.percentile(lat, 0.5) * 1e3, "p99": serve.percentile(lat, 0.99) * 1e3,
                           "at": f"{rate} tasks/s offered"},
            "queue_depth": {"max": max(depth, default=0), "mean": statistics.mean(depth) if depth else 0},
            "saturation": {"value": world * len(burst) / sat_s, "unit": "tasks/s",
                           "what": "the same requests submitted at once"},
            "meets_offered_rate": achieved >= 0.95 * rate,
            "batches": len(srv.batches), "peak_in_flight_bytes": srv.peak_in_flight, "setup_s": setup_s,
            "precisions": [512, 768, 1024, 1280], "pole_shifting": "half (kept 20, or none)",
            "results": "copied to host (pinned)"}


def run_stream(args):
    """--workload cfg4: the serving stream at --rate tasks/s (the configuration states 200)"""
    import torch
    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    r = measure_stream(dev, args.rate, args.requests, world)
    if rank == 0:
        line = {"metric": "blocks_3d tasks/s", "value": r["achieved"]["value"], "unit": "tasks/s", "n_gpus": world,
                "steps": r["requests"], "warmup": 8, "ms_per_step": 1e3 / r["achieved"]["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "mpf int32 limbs",
                "data": "synthetic (Poisson stream of random config-2-shaped tasks)",
                "config": {"workload": "cfg4", "arrival_rate": args.rate, "requests": r["requests"]}, "cfg4": r}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    from blocksvibe_b200 import derivatives as DV, recursion as RC
    if args.cauchy:
        RC.CAUCHY = args.cauchy
    if args.pole:
        RC.POLE = args.pole
    if args.moments:
        DV.MOMENTS = args.moments
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "set644":
        run_set(args)
    elif args.workload == "cfg4":
        run_stream(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
