#!/usr/bin/env python
"""Benchmark of the direct-summation gravity path on B200.

Metric: G pair-interactions/s of the split-FP32 kernel (pairs = sum over sets
of N_s^2, self pair included), with the plain FP64 GPU kernel, the accuracy of
split-FP32 against it, and the reference's CPU path (C restatement of
cpu_grav.f) on a bounded sample reported beside it.

One step = one gravity call over the whole workload with inputs resident in
HBM (``value``); ``e2e`` repeats it through the reference-facing Fortran
C-ABI (firsthalf_grav_forces_/lasthalf_grav_forces_) from host arrays, copies
included.  Default workload: config3, the N=1,048,576 red-giant model; the
default run also measures the batched launch on config4 (64 uneven models,
against one call per model) and the graph-captured sweep on config5
(``config4_batched``, ``config5_graph_sweep``).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload config1..config5]

Multi-GPU (torchrun, one process per GPU): the reference's own split of the
gravity rows across GPU ranks (main.f:283-295).  Every rank holds its own
rows' positions; each step all-gathers the five source arrays over NCCL,
evaluates the rank's rows against all n sources and all-gathers the results
(balAV3.f:423-434 gathers them too).  The total work is fixed as N grows
(strong scaling); ``value`` = all pairs / the slowest rank's time.  Batched
workloads are sharded by whole sets instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "G pair-interactions/s: split-FP32 vs plain FP64 GPU at <=1e-6 rel accel error"
UNIT = "G pair-interactions/s"
FLOPS_PER_PAIR = 20  # far-field acc + pot convention (FMA = 2, rsqrt = 1)
FP64_INSTR_PER_PAIR = 18  # FP64 pipe instructions per far pair of the FP64 kernel
F32_LANE_OPS_PER_PAIR = 13  # FMA-pipe lane-ops per far pair of the split-FP32 kernel


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="config3")
    p.add_argument("--precision", default="f32split", choices=["f32split", "fp64"])
    p.add_argument("--nkernel", type=int, default=0)
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target length of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the config4 (batched) and config5 (graph sweep) sections")
    p.add_argument("--graph-calls", type=int, default=20,
                   help="timed graph replays in the config5 section (and with --graph)")
    p.add_argument("--variant", type=int, default=-1,
                   help="force a kernel variant of --precision (default: tuned/automatic)")
    p.add_argument("--fp64-band", type=float, default=None,
                   help="split-FP32: pairs with r < band * max(H) are evaluated in FP64 "
                        "(default: the library's)")
    p.add_argument("--refine", type=float, default=None,
                   help="split-FP32: FP64 refine of rows with error scale G > T |a| "
                        "(default: the library's; 0 = off)")
    p.add_argument("--graph", action="store_true",
                   help="batched workloads: each step replays a captured CUDA graph of "
                        "(seeded 1e-3 position kick + gravity) on device-resident state")
    p.add_argument("--no-separate", action="store_true",
                   help="batched workloads: skip the one-call-per-set comparison")
    p.add_argument("--l2-flush", default="write", choices=["write", "read"],
                   help="L2 flush before every timed step: write 256 MB (default), or read "
                        "512 MB, which evicts without leaving dirty lines for the next "
                        "kernel to write back (for DRAM-traffic captures)")
    p.add_argument("--phases", action="store_true",
                   help="load the diagnostic build (python -m starsmasher_b200.build --phases) and "
                        "report the split-FP32 kernel's cycles per phase over 2 extra calls")
    p.add_argument("--parallel", default="auto", choices=["auto", "rowsplit", "setshard"],
                   help="multi-rank decomposition; auto: the reference's row split for one set, "
                        "whole sets per rank for batches.  rowsplit/setshard also force the "
                        "multi-rank path (NCCL) with a single rank, to exercise it on one GPU")
    p.add_argument("--tree-thetas", default="0.3,0.5",
                   help="single-set workloads: opening angles of the Barnes-Hut tree "
                        "section ('' skips it); accuracy against the FP64 kernel")
    return p.parse_args()


class Clocks:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(ws, target_s: float):
    """The reference's CPU path (oracle: C restatement of cpu_grav.f, the
    j >= i triangle with Newton's third law, all host cores) on a bounded
    sample of rows of the same workload; credited ordered pairs = 2 x triangle
    evaluations - self pairs."""
    import oracle
    threads = oracle.max_threads()
    results = []
    total_pairs = 0
    total_t = 0.0
    for s in range(ws.nsets):
        if total_t >= target_s:
            break
        a, b = int(ws.offsets[s]), int(ws.offsets[s + 1])
        n = b - a
        x, y, z, m, r2 = (arr[a:b] for arr in (ws.x, ws.y, ws.z, ws.m, ws.range2))
        # calibrate on a slice in the middle of the triangle (>= 0.3 s of work)
        lo = n // 3
        rows = max(threads, min(n - lo, 2 * threads))
        while True:
            t0 = time.perf_counter()
            oracle.triangle(x, y, z, m, r2, 0, lo, lo + rows, threads)
            dt = time.perf_counter() - t0
            if dt >= 0.3 or lo + rows >= n or dt >= target_s:
                break
            rows = min(n - lo, int(rows * max(2.0, 0.4 / max(dt, 1e-3))))
        evals = sum(n - i for i in range(lo, lo + rows))
        rate = evals / max(dt, 1e-9)
        want = max(0.0, target_s - total_t) * rate
        hi = lo
        acc = 0
        while hi < n and acc < want:
            acc += n - hi
            hi += 1
        hi = max(hi, lo + 1)
        t0 = time.perf_counter()
        oracle.triangle(x, y, z, m, r2, 0, lo, hi, threads)
        dt = time.perf_counter() - t0
        evals = sum(n - i for i in range(lo, hi))
        credited = 2 * evals - (hi - lo)
        total_pairs += credited
        total_t += dt
        results.append({"set": s, "rows": [lo, hi], "seconds": dt})
    value = total_pairs / total_t / 1e9
    sample = ("triangle rows " + ", ".join(f"set{r['set']}[{r['rows'][0]}:{r['rows'][1]}]"
                                           for r in results)
              + f" of {ws.name}; {total_pairs:.3e} credited ordered pairs in {total_t:.1f} s")
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}


def load_workload(name: str):
    """configN (the five benchmark workloads) or polytrope:N (one equal-mass
    n=3 polytrope of N particles, for small profiling cases)."""
    from starsmasher_b200 import inputs
    if name.startswith("polytrope:"):
        n = int(name.split(":")[1])
        return inputs.single_polytrope(n, 3.0, seed=10)
    seed = {"config1": 1, "config2": 2, "config3": 3, "config4": 4, "config5": 5}[name]
    return inputs.cached(name, seed=seed)


def accuracy(res_f32, res64):
    """Per-particle relative errors of (ax, ay, az, pot) against the FP64
    kernel's; rows with |a| < 1e-3 median |a| are reported separately."""
    num = np.sqrt(sum((a - b) ** 2 for a, b in zip(res_f32[:3], res64[:3])))
    amag = np.sqrt(sum(b ** 2 for b in res64[:3]))
    e = num / amag
    ill = amag < 1e-3 * np.median(amag)
    ep = np.abs(res_f32[3] - res64[3]) / np.abs(res64[3])
    med = float(np.median(amag))
    worst = int(np.argmax(np.where(ill, -1.0, e)))
    return {"reference": "plain FP64 GPU kernel, all rows",
            "acc_rel_max": float(e[~ill].max()), "acc_rel_rms": float(np.sqrt(np.mean(e[~ill] ** 2))),
            "acc_abs_max_over_median_a": float(num.max() / med),
            "worst_particle_a_over_median_a": float(amag[worst] / med),
            "acc_rel_max_illconditioned": float(e[ill].max()) if ill.any() else None,
            "n_illconditioned": int(ill.sum()),
            "pot_rel_max": float(ep.max()), "pot_rel_rms": float(np.sqrt(np.mean(ep ** 2)))}


def run_reference_arm(args, world, rank):
    """--impl reference: the reference's CPU gravity path (the Fortran does
    not compile here -- no Fortran compiler -- so its C restatement in
    oracle/ is timed) on all host cores, K bounded samples of the workload."""
    if rank != 0:
        return
    ws = load_workload(args.workload)
    for _ in range(args.warmup):
        cpu_baseline(ws, 0.5)
    vals = []
    last = None
    t_all = time.perf_counter()
    per_step = max(2.0, args.cpu_seconds / max(1, args.steps))
    for _ in range(args.steps):
        last = cpu_baseline(ws, per_step)
        vals.append(last["value"])
    elapsed = time.perf_counter() - t_all
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": ws.name, "n": ws.n, "nsets": ws.nsets, "pairs_per_step": ws.pairs,
                   "nkernel": 0, "algorithm": "cpu_grav.f triangle (C restatement), sampled rows"},
        "cpu_baseline": dict(last, value=value),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class Timer:
    """CUDA-event timing of steps on one stream, with an L2 flush (a 256 MB
    write, > 126 MB of L2; or a 512 MB read) before every timed step."""

    def __init__(self, torch, stream, device, mode="write"):
        self.torch = torch
        self.stream = stream
        self.mode = mode
        n = (64 if mode == "write" else 128) * 1024 * 1024
        self.flush = torch.ones(n, dtype=torch.float32, device=f"cuda:{device}")

    def do_flush(self):
        if self.mode == "write":
            self.flush.zero_()
        else:
            self.flush.sum()

    def run(self, fn, steps):
        torch = self.torch
        evs = []
        for _ in range(steps):
            self.do_flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            fn()
            e1.record(self.stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / max(1, steps)


def phase_shares(ph):
    """Shares of consumer-warp and producer-warp cycles per phase, and the
    tile counts, from Context.phase_read()."""
    cons = ("item", "rows", "wait_full", "far", "checked", "near", "end")
    prod = ("producer_wait", "producer_work")
    ct = sum(ph[k] for k in cons) or 1
    pt = sum(ph[k] for k in prod) or 1
    nf, nc = ph["n_far"], ph["n_checked"]
    return {"consumer_share": {k: ph[k] / ct for k in cons},
            "producer_share": {k: ph[k] / pt for k in prod},
            "checked_tile_fraction": nc / max(1, nf + nc),
            "cycles_per_far_tile": ph["far"] / max(1, nf),
            "cycles_per_checked_tile": ph["checked"] / max(1, nc),
            "near_eval_calls": ph["n_near"], "items_per_consumer_warp_total": ph["n_items"],
            "raw": ph}


def upload(torch, ws, device):
    dt = torch.float64
    X = [torch.as_tensor(a).to(device=f"cuda:{device}", dtype=dt)
         for a in (ws.x, ws.y, ws.z, ws.m, ws.range2)]
    outs = [torch.empty(ws.n, dtype=dt, device=f"cuda:{device}") for _ in range(4)]
    return X, outs


def config4_section(torch, ctx, timer, device, args):
    """The batched persistent launch on the uneven-N batch (config4): one
    batched call against one call per model (split-FP32, and plain FP64),
    with its accuracy against the FP64 kernel."""
    ws = load_workload("config4")
    X, outs = upload(torch, ws, device)

    def batched(prec="f32split"):
        ctx.batch_forces_device(ws.offsets, *X, *outs, nkernel=args.nkernel, precision=prec)

    def separate(prec="f32split"):
        for s in range(ws.nsets):
            a, b = int(ws.offsets[s]), int(ws.offsets[s + 1])
            ctx.forces_device(b - a, *(t[a:b] for t in X), *(o[a:b] for o in outs),
                              nkernel=args.nkernel, precision=prec)

    batched()
    torch.cuda.synchronize()
    ms_b = timer.run(batched, 3)
    res32 = [o.cpu().numpy() for o in outs]
    refined = ctx.last_refine_rows()
    separate()
    torch.cuda.synchronize()
    ms_s = timer.run(separate, 2)
    separate("fp64")
    ms_s64 = timer.run(lambda: separate("fp64"), 1)
    batched("fp64")
    ms_b64 = timer.run(lambda: batched("fp64"), 1)
    res64 = [o.cpu().numpy() for o in outs]
    pairs = ws.pairs
    return {"workload": ws.name, "n": ws.n, "nsets": ws.nsets, "pairs_per_step": pairs,
            "batched_ms": ms_b, "batched_value": pairs / (ms_b * 1e-3) / 1e9,
            "separate_calls_ms": ms_s, "speedup_batched_vs_separate": ms_s / ms_b,
            "separate": f"{ws.nsets} sphgrav_forces_device calls, one per model (split-FP32)",
            "separate_fp64_calls_ms": ms_s64, "speedup_batched_vs_separate_fp64": ms_s64 / ms_b,
            "batched_fp64_ms": ms_b64, "speedup_f32split_vs_fp64_batched": ms_b64 / ms_b,
            "refined_rows": refined, "accuracy_vs_fp64": accuracy(res32, res64),
            "l2": "flushed before every timed call"}


def single_set_section(torch, ctx, timer, device, args, name):
    """A single-set benchmark workload other than the headline one (config1,
    config2): split-FP32 whole-call rate, its pair kernel's share of the
    FP32 peak probe, the FP64 kernel's rate and the accuracy against it."""
    ws = load_workload(name)
    X, outs = upload(torch, ws, device)

    def call(prec="f32split"):
        ctx.forces_device(ws.n, *X, *outs, nkernel=args.nkernel, precision=prec)

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    ctx.profile_enable(True)
    ctx.profile_read()
    ms = timer.run(call, 5)
    kern_ms, kern_n = ctx.profile_read()
    ctx.profile_enable(False)
    res32 = [o.cpu().numpy() for o in outs]
    refined = ctx.last_refine_rows()
    call("fp64")
    ms64 = timer.run(lambda: call("fp64"), 2)
    res64 = [o.cpu().numpy() for o in outs]
    pairs = ws.pairs
    kms = kern_ms / max(1, kern_n)
    return {"workload": ws.name, "n": ws.n, "pairs_per_step": pairs, "ms_per_step": ms,
            "value": pairs / (ms * 1e-3) / 1e9, "kernel_ms_per_launch": kms,
            "kernel_tflops": pairs * FLOPS_PER_PAIR / (kms * 1e-3) / 1e12,
            "fp64_ms_per_step": ms64, "fp64_value": pairs / (ms64 * 1e-3) / 1e9,
            "speedup_f32split_vs_fp64": ms64 / ms, "refined_rows": refined,
            "accuracy_vs_fp64": accuracy(res32, res64),
            "l2": "flushed before every timed step"}


def config5_section(torch, ctx, timer, stream, device, args):
    """The graph-captured sweep (config5): a CUDA graph of (seeded position
    kick, sigma = 1e-3 R, + batched gravity) replayed on device-resident
    state; time per replay and the accuracy at call 1 and at the last call
    against the FP64 kernel on the same kicked positions."""
    from starsmasher_b200 import Context
    ws = load_workload("config5")
    X, outs = upload(torch, ws, device)
    sigma, seed = 1e-3, 12345
    o64 = [torch.empty_like(o) for o in outs]

    def fp64_now():
        ctx.batch_forces_device(ws.offsets, *X, *o64, nkernel=args.nkernel, precision="fp64")
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in o64]

    with Context(device) as g:
        g.set_stream(stream.cuda_stream)
        g.batch_forces_device(ws.offsets, *X, *outs, nkernel=args.nkernel, precision="f32split")
        torch.cuda.synchronize()
        g.kick_reset(0)
        with g.capture() as cap:
            g.kick_device(ws.n, X[0], X[1], X[2], sigma, seed)
            g.batch_forces_device(ws.offsets, *X, *outs, nkernel=args.nkernel, precision="f32split")
        graph = cap.graph
        graph.launch(1)
        torch.cuda.synchronize()
        first = [o.cpu().numpy() for o in outs]
        acc1 = accuracy(first, fp64_now())
        ms = timer.run(lambda: graph.launch(1), args.graph_calls)
        calls = 1 + args.graph_calls
        last = [o.cpu().numpy() for o in outs]
        refined = g.last_refine_rows()
        graph.close()
    acc_last = accuracy(last, fp64_now())
    return {"workload": ws.name, "n": ws.n, "nsets": ws.nsets, "pairs_per_call": ws.pairs,
            "ms_per_call": ms, "value": ws.pairs / (ms * 1e-3) / 1e9, "calls_timed": args.graph_calls,
            "calls_total": calls, "kick_sigma": sigma,
            "graph": "kick + keys/sort/gather/tiles + pair kernel + merge + FP64 refine, one CUDA graph",
            "refined_rows_last_call": refined, "accuracy_call_1": acc1,
            f"accuracy_call_{calls}": acc_last, "l2": "flushed before every timed replay"}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    if args.phases:
        os.environ["SPHGRAV_B200_BUILD"] = "phases"
    from starsmasher_b200 import Context, api, launch_count, multirank

    # the multi-rank code path: several ranks, or one rank when forced
    dist_mode = world > 1 or args.parallel != "auto"
    if dist_mode:
        if "MASTER_ADDR" not in os.environ:  # one rank outside torchrun
            import socket
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                port = sk.getsockname()[1]
            os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                               "RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)

    # every rank loads the same model; the ranks divide its work
    ws = load_workload(args.workload)
    n = ws.n
    pairs = ws.pairs
    batched = ws.nsets > 1

    # one dedicated stream for the library, the collectives, the flush and the events
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    ctx = Context(device)
    ctx.set_stream(stream.cuda_stream)
    if args.variant >= 0:
        ctx.force_variant(args.precision, args.variant)
    if args.fp64_band is not None:
        ctx.set_fp64_band(args.fp64_band)
    if args.refine is not None:
        ctx.set_refine(args.refine)
    timer = Timer(torch, stream, device, args.l2_flush)

    X, outs = upload(torch, ws, device)
    W = torch.empty(ws.nsets, dtype=torch.float64, device=f"cuda:{device}")

    def gravity(precision):
        if batched:
            ctx.batch_forces_device(ws.offsets, *X, *outs, W=W, nkernel=args.nkernel,
                                    precision=precision)
        else:
            ctx.forces_device(n, *X, *outs, W=W, nkernel=args.nkernel, precision=precision)

    # ----------------------------------------------------- the step
    rowsplit = dist_mode and ((not batched and args.parallel != "setshard")
                              or args.parallel == "rowsplit")
    if not dist_mode:
        mode = "single GPU"

        def step(precision):
            gravity(precision)
    elif rowsplit:
        # the reference's gravity row split: this rank owns rows [lo, hi)
        lo, hi = multirank.gpu_row_range(n, world, rank)
        own = torch.stack([t[lo:hi] for t in X]).contiguous()
        split = {p: multirank.RowSplitStep(multirank.gpu_compute_device(ctx, args.nkernel, p), own, n)
                 for p in ("f32split", "fp64")}
        mode = f"row split x{world} (main.f:283-295): NCCL all-gather of sources and rows"

        def step(precision):
            split[precision]()
    else:
        shards = multirank.shard_sets(np.diff(ws.offsets), world)[rank]
        sub = [(int(ws.offsets[s]), int(ws.offsets[s + 1])) for s in shards]
        offs = np.concatenate([[0], np.cumsum([b - a for a, b in sub])]).astype(np.int32)
        Xs = [torch.cat([t[a:b] for a, b in sub]) if sub else t[:0] for t in X]
        outs_s = [torch.empty_like(t) for t in Xs[:4]]
        mode = f"set shard x{world}: whole models per rank, longest first"

        def step(precision):
            if sub:
                ctx.batch_forces_device(offs, *Xs, *outs_s, nkernel=args.nkernel,
                                        precision=precision)

    graph = None
    sigma, kick_seed = 1e-3, 12345

    def timed_step(precision):
        if graph is not None and precision == args.precision:
            graph.launch(1)
        else:
            step(precision)

    for _ in range(max(3, args.warmup)):
        step(args.precision)
    torch.cuda.synchronize()
    acc_first_call = None
    calls = 0
    if args.graph and not dist_mode:
        ctx.kick_reset(0)
        with ctx.capture() as cap:
            ctx.kick_device(n, X[0], X[1], X[2], sigma, kick_seed)
            gravity(args.precision)
        graph = cap.graph
        graph.launch(1)
        calls = 1
        if not args.no_fp64:
            with Context(device) as ctx64:
                ctx64.set_stream(stream.cuda_stream)
                o64 = [torch.empty_like(o) for o in outs]
                if batched:
                    ctx64.batch_forces_device(ws.offsets, *X, *o64, nkernel=args.nkernel,
                                              precision="fp64")
                else:
                    ctx64.forces_device(n, *X, *o64, nkernel=args.nkernel, precision="fp64")
                torch.cuda.synchronize()
                acc_first_call = accuracy([o.cpu().numpy() for o in outs],
                                          [o.cpu().numpy() for o in o64])
        for _ in range(max(3, args.warmup) - 1):
            graph.launch(1)
            calls += 1
        torch.cuda.synchronize()

    def barrier():
        if dist_mode:
            dist.barrier()

    # ------------------------------------------------------- timed region
    ctx.profile_enable(True)
    ctx.profile_read()
    clocks = Clocks(device)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = launch_count()
    ms_per_step = timer.run(lambda: timed_step(args.precision), args.steps)
    barrier()
    launches = launch_count() - l0
    clk = clocks.stop()
    kern_ms, kern_n = ctx.profile_read()
    ctx.profile_enable(False)
    if dist_mode:
        t = torch.tensor([ms_per_step], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    value = pairs / (ms_per_step * 1e-3) / 1e9
    refined = ctx.last_refine_rows() if not dist_mode else None
    res_f32 = [o.cpu().numpy() for o in outs] if not dist_mode else None
    graph_info = None
    if graph is not None:
        calls += args.steps
        graph_info = {"calls_timed": args.steps, "ms_per_call": ms_per_step,
                      "kick_sigma": sigma, "nodes": "kick + keys/sort/gather/tiles + pair kernel + merge + refine",
                      "calls_total": calls, "accuracy_call_1": acc_first_call,
                      "accuracy_last_call": f"accuracy_vs_fp64 (call {calls})"}
        graph.close()
        graph = None

    # ------------------------------------- batched vs one call per set
    batch_cmp = None
    if not dist_mode and batched and not args.no_separate:
        def separate(prec):
            for s in range(ws.nsets):
                a, b = int(ws.offsets[s]), int(ws.offsets[s + 1])
                ctx.forces_device(b - a, *(t[a:b] for t in X), *(o[a:b] for o in outs),
                                  nkernel=args.nkernel, precision=prec)
        separate(args.precision)
        torch.cuda.synchronize()
        sep_ms = timer.run(lambda: separate(args.precision), max(1, min(args.steps, 3)))
        separate("fp64")
        sep64_ms = timer.run(lambda: separate("fp64"), 1)
        batch_cmp = {"separate_calls_ms_per_step": sep_ms, "batched_ms_per_step": ms_per_step,
                     "speedup_batched_vs_separate": sep_ms / ms_per_step,
                     "separate": f"{ws.nsets} sphgrav_forces_device calls, one per set",
                     "separate_fp64_calls_ms_per_step": sep64_ms,
                     "speedup_batched_vs_separate_fp64": sep64_ms / ms_per_step}

    # --------------------------------------------- FP64 kernel and accuracy
    fp64 = None
    acc = None
    res64 = None
    if not dist_mode and not args.no_fp64:
        step("fp64")
        torch.cuda.synchronize()
        ms64 = timer.run(lambda: step("fp64"), 2)
        v64 = pairs / (ms64 * 1e-3) / 1e9
        res64 = [o.cpu().numpy() for o in outs]
        acc = accuracy(res_f32, res64)
        peak64 = max(ctx.fp64_peak_probe(100000) for _ in range(3))  # best of 3: clock dips
        ach64 = v64 * 1e9 * FLOPS_PER_PAIR / 1e12
        fp64 = {"value": v64, "unit": UNIT, "ms_per_step": ms64,
                "speedup_f32split_vs_fp64": value / v64,
                "roofline": {"bound": "fp64-fma", "achieved": ach64, "peak": peak64, "unit": "TFLOP/s",
                             "frac": ach64 / peak64, "flops_per_pair": FLOPS_PER_PAIR,
                             "time": "whole step (preparation included)",
                             "peak_source": "measured in-run: DFMA throughput probe on this GPU, best of 3",
                             # the kernel issues 18 FP64 instructions per far pair
                             # (its 1/r takes 5 after the rsqrt seed), so the
                             # FP64 pipe bounds it at peak/2 lanes/18 pairs
                             "fp64_instructions_per_far_pair": FP64_INSTR_PER_PAIR,
                             "instruction_bound": peak64 / 2 * 1e3 / FP64_INSTR_PER_PAIR,
                             "frac_of_instruction_bound":
                                 v64 / (peak64 / 2 * 1e3 / FP64_INSTR_PER_PAIR),
                             "instruction_bound_unit": UNIT}}

    # ------------------------------------- Barnes-Hut tree (approximate)
    tree = None
    thetas = [float(v) for v in args.tree_thetas.split(",") if v.strip()]
    if not dist_mode and not batched and thetas and res64 is not None:
        tree = {"what": "SPHGRAV_TREE: octree, quadrupole nodes, FP64 softened pairs; "
                        "approximate, error set by theta (not the direct-sum metric)",
                "time": "whole call, device arrays (build syncs once per 4 tree levels)",
                "direct_f32split_ms_per_step": ms_per_step}
        for th in thetas:
            ctx.set_theta(th)
            gravity("tree")
            torch.cuda.synchronize()
            res_t = [o.cpu().numpy() for o in outs]
            ngroups, nheavy = ctx.tree_stats()
            ms_t = timer.run(lambda: gravity("tree"), 3)
            tree[f"theta_{th:g}"] = {
                "ms_per_step": ms_t, "speedup_vs_f32split_direct": ms_per_step / ms_t,
                "speedup_vs_fp64_direct": fp64["ms_per_step"] / ms_t,
                "walking_groups": ngroups, "groups_direct_fp64": nheavy,
                "accuracy_vs_fp64": accuracy(res_t, res64)}
        ctx.set_theta(0.3)

    # ------------------------------------------------------------ roofline
    # best of 3 runs: a probe that lands on a clock or power dip would
    # understate the peak and overstate the fraction
    peak = max(ctx.fp32_peak_probe(200000) for _ in range(3))
    if kern_n == 0:
        # graph replays record no per-kernel events: time the pair kernel on
        # eager calls of the same workload instead
        ctx.profile_enable(True)
        ctx.profile_read()
        for _ in range(2):
            step(args.precision)
        kern_ms, kern_n = ctx.profile_read()
        ctx.profile_enable(False)
    kernel_ms = kern_ms / max(1, kern_n)
    kernel_pairs = pairs if world == 1 else pairs / world
    achieved = kernel_pairs * FLOPS_PER_PAIR / (kernel_ms * 1e-3) / 1e12
    # DRAM bytes of one pair-kernel launch on this workload, from a one-pass
    # ncu capture of this same command (profiles/traffic_*.json), if recorded
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"traffic_{args.precision}_{args.workload}.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")
    roofline = {"bound": "fp32-fma", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic,
                # 13 FMA-pipe lane-ops per far pair against 20 counted flops:
                # the kernel can reach at most 20 / 26 of the FMA peak
                "fma_lane_ops_per_pair": F32_LANE_OPS_PER_PAIR,
                "frac_cap": FLOPS_PER_PAIR / (2 * F32_LANE_OPS_PER_PAIR),
                "frac_of_cap": achieved / peak / (FLOPS_PER_PAIR / (2 * F32_LANE_OPS_PER_PAIR)),
                "kernel_ms_per_launch": kernel_ms, "flops_per_pair": FLOPS_PER_PAIR,
                "peak_source": "measured in-run: packed-FFMA throughput probe on this GPU, best of 3 "
                               "(MEASURED_PEAKS.json has no FP32 CUDA-core figure)",
                "time_share_kernel": kernel_ms / ms_per_step if ms_per_step else None}

    # ----------------------------------------------------------------- e2e
    e2e = None
    if not args.no_e2e:
        if rowsplit:
            # host arrays: this rank's rows in pinned memory, copied in every
            # step; the gathered result read back every step
            own_h = torch.stack([torch.as_tensor(a[lo:hi]) for a in
                                 (ws.x, ws.y, ws.z, ws.m, ws.range2)]).pin_memory()
            res_h = torch.empty((4, n), dtype=torch.float64).pin_memory()

            def e2e_step():
                own_d = own_h.to(f"cuda:{device}", non_blocking=True)
                src, res = split[args.precision](own_d)
                res_h.copy_(res, non_blocking=True)
                torch.cuda.current_stream().synchronize()
            how = "row split from host arrays (pinned H2D of own rows, D2H of all rows)"
            h2d, d2h = 5 * 8 * (hi - lo), 4 * 8 * n
        elif batched:
            def e2e_step():
                ctx.batch_forces(ws.offsets, ws.x, ws.y, ws.z, ws.m, ws.range2, args.nkernel,
                                 args.precision)
            how = "sphgrav_batch_forces (host arrays)"
            h2d, d2h = 5 * 8 * n, 4 * 8 * n
        else:
            api.gpu_init_dev(device, 0.3)
            api.set_legacy_precision(args.precision)
            gx, gy, gz, gp = (np.zeros(n) for _ in range(4))

            def e2e_step():
                api.firsthalf_grav_forces(n, 1, n, ws.x, ws.y, ws.z, ws.m, ws.range2, 1,
                                          args.nkernel)
                api.lasthalf_grav_forces(n, gx, gy, gz, gp)
            how = "firsthalf_grav_forces_/lasthalf_grav_forces_ (Fortran C-ABI, host arrays)"
            h2d, d2h = 5 * 8 * n, 4 * 8 * n
        if not dist_mode or rowsplit:
            e2e_step()
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            t_e2e = time.perf_counter() - t0
            if dist_mode:
                t = torch.tensor([t_e2e], dtype=torch.float64, device=f"cuda:{device}")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                t_e2e = float(t.item())
            e2e = {"value": pairs * args.steps / t_e2e / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "ms_per_step": t_e2e / args.steps * 1e3, "path": how}

    # -------------------------------- config4 / config5 sections (1 GPU)
    extras = {}
    if not dist_mode and args.workload == "config3" and not args.no_extras:
        extras["config4_batched"] = config4_section(torch, ctx, timer, device, args)
        extras["config5_graph_sweep"] = config5_section(torch, ctx, timer, stream, device, args)
        for name in ("config1", "config2"):
            extras[f"{name}_single_set"] = single_set_section(torch, ctx, timer, device, args, name)

    phases = None
    if args.phases and args.precision == "f32split":
        # untimed: the diagnostic build's per-phase cycle counters
        ctx.profile_enable(True)
        ctx.profile_read()
        ctx.phase_read()
        for _ in range(2):
            step(args.precision)
        ctx.profile_read()
        phases = phase_shares(ctx.phase_read())
        ctx.profile_enable(False)

    # -------------------------------------------------------- CPU baseline
    cpu = None
    if rank == 0 and not dist_mode and not args.no_cpu_baseline:
        cpu = cpu_baseline(ws, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.precision == "f32split" else "f64",
            "data": "synthetic: seeded polytropic star models (no public dataset)",
            "config": {"workload": ws.name, "n": n, "nsets": ws.nsets, "pairs_per_step": pairs,
                       "precision": args.precision, "nkernel": args.nkernel,
                       "fp64_band": args.fp64_band if args.fp64_band is not None else "library default",
                       "refine": args.refine if args.refine is not None else "library default",
                       "l2": ("flushed before every timed step (256 MB write)" if args.l2_flush == "write"
                              else "flushed before every timed step (512 MB read)"),
                       "parallelism": mode},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "fp64": fp64, "accuracy_vs_fp64": acc, "refined_rows": refined,
        }
        if batch_cmp:
            line["batch_vs_separate"] = batch_cmp
        if graph_info:
            line["graph_sweep"] = graph_info
        if tree:
            line["tree"] = tree
        if phases:
            line["phases"] = phases
        line.update(extras)
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist_mode:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
