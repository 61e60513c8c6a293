#!/usr/bin/env python
"""Benchmark of the B200 "cuda" backend for loop_tool.

Headline (one JSON line, `value`): the bandwidth-bound FP32 nests of the
reference's headline configuration, each a loop tree built with the lazy
frontend and run through the backend's Compiled::run entry point (C ABI):
  (i)   C = A + B over 2^28 elements
  (ii)  row softmax of x[8192, 4096] (max, subtract, exp, sum, divide)
  (iii) 2x2 stride-2 max-pool of X[64, 128, 112, 112]
one step = the three nests; value = HBM GB/s of algorithmic traffic (every
input element read once, every output element written once) over the step.

The same line carries the other configurations under "configs":
  c1  (A.to(m,k) * B.to(k,n)).sum(k), 128^3, FP32, checked against the
      reference CPU backend on the same IR
  c3  conv [32,64,56,56] * [128,64,3,3], stride 1, pad 1: FP32 CUDA cores,
      BF16 and split-BF16 tensor cores, error vs FP64 on sampled outputs
  c4  512 uneven matmuls (M, N, K log-uniform in [64, 4096], multiples of 16)
      in one graph-captured grouped launch (BF16, split-BF16, FP32), and a
      single 8192^3 matmul (tensor-pipe share of the measured BF16 peak)
  c5  serving: a seeded Poisson trace (50% matmul, 30% conv, 20% softmax) on
      the continuous-batching server vs the plain FP32 one-stream path

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
      [--serve-requests R] [--no-extras]

--impl reference times the reference's own CPU backend ("cpp": generated C
compiled by cc -O3, single-threaded as the reference is) on the host cores,
on a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")
BF16_DENSE_NOMINAL = 2250.0


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def read_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    return json.load(open(p)) if os.path.exists(p) else {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.path = index, None, None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [[x.strip() for x in line.split(",")] for line in open(self.path)]
        rows = [r for r in rows if len(r) >= 9]
        os.unlink(self.path)
        if not rows:
            return None
        num = lambda x: x.replace(".", "", 1).isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if num(rows[0][2]) else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def max_over_ranks(x, device=None):
    """The largest of a per-rank value (the slowest rank's time); x itself
    when no process group spans more than one rank."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_rank_step, steps, max_seconds, world):
    """Whole-job GB/s: every rank moves bytes_per_rank_step per step (weak
    scaling, replicas), over the slowest rank's time."""
    return world * bytes_per_rank_step * steps / max_seconds / 1e9


def dist_setup():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


# ------------------------------------------------------------- workloads
def nests(add_log2=28):
    """The three bandwidth nests, built with the lazy frontend."""
    import loop_tool_b200.lazy as lt
    import loop_tool_b200.nn as nn

    A, B = lt.Tensor(1 << add_log2), lt.Tensor(1 << add_log2)
    N = lt.Symbol("N")
    add = A.to(N) + B.to(N)
    X = lt.Tensor(8192, 4096)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    x = X.to(r, n)
    e = (x - x.max_reduce(n)).exp()
    softmax = e / e.sum(n)
    P = lt.Tensor(64, 128, 112, 112)
    b, c, h, w = (lt.Symbol(s) for s in "nchw")
    pool = nn.maxpool(P.to(b, c, h, w), [h, w], 2, 2)
    return [(f"add_2p{add_log2}", add.ir, 1.0), ("softmax_8192x4096", softmax.ir, 4.0),
            ("maxpool_64x128x112x112", pool.ir, 1.0)]


def mm_ir(M, K, N):
    import loop_tool_b200.lazy as lt

    A, B = lt.Tensor(M, K), lt.Tensor(K, N)
    m, k, n = lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
    return (A.to(m, k) * B.to(k, n)).sum(k).ir


def conv_ir(b=32):
    from loop_tool_b200.serve import _program

    return _program("conv", (b,)).ir


# --------------------------------------------------------- CPU reference
def reference_time(samples=None, cores=1):
    """Times the reference CPU backend ("cpp") on a bounded sample of each
    nest: the same loop trees at reduced size, scaled by bytes.  cores > 1
    runs that many single-threaded reference processes at once, each pinned
    to its own core (the reference backend has no threading of its own),
    and returns their aggregate GB/s."""
    samples = samples or [("add", [1 << 24]), ("softmax", [512, 4096]),
                          ("maxpool", [4, 128, 112, 112, 2, 2])]
    total_bytes = total_s = 0.0
    cpus = sorted(os.sched_getaffinity(0))[:cores]
    for prog, params in samples:
        with tempfile.TemporaryDirectory() as td:
            ir = subprocess.run([HARNESS, "ir", prog, *map(str, params)], capture_output=True,
                                text=True, check=True).stdout
            irf = os.path.join(td, "ir.txt")
            open(irf, "w").write(ir)
            sizes = json.loads(subprocess.run([HARNESS, "sizes", irf], capture_output=True,
                                              text=True, check=True).stdout)
            rng = np.random.default_rng(1)
            for i, n in enumerate(sizes["inputs"]):
                rng.standard_normal(n, dtype=np.float32).tofile(os.path.join(td, f"in{i}.f32"))
            # every process compiles and runs once, then waits at a gate
            # file so that all timed runs overlap
            gate = os.path.join(td, "go")
            procs, ods = [], []
            for cpu in cpus:
                od = os.path.join(td, f"out{cpu}")
                os.makedirs(od)
                ods.append(od)
                cmd = [HARNESS, "run", irf, "cpp", td, od, "3", gate]
                procs.append(subprocess.Popen(["taskset", "-c", str(cpu)] + cmd,
                                              stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                              text=True))
            t_end = time.time() + 300
            while time.time() < t_end and not all(
                    os.path.exists(os.path.join(od, "ready")) or pr.poll() is not None
                    for od, pr in zip(ods, procs)):
                time.sleep(0.01)
            open(gate, "w").close()
            secs = []
            for pr in procs:
                out, _ = pr.communicate()
                if pr.returncode != 0:  # no taskset: unpinned single run
                    out = subprocess.run([HARNESS, "run", irf, "cpp", td, td, "3"],
                                         capture_output=True, text=True, check=True).stdout
                secs.append(min(json.loads(out.strip().splitlines()[-1])["seconds"]))
            nbytes = 4 * (sum(sizes["inputs"]) + sum(sizes["outputs"]))
            rate = sum(nbytes / t for t in secs)  # aggregate bytes/s of the processes
            total_bytes += nbytes * len(secs)
            total_s += nbytes * len(secs) / rate
    desc = "; ".join(f"{p}{q}" for p, q in samples)
    return total_bytes / total_s / 1e9, desc, len(cpus)


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    if not os.path.exists(HARNESS):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU build absent (make -C oracle)"}))
        return
    cores = min(len(os.sched_getaffinity(0)), 64)
    for _ in range(args.warmup):
        reference_time(cores=cores)
    vals = []
    desc = ""
    for _ in range(args.steps):
        v, desc, cores = reference_time(cores=cores)
        vals.append(v)
    v = statistics.median(vals)
    print(json.dumps({
        "impl": "reference", "metric": "hbm_gbs_bandwidth_nests", "value": v, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
        "config": {"workload": "bandwidth nests: add 2^28, softmax 8192x4096, maxpool "
                               "64x128x112x112 (FP32)",
                   "parallelism": f"cpu, {cores} single-threaded reference processes, one "
                                  f"pinned per core"},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": "reference",
                         "sample": desc + f" per process, {cores} processes at once"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------- headline
def headline(args, world, rank, dev):
    import torch

    import loop_tool_b200 as ltb

    comps, bufs, bytes_per, schedules = [], [], [], {}
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    for name, ir, scale in nests():
        c = ltb.Compiled(ir)
        ins = [scale * torch.randn(n, device=dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
        outs = [torch.empty(n, device=dev) for n in c.io_sizes[c.n_inputs:]]
        comps.append((name, c))
        bufs.append(ins + outs)
        bytes_per.append(4 * sum(c.io_sizes))
        if args.tune:  # the autotuner picks each stage's schedule (untimed)
            schedules[name] = [ln.strip() for ln in c.tune(ins + outs, reps=5).splitlines()
                               if ln.startswith("  ")]
    stream = torch.cuda.current_stream()

    # the three nests are independent programs: each runs on its own stream,
    # so one nest's tail overlaps the next one's start
    nest_streams = [torch.cuda.Stream() for _ in comps]

    def concurrent_steps(k, start, end):
        start.record(stream)
        for ns in nest_streams:
            ns.wait_event(start)
        for _ in range(k):
            for ns, (_, c), b in zip(nest_streams, comps, bufs):
                c.run(b, sync=False, stream=ns.cuda_stream)
        for ns in nest_streams:
            done = torch.cuda.Event()
            done.record(ns)
            stream.wait_event(done)
        end.record(stream)

    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    concurrent_steps(max(args.warmup, 3), torch.cuda.Event(), torch.cuda.Event())
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")  # ncu --nvtx --nvtx-include timed/
    concurrent_steps(args.steps, t0, t1)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    clocks = sampler.stop()
    ms = max_over_ranks(t0.elapsed_time(t1), dev)
    # per-nest device times (roofline of each kernel) from a serial pass
    # per-nest kernel times for the roofline: each nest alone, launched
    # `steps` times back to back (steady state: a kernel's own L2 write-back
    # lands in its own launches, not in the next nest's)
    nest_ms = []
    for (_, c), b in zip(comps, bufs):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c.run(b, sync=False)
        e0.record(stream)
        for _ in range(args.steps):
            c.run(b, sync=False)
        e1.record(stream)
        e1.synchronize()
        nest_ms.append(e0.elapsed_time(e1) / args.steps)
    step_bytes = sum(bytes_per)
    value = whole_job_gbs(step_bytes, args.steps, ms / 1e3, world)

    # e2e: the same step through the C ABI with pinned host buffers; the
    # host->device copies of the inputs and device->host copies of the
    # outputs happen inside the timed region (the backend stages host
    # pointers through HBM)
    hbufs = []
    for (_, c), b in zip(comps, bufs):
        hb = [x.cpu().pin_memory() for x in b[:c.n_inputs]]
        hb += [torch.empty(n, pin_memory=True) for n in c.io_sizes[c.n_inputs:]]
        hbufs.append(hb)
    for (_, c), hb in zip(comps, hbufs):
        c.run(hb, sync=True)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e2e_steps = max(1, min(args.steps, 3))
    # device time from the first upload to the last download: each nest runs
    # on its own stream (asynchronous runs on pinned host buffers), so one
    # nest's downloads overlap another's uploads on the host link
    nest_streams = [torch.cuda.Stream() for _ in comps]
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for ns in nest_streams:
        ns.wait_event(s0)
    for _ in range(e2e_steps):
        for ns, (_, c), hb in zip(nest_streams, comps, hbufs):
            c.run(hb, sync=False, stream=ns.cuda_stream)
    for ns in nest_streams:
        done = torch.cuda.Event()
        done.record(ns)
        stream.wait_event(done)
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(s0.elapsed_time(s1) / 1e3 / e2e_steps, dev)
    link = host_link_gbs(dev)
    h2d = sum(4 * sum(c.io_sizes[:c.n_inputs]) for _, c in comps)
    d2h = sum(4 * sum(c.io_sizes[c.n_inputs:]) for _, c in comps)
    hbm_peak, _, peak_kind = load_peaks()
    dom = int(np.argmax(nest_ms))
    achieved = bytes_per[dom] / (nest_ms[dom] / 1e3) / 1e9
    return {
        "metric": "hbm_gbs_bandwidth_nests", "value": value, "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "bandwidth nests: add 2^28, softmax 8192x4096, maxpool "
                               "64x128x112x112 (FP32 lazy-frontend loop trees)",
                   "l2": "inputs larger than L2 (126 MB), no flush needed",
                   "issue": "each step's three independent nests on three streams; per-nest "
                            "times (roofline): each nest alone, launched `steps` times back "
                            "to back",
                   "schedules": "autotuned before warm-up" if args.tune else "heuristic",
                   "parallelism": f"replicas{world}"},
        "schedules": schedules,
        "nests_ms": {n: t for (n, _), t in zip(comps, nest_ms)},
        "nests_gbs": {n: b / (t / 1e3) / 1e9 for (n, _), b, t in zip(comps, bytes_per, nest_ms)},
        "nests_frac_of_hbm": {n: b / (t / 1e3) / 1e9 / hbm_peak
                              for (n, _), b, t in zip(comps, bytes_per, nest_ms)},
        "roofline": {"bound": "hbm", "kernel": comps[dom][0], "achieved": achieved,
                     "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": read_traffic().get(comps[dom][0])},
        "e2e": {"value": whole_job_gbs(step_bytes, 1, e2e_s, world), "unit": "GB/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "host_link_gbs": link},
        "gpu_launches": sum(c.int_property("launches") for _, c in comps) * args.steps,
        "clocks": clocks,
    }


def host_link_gbs(dev, nbytes=256 << 20, reps=3):
    """Plain pinned-memory copy bandwidth of this GPU's host link (GB/s per
    direction, best of reps), the ceiling the e2e figure is read against."""
    import torch

    h = torch.empty(nbytes // 4, pin_memory=True)
    d = torch.empty(nbytes // 4, device=dev)
    out = {}
    for name, fn in (("h2d", lambda: d.copy_(h, non_blocking=True)),
                     ("d2h", lambda: h.copy_(d, non_blocking=True))):
        fn()
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            best = max(best, nbytes / (a.elapsed_time(b) / 1e3) / 1e9)
        out[name] = best
    return out


def timed(fn, reps, stream=None):
    import torch

    stream = stream or torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


# ----------------------------------------------------------------- c1
def extra_c1(dev):
    import torch

    import loop_tool_b200 as ltb

    ir = mm_ir(128, 128, 128)
    rng = np.random.default_rng(101)
    a = rng.standard_normal(128 * 128).astype(np.float32)
    b = np.random.default_rng(102).standard_normal(128 * 128).astype(np.float32)
    out = {"workload": "(A.to(m,k) * B.to(k,n)).sum(k), 128^3 FP32, lazy frontend"}
    A, B = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    for prec in ("fp32", "bf16x3"):
        c = ltb.Compiled(ir, precision=prec)
        C = torch.empty(128 * 128, device=dev)
        us = timed(lambda: c.run([A, B, C], sync=False), 200) * 1e3
        # device time per call: the same run captured once and replayed (no
        # Python / ABI overhead between launches)
        cap = c.capture([A, B, C])
        graph_us = timed(lambda: cap.run(sync=False), 200) * 1e3
        del cap
        ch = np.empty(128 * 128, np.float32)
        w0 = time.perf_counter()
        for _ in range(50):
            c([a, b, ch])
        e2e_us = (time.perf_counter() - w0) / 50 * 1e6
        res = {"device_us_per_call": us, "gflops": 2 * 128 ** 3 / (us * 1e-6) / 1e9,
               "graph_replay_us_per_call": graph_us,
               "gflops_graph_replay": 2 * 128 ** 3 / (graph_us * 1e-6) / 1e9,
               "e2e_us_per_call_host_buffers": e2e_us}
        # checked against the reference CPU backend on the same IR
        if os.path.exists(HARNESS):
            with tempfile.TemporaryDirectory() as td:
                open(os.path.join(td, "ir.txt"), "w").write(ir)
                a.tofile(os.path.join(td, "in0.f32"))
                b.tofile(os.path.join(td, "in1.f32"))
                subprocess.run([HARNESS, "run", os.path.join(td, "ir.txt"), "cpp", td, td],
                               check=True, capture_output=True)
                ref = np.fromfile(os.path.join(td, "out0.f32"), np.float32)
            res["max_abs_diff_vs_reference_cpp"] = float(np.abs(ch - ref).max())
        exact = a.reshape(128, 128).astype(np.float64) @ b.reshape(128, 128).astype(np.float64)
        res["normwise_err_vs_fp64"] = float(np.linalg.norm(ch.reshape(128, 128) - exact) /
                                            np.linalg.norm(exact))
        out[prec] = res
    return out


# ----------------------------------------------------------------- c3
def extra_c3(dev):
    import torch

    import loop_tool_b200 as ltb

    ir = conv_ir(32)
    flops = 2.0 * 32 * 128 * 56 * 56 * 64 * 9
    x = torch.from_numpy(np.random.default_rng(301).standard_normal(32 * 64 * 56 * 56)
                         .astype(np.float32)).to(dev)
    bound = math.sqrt(6.0 / 576)
    w = torch.from_numpy(np.random.default_rng(302).uniform(-bound, bound, 128 * 64 * 9)
                         .astype(np.float32)).to(dev)
    xs = x.cpu().numpy().reshape(32, 64, 56, 56).astype(np.float64)
    ws = w.cpu().numpy().reshape(128, 64, 3, 3).astype(np.float64)
    xp = np.pad(xs, ((0, 0), (0, 0), (1, 1), (1, 1)))
    rng = np.random.default_rng(7)
    pts = rng.integers(0, [32, 56, 56, 128], size=(512, 4))
    exact = np.array([(xp[n, :, h:h + 3, wo:wo + 3] * ws[co]).sum() for n, h, wo, co in pts])
    out = {"workload": "conv [32,64,56,56]*[128,64,3,3] s1 p1 (output [n,ho,wo,co])",
           "gflop": flops / 1e9}
    for prec in ("fp32", "bf16", "bf16x3"):
        c = ltb.Compiled(ir, precision=prec)
        y = torch.empty(c.io_sizes[-1], device=dev)
        schedule = c.tune([x, w, y], reps=3).strip().splitlines()
        ms = timed(lambda: c.run([x, w, y], sync=False), 5)
        got = y.cpu().numpy().reshape(32, 56, 56, 128)[pts[:, 0], pts[:, 1], pts[:, 2], pts[:, 3]]
        out[prec] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                     "normwise_err_vs_fp64_sampled": float(np.linalg.norm(got - exact) /
                                                           np.linalg.norm(exact)),
                     "schedule": [ln.strip() for ln in schedule if ln.startswith("  ")]}
        if prec != "fp32":  # im2col packing vs tensor-core time
            b1 = ltb.Batch([(c, [x, w, y])])
            b1.run_timed()
            out[prec]["pack_ms"], out[prec]["gemm_ms"] = b1.run_timed()
            del b1
    return out


# ----------------------------------------------------------------- c4
def extra_c4(dev):
    import torch

    import loop_tool_b200 as ltb

    _, bf16_peak, _ = load_peaks()
    rng = np.random.default_rng(401)
    v = np.exp(rng.uniform(math.log(64), math.log(4096), size=(512, 3)))
    sizes = [tuple(int(max(16, 16 * round(x / 16))) for x in row) for row in v]
    irs = [mm_ir(M, K, N) for M, N, K in sizes]
    g = torch.Generator(device=dev).manual_seed(402)
    bufs = []
    for M, N, K in sizes:
        bufs.append([torch.randn(M * K, device=dev, generator=g) / math.sqrt(K),
                     torch.randn(K * N, device=dev, generator=g),
                     torch.empty(M * N, device=dev)])
    flops = sum(2.0 * M * N * K for M, N, K in sizes)
    out = {"workload": "512 matmuls, M,N,K log-uniform [64,4096] x16, one grouped launch",
           "tflop": flops / 1e12}
    st = torch.cuda.Stream()
    for prec in ("bf16", "bf16x3", "fp32"):
        members = [(ltb.Compiled(ir, precision=prec), b) for ir, b in zip(irs, bufs)]
        tiles = "cuda cores (128 x 128)"
        if prec == "fp32":
            batch = ltb.Batch(members, capture_stream=st.cuda_stream)
        else:  # tile widths chosen by the autotuner on the grouped launch
            batch, best, tiles = ltb.tune_batch(members, capture_stream=st.cuda_stream)
        with torch.cuda.stream(st):
            ms = timed(lambda: batch.run(sync=False, stream=st.cuda_stream),
                       3 if prec != "fp32" else 1, stream=st)
            pack_ms, gemm_ms = batch.run_timed(stream=st.cuda_stream)
        # sampled FP64 check of a few problems
        errs = []
        for i in (0, 100, 257, 511):
            M, N, K = sizes[i]
            a = bufs[i][0].cpu().numpy().reshape(M, K).astype(np.float64)
            bb = bufs[i][1].cpu().numpy().reshape(K, N).astype(np.float64)
            ex = a @ bb
            errs.append(float(np.linalg.norm(bufs[i][2].cpu().numpy().reshape(M, N) - ex) /
                              np.linalg.norm(ex)))
        out[prec] = {"graph_replay_ms": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                     "pack_ms": pack_ms, "gemm_ms": gemm_ms,
                     "gemm_tflops": flops / (gemm_ms * 1e-3) / 1e12,
                     "launches_per_replay": batch.int_property("launches"),
                     "tiles": tiles,
                     "tiles_128_256": [batch.int_property("tiles_128"),
                                       batch.int_property("tiles_256")],
                     "max_normwise_err_vs_fp64_sampled": max(errs)}
        del batch, members
    del bufs
    torch.cuda.empty_cache()
    n = 8192
    A = torch.randn(n * n, device=dev, generator=g)
    B = torch.randn(n * n, device=dev, generator=g)
    C = torch.empty(n * n, device=dev)
    ir = mm_ir(n, n, n)
    big = {"workload": "8192^3 matmul"}
    for prec in ("bf16", "bf16x3"):
        c1 = ltb.Compiled(ir, precision=prec)
        b1, _, sched = ltb.tune_batch([(c1, [A, B, C])], reps=2)
        b1.run_timed()
        pack_ms, gemm_ms = b1.run_timed()
        products = {"bf16": 1, "bf16x3": 3}[prec]
        big[prec] = {"total_ms": pack_ms + gemm_ms, "pack_ms": pack_ms, "gemm_ms": gemm_ms,
                     "tile_variant": c1.schedule(0)[2],
                     "pack_schedule": [b1.int_property("pack_chunk"),
                                       b1.int_property("pack_cta_per_sm")],
                     "tflops_total": 2 * n ** 3 / ((pack_ms + gemm_ms) * 1e-3) / 1e12,
                     "tensor_tflops_gemm": products * 2 * n ** 3 / (gemm_ms * 1e-3) / 1e12,
                     "frac_of_measured_bf16_peak": products * 2 * n ** 3 / (gemm_ms * 1e-3) /
                     1e12 / bf16_peak}
        del b1
    out["mm_8192"] = big
    return out


# ----------------------------------------------------------------- c5
def extra_c5(dev, n_requests, rates):
    """Each server configuration compiles the trace's distinct programs once
    (untimed), reserves its slot workspaces, then serves the trace at every
    arrival rate."""
    from loop_tool_b200.serve import Server, make_trace

    out = {"workload": f"{n_requests} requests, Poisson arrivals, 50% matmul (c4 shapes), "
                       f"30% conv (batch U[1,64]), 20% softmax (rows U[1,8192] x 4096)",
           "kernel_cache": "warm (every distinct program compiled before serving)",
           "workspaces": "reserved per slot before serving"}
    configs = [("b200_bf16x3_8slots", dict(slots=8, precision="bf16x3")),
               ("plain_fp32_1slot", dict(slots=1, precision="fp32"))]
    rows = {f"rate_{int(rate)}": {} for rate in rates}
    for name, kw in configs:
        srv = Server(hbm_budget=24 << 30, **kw)
        warm = make_trace(n_requests, rate=1e9, seed=501)
        w0 = time.perf_counter()
        for r in warm:  # populate the kernel cache (one compile per distinct program)
            srv.bytes_of(r)
        srv.reserve(warm)  # slot workspaces sized before the clock starts
        warm_s = time.perf_counter() - w0
        for rate in rates:
            stats, _ = srv.serve(make_trace(n_requests, rate=rate, seed=501))
            row = {k: stats[k] for k in ("req_per_s", "p50_ms", "p99_ms", "mean_ms",
                                         "peak_inflight", "compiles")}
            row["compile_s"] = warm_s
            rows[f"rate_{int(rate)}"][name] = row
        del srv
    out.update(rows)
    return out


# ------------------------------------------------------- profiling cases
NCU_CASES = ("add", "softmax", "maxpool", "mm_bf16", "mm_bf16x3", "mm_fp32", "conv_bf16",
             "conv_fp32", "batch_bf16", "mm_bf16_batch")


def ncu_case(name, reps, tune=True, schedules=None):
    """One workload at a profiling size (inputs above L2, about 1 GB on the
    device), autotuned as in the benchmark, then run `reps` times inside the
    NVTX range "profile" (capture with ncu --nvtx --nvtx-include profile/).
    With `schedules` (a file path): if the file exists its schedules are
    loaded and nothing is tuned, else the tuned schedules are written there,
    so a capture under ncu runs what the plain run before it chose."""
    import torch

    import loop_tool_b200 as ltb

    if schedules and os.path.exists(schedules):
        ltb.tune_load(schedules)
        tune = False

    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(9)
    opts = {}
    if name in ("add", "softmax", "maxpool"):
        ir = {n.split("_")[0]: t for n, t, _ in nests(add_log2=26)}[name]
    elif name == "mm_bf16_batch":  # 8192^3 through the grouped (batch) launch path
        n = 8192
        c = ltb.Compiled(mm_ir(n, n, n), precision="bf16")
        bufs = [torch.randn(n * n, device=dev, generator=g) for _ in range(2)]
        bufs.append(torch.empty(n * n, device=dev))
        if tune:
            c.tune(bufs, reps=2)
            if schedules:
                ltb.tune_save(schedules)
        b = ltb.Batch([(c, bufs)])
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("profile")
        for _ in range(reps):
            b.run(sync=False)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        return
    elif name.startswith("mm_"):
        ir, opts = mm_ir(8192, 8192, 8192), {"precision": name[3:]}
    elif name.startswith("conv_"):
        ir, opts = conv_ir(32), {"precision": name[5:]}
    else:
        rng = np.random.default_rng(401)
        v = np.exp(rng.uniform(math.log(64), math.log(4096), size=(128, 3)))
        members = []
        for row in v:
            M, N, K = (int(max(16, 16 * round(x / 16))) for x in row)
            c = ltb.Compiled(mm_ir(M, K, N), precision="bf16")
            members.append((c, [torch.randn(M * K, device=dev, generator=g),
                                torch.randn(K * N, device=dev, generator=g),
                                torch.empty(M * N, device=dev)]))
        if tune:
            b, _, _ = ltb.tune_batch(members)
            if schedules:
                ltb.tune_save(schedules)
        else:
            b = ltb.Batch(members)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("profile")
        for _ in range(reps):
            b.run(sync=False)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        return
    c = ltb.Compiled(ir, **opts)
    bufs = [torch.randn(n, device=dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
    bufs += [torch.empty(n, device=dev) for n in c.io_sizes[c.n_inputs:]]
    if tune:
        print(c.tune(bufs, reps=3))
        if schedules:
            ltb.tune_save(schedules)
    print(c.code.splitlines()[-1] if c.code else "")
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("profile")
    for _ in range(reps):
        c.run(bufs, sync=False)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep the heuristic schedules (no autotuning before warm-up)")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-rates", default="1000,4000")
    ap.add_argument("--ncu-case", choices=NCU_CASES,
                    help="run one workload at a profiling size and exit")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--schedules",
                    help="with --ncu-case: schedule file written by a tuning run and loaded "
                         "(no tuning) by a later run, e.g. the same case under ncu")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu_case:
        return ncu_case(args.ncu_case, args.reps, args.tune, args.schedules)

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.init()
    line = headline(args, world, rank, dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and os.path.exists(HARNESS):
        try:
            v, desc, _ = reference_time(cores=1)
            cpu = {"value": v, "unit": "GB/s", "cores": 1, "kind": "reference", "sample": desc}
        except Exception as e:  # reported, never fatal to the GPU number
            cpu = {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"}
    line["cpu_baseline"] = cpu
    if rank == 0 and world == 1 and not args.no_extras:
        configs = {}
        for key, fn in (("c1_mm128", lambda: extra_c1(dev)), ("c3_conv", lambda: extra_c3(dev)),
                        ("c4_batched", lambda: extra_c4(dev)),
                        ("c5_serving", lambda: extra_c5(
                            dev, args.serve_requests,
                            [float(r) for r in args.serve_rates.split(",")]))):
            try:
                configs[key] = fn()
            except Exception as e:  # one failing extra must not hide the headline
                configs[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
        line["configs"] = configs
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
