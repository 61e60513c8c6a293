#!/usr/bin/env python
"""Benchmark of the B200 "cuda" backend for loop_tool.

Headline (one JSON line, `value`): the bandwidth-bound FP32 nests of the
reference's headline configuration, each the loop tree the reference's lazy
frontend emits (tests/golden/ir/) run through the backend's Compiled::run
entry point (C ABI):
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
# Loop trees the reference's own lazy frontend emitted for these
# configurations (tests/golden/ir/, written by the oracle harness `ir` mode:
# serialize() of the reference's IR), run here as the text the drop-in
# "cuda" backend receives.
GOLDEN_IR = os.path.join(ROOT, "tests", "golden", "ir")


def reference_ir(name, sizes=None):
    """tests/golden/ir/<name>.txt with the loop sizes of some vars replaced
    (sizes: {var id: size}); only for trees whose sizes live in their loop
    orders alone (pointwise maps, matmuls)."""
    text = open(os.path.join(GOLDEN_IR, name + ".txt")).read()
    if not sizes:
        return text
    lines = []
    for ln in text.splitlines():
        if ln.startswith("n:"):
            f = ln.split(":")
            ents = []
            for e in f[7].split(","):
                if e:
                    v, sz, tail = (int(x) for x in e.split(";"))
                    e = f"{v};{sizes.get(v, sz)};{tail}"
                ents.append(e)
            f[7] = ",".join(ents)
            ln = ":".join(f)
        lines.append(ln)
    return "\n".join(lines) + "\n"


def nests(add_log2=28):
    """The three bandwidth nests as the reference lazy frontend emits them:
    (name, IR text, input scale)."""
    add = reference_ir("add_2p28", None if add_log2 == 28 else {0: 1 << add_log2})
    return [(f"add_2p{add_log2}", add, 1.0),
            ("softmax_8192x4096", reference_ir("softmax_8192x4096"), 4.0),
            ("maxpool_64x128x112x112", reference_ir("maxpool_64x128x112x112"), 1.0)]


def mm_ir(M, K, N):
    """(A.to(m,k) * B.to(k,n)).sum(k): the reference's 128^3 tree resized
    (vars m = 0, k = 1, n = 2)."""
    return reference_ir("mm_128", {0: M, 1: K, 2: N})


def conv_ir(b=32):
    """nn.pad + nn.conv of [b,64,56,56] * [128,64,3,3]: the reference's own
    tree for b = 32; other batches (profiling cases) through the serving
    loop's program builder."""
    if b == 32:
        return reference_ir("conv_32x64x56x56_co128")
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

    comps, sets, bytes_per, schedules = [], [], [], {}
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    for name, ir, scale in nests():
        c = ltb.Compiled(ir)
        # two buffer sets per nest, used in turn: consecutive launches of a
        # nest never find their inputs or dirty outputs in L2
        rot = []
        for _ in range(2):
            ins = [scale * torch.randn(n, device=dev, generator=g)
                   for n in c.io_sizes[:c.n_inputs]]
            outs = [torch.empty(n, device=dev) for n in c.io_sizes[c.n_inputs:]]
            rot.append(ins + outs)
        comps.append((name, c))
        sets.append(rot)
        bytes_per.append(4 * sum(c.io_sizes))
        if args.tune:  # the autotuner picks each stage's schedule (untimed)
            schedules[name] = [ln.strip() for ln in c.tune(rot[0], reps=5).splitlines()
                               if ln.startswith("  ")]
    bufs = [rot[0] for rot in sets]
    stream = torch.cuda.current_stream()

    # the three nests are independent programs: each runs on its own stream,
    # so one nest's tail overlaps the next one's start
    nest_streams = [torch.cuda.Stream() for _ in comps]

    def concurrent_steps(k, start, end):
        start.record(stream)
        for ns in nest_streams:
            ns.wait_event(start)
        for it in range(k):
            for ns, (_, c), rot in zip(nest_streams, comps, sets):
                c.run(rot[it % 2], sync=False, stream=ns.cuda_stream)
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
    for (_, c), rot in zip(comps, sets):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c.run(rot[1], sync=False)
        e0.record(stream)
        for it in range(args.steps):
            c.run(rot[it % 2], sync=False)
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
    e2e_steps = max(1, min(args.steps, 10))
    # device time from the first upload to the last download: each nest runs
    # on its own stream (asynchronous runs on pinned host buffers), so one
    # nest's downloads overlap another's uploads on the host link
    nest_streams = [torch.cuda.Stream() for _ in comps]

    def e2e_pass(s0, s1):
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

    # untimed passes of the same pattern first (as many as the warm-up
    # steps): the staging blocks of steps in flight on three streams at once
    # are reserved by the stream-ordered pool there, not mapped inside the
    # timed pass
    for _ in range(max(1, args.warmup)):
        e2e_pass(torch.cuda.Event(), torch.cuda.Event())
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_pass(s0, s1)
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
                               "64x128x112x112 (FP32 loop trees emitted by the reference's lazy "
                               "frontend)",
                   "l2": "two buffer sets per nest used in turn (each set's inputs and "
                         "outputs exceed L2, 126 MB): no launch finds its data in L2",
                   "issue": "each step's three independent nests on three streams; per-nest "
                            "times (roofline): each nest alone, launched `steps` times back "
                            "to back",
                   "schedules": "autotuned before warm-up" if args.tune else "heuristic",
                   "parallelism": f"replicas{world}"},
        "schedules": schedules,
        "nests_ms": {n: t for (n, _), t in zip(comps, nest_ms)},
        "nests_bytes": {n: b for (n, _), b in zip(comps, bytes_per)},
        "nests_gbs": {n: b / (t / 1e3) / 1e9 for (n, _), b, t in zip(comps, bytes_per, nest_ms)},
        "nests_frac_of_hbm": {n: b / (t / 1e3) / 1e9 / hbm_peak
                              for (n, _), b, t in zip(comps, bytes_per, nest_ms)},
        "roofline": {"bound": "hbm", "kernel": comps[dom][0], "achieved": achieved,
                     "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": read_traffic().get(comps[dom][0])},
        "e2e": {"value": whole_job_gbs(step_bytes, 1, e2e_s, world), "unit": "GB/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "host_link_gbs": link,
                # the step's algorithmic bytes over the least time its copies
                # need on this link (each direction alone, and both at once)
                "link_bound_gbs": world * step_bytes / max(h2d / link["h2d"], d2h / link["d2h"],
                                                           (h2d + d2h) / link["both"])},
        "gpu_launches": sum(c.int_property("launches") for _, c in comps) * args.steps,
        "clocks": clocks,
    }


def reference_frontend(nest_bytes):
    """The drop-in path end to end: the reference's own lazy frontend
    (TensorImpl::data, lazy.h:219-260: output allocated on the default
    hardware, compile on the first call, Compiled::run with sync, result
    read on the host) with the plugin registered as its "cuda" backend and
    hardware, timed per call by the oracle harness (`lazytime`).  Buffers
    are the hardware's: managed memory (the reference CudaGPUHardware's
    kind, the default) or pinned host memory (LOOP_TOOL_B200_HOST_MEMORY).
    nest_bytes: {nest name: algorithmic bytes per call}."""
    plugin = os.path.join(ROOT, "oracle", "_ref", "libloop_tool_cuda_b200.so")
    if not (os.path.exists(HARNESS) and os.path.exists(plugin)):
        return {"unavailable": "reference CPU build or plugin absent (make -C oracle all plugin)"}
    progs = [("add_2p28", "add", [1 << 28], 3), ("softmax_8192x4096", "softmax", [8192, 4096], 5),
             ("maxpool_64x128x112x112", "maxpool", [64, 128, 112, 112, 2, 2], 5)]
    out = {"path": "reference lazy::Tensor -> Backend \"cuda\" (plugin) -> C ABI, per call: "
                   "output allocation, run with sync, host read"}

    def lazytime(env, reps, prog, params):
        r = subprocess.run([HARNESS, "lazytime", str(reps), prog, *map(str, params)], env=env,
                           capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-300:])
        return statistics.median(json.loads(r.stdout.strip().splitlines()[-1])["seconds"])

    for mem in ("managed", "pinned"):
        env = dict(os.environ, LT_PLUGIN=plugin)
        if mem == "pinned":
            env["LOOP_TOOL_B200_HOST_MEMORY"] = "pinned"
        try:
            per = {name: lazytime(env, reps, prog, params) for name, prog, params, reps in progs}
            c1 = lazytime(env, 200, "mm", [128, 128, 128])
        except Exception as e:  # reported, not fatal for the headline
            out[mem] = {"error": str(e)}
            continue
        total_b = sum(nest_bytes[n] for n in per)
        out[mem] = {"gbs_bandwidth_nests": total_b / sum(per.values()) / 1e9,
                    "ms_per_call": {n: t * 1e3 for n, t in per.items()},
                    "gbs_per_nest": {n: nest_bytes[n] / t / 1e9 for n, t in per.items()},
                    "c1_mm128_us_per_call": c1 * 1e6}
    return out


def host_link_gbs(dev, nbytes=256 << 20, reps=3):
    """Plain pinned-memory copy bandwidth of this GPU's host link (GB/s, best
    of reps): each direction alone ("h2d", "d2h") and both at once on two
    streams ("both", the two directions' bytes together), the ceilings the
    e2e figure is read against."""
    import torch

    h = torch.empty(nbytes // 4, pin_memory=True)
    d = torch.empty(nbytes // 4, device=dev)
    h2 = torch.empty(nbytes // 4, pin_memory=True)
    d2 = torch.empty(nbytes // 4, device=dev)
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()

    def both():
        cur = torch.cuda.current_stream()
        s_up.wait_stream(cur)
        s_down.wait_stream(cur)
        with torch.cuda.stream(s_up):
            d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_down):
            h2.copy_(d2, non_blocking=True)
        cur.wait_stream(s_up)
        cur.wait_stream(s_down)

    out = {}
    for name, fn, moved in (("h2d", lambda: d.copy_(h, non_blocking=True), nbytes),
                            ("d2h", lambda: h.copy_(d, non_blocking=True), nbytes),
                            ("both", both, 2 * nbytes)):
        fn()
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            best = max(best, moved / (a.elapsed_time(b) / 1e3) / 1e9)
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


def elementwise_report(got, ref32, exact):
    """Accuracy of `got` entry by entry against the FP64 value `exact`, next
    to the reference's own FP32 result `ref32` of the same entries: the
    normwise error, the largest elementwise relative error, the entries
    whose error exceeds max(1e-5 |e|, the reference's own error there) (the
    parity bar of the tests), and whether `got` equals the reference bit
    for bit."""
    got = np.asarray(got, np.float64).ravel()
    ref32 = np.asarray(ref32, np.float64).ravel()
    exact = np.asarray(exact, np.float64).ravel()
    err = np.abs(got - exact)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(exact != 0, err / np.abs(exact), np.where(err == 0, 0.0, np.inf))
    tol = np.maximum(1e-5 * np.abs(exact), np.abs(ref32 - exact) * (1 + 1e-6))
    return {"normwise_rel_err_vs_fp64": float(np.linalg.norm(got - exact) /
                                              max(np.linalg.norm(exact), 1e-300)),
            "max_elementwise_rel_err_vs_fp64": float(rel.max()) if rel.size else 0.0,
            "entries_over_tolerance": int((err > tol).sum()), "entries": int(err.size),
            "bit_exact_with_reference": bool(np.array_equal(
                got.astype(np.float32).view(np.uint32), ref32.astype(np.float32).view(np.uint32)))}


def sequential_fp32_rows(a, b):
    """The reference's FP32 contraction of rows of A with B: acc = acc + a*b
    in ascending k, each multiply and add rounded to FP32 (the C path,
    cpp.cpp:172-270, compiled without contraction)."""
    acc = np.zeros((a.shape[0], b.shape[1]), np.float32)
    for k in range(a.shape[1]):
        acc = acc + np.outer(a[:, k], b[k]).astype(np.float32)
    return acc


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
    ref = None
    if os.path.exists(HARNESS):  # the reference CPU backend on the same IR
        with tempfile.TemporaryDirectory() as td:
            open(os.path.join(td, "ir.txt"), "w").write(ir)
            a.tofile(os.path.join(td, "in0.f32"))
            b.tofile(os.path.join(td, "in1.f32"))
            subprocess.run([HARNESS, "run", os.path.join(td, "ir.txt"), "cpp", td, td],
                           check=True, capture_output=True)
            ref = np.fromfile(os.path.join(td, "out0.f32"), np.float32)
    exact = a.reshape(128, 128).astype(np.float64) @ b.reshape(128, 128).astype(np.float64)
    for prec in ("fp32", "bf16x3", "bf16x6"):
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
        # checked against the reference CPU backend on the same IR and FP64
        if ref is not None:
            res["max_abs_diff_vs_reference_cpp"] = float(np.abs(ch - ref).max())
            res.update(elementwise_report(ch, ref, exact))
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
    # the reference's FP32 value of the sampled outputs: products rounded to
    # FP32 and added in its fold order (c, kh, kw), the conv node's loop order
    x32 = np.pad(x.cpu().numpy().reshape(32, 64, 56, 56), ((0, 0), (0, 0), (1, 1), (1, 1)))
    w32 = w.cpu().numpy().reshape(128, 64, 3, 3)
    terms = np.stack([(x32[n, :, h:h + 3, wo:wo + 3] * w32[co]).ravel()
                      for n, h, wo, co in pts]).astype(np.float32)
    ref32 = np.zeros(len(pts), np.float32)
    for t in range(terms.shape[1]):
        ref32 = ref32 + terms[:, t]
    out = {"workload": "conv [32,64,56,56]*[128,64,3,3] s1 p1 (output [n,ho,wo,co])",
           "gflop": flops / 1e9}
    for prec in ("fp32", "bf16", "bf16x3", "bf16x6"):
        c = ltb.Compiled(ir, precision=prec)
        y = torch.empty(c.io_sizes[-1], device=dev)
        schedule = c.tune([x, w, y], reps=3).strip().splitlines()
        api_ms = timed(lambda: c.run([x, w, y], sync=False), 5)
        # device time: the run's launches captured once and replayed (back
        # to back API calls can leave the GPU idle between runs)
        cap = c.capture([x, w, y])
        ms = timed(lambda: cap.run(sync=False), 20)
        del cap
        got = y.cpu().numpy().reshape(32, 56, 56, 128)[pts[:, 0], pts[:, 1], pts[:, 2], pts[:, 3]]
        out[prec] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12, "api_call_ms": api_ms,
                     "sampled_entries": elementwise_report(got, ref32, exact),
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
    # every member's first 8 rows: FP64 and the reference's FP32 value
    row_refs = []
    for (M, N, K), b in zip(sizes, bufs):
        a8 = b[0][:8 * K].cpu().numpy().reshape(8, K)
        bm = b[1].cpu().numpy().reshape(K, N)
        row_refs.append((a8.astype(np.float64) @ bm.astype(np.float64), sequential_fp32_rows(a8, bm)))
    for prec in ("bf16", "bf16x3", "bf16x6", "fp32"):
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
        # every member's first 8 rows against FP64 and the reference's FP32
        reps_ = [elementwise_report(b[2][:8 * N].cpu().numpy(), r32, ex)
                 for (M, N, K), b, (ex, r32) in zip(sizes, bufs, row_refs)]
        errs = [r["normwise_rel_err_vs_fp64"] for r in reps_]
        out[prec] = {"graph_replay_ms": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                     "pack_ms": pack_ms, "gemm_ms": gemm_ms,
                     "gemm_tflops": flops / (gemm_ms * 1e-3) / 1e12,
                     "launches_per_replay": batch.int_property("launches"),
                     "tiles": tiles,
                     "tiles_128_256_pair": [batch.int_property("tiles_128"),
                                            batch.int_property("tiles_256"),
                                            batch.int_property("tiles_pair")],
                     "max_normwise_err_vs_fp64_sampled": max(errs),
                     "rows_checked": "first 8 rows of all 512 members",
                     "max_elementwise_rel_err_vs_fp64": max(
                         r["max_elementwise_rel_err_vs_fp64"] for r in reps_),
                     "entries_over_tolerance": sum(r["entries_over_tolerance"] for r in reps_),
                     "entries": sum(r["entries"] for r in reps_),
                     "members_bit_exact_with_reference": sum(
                         r["bit_exact_with_reference"] for r in reps_)}
        del batch, members
    del bufs
    torch.cuda.empty_cache()
    n = 8192
    A = torch.randn(n * n, device=dev, generator=g)
    B = torch.randn(n * n, device=dev, generator=g)
    C = torch.empty(n * n, device=dev)
    ir = mm_ir(n, n, n)
    big = {"workload": "8192^3 matmul"}
    rows = np.random.default_rng(9).choice(n, 16, replace=False)
    a16 = A.view(n, n)[torch.from_numpy(rows).to(dev)].cpu().numpy()
    bn = B.view(n, n).cpu().numpy()
    ex16, r16 = a16.astype(np.float64) @ bn.astype(np.float64), sequential_fp32_rows(a16, bn)
    del bn
    for prec in ("bf16", "bf16x3", "bf16x6"):
        c1 = ltb.Compiled(ir, precision=prec)
        b1, _, sched = ltb.tune_batch([(c1, [A, B, C])], reps=2)
        b1.run_timed()
        pack_ms, gemm_ms = b1.run_timed()
        products = {"bf16": 1, "bf16x3": 3, "bf16x6": 6}[prec]
        big[prec] = {"total_ms": pack_ms + gemm_ms, "pack_ms": pack_ms, "gemm_ms": gemm_ms,
                     "tile_variant": c1.schedule(0)[2],
                     "pack_schedule": [b1.int_property("pack_chunk"),
                                       b1.int_property("pack_cta_per_sm")],
                     "tflops_total": 2 * n ** 3 / ((pack_ms + gemm_ms) * 1e-3) / 1e12,
                     "tensor_tflops_gemm": products * 2 * n ** 3 / (gemm_ms * 1e-3) / 1e12,
                     "frac_of_measured_bf16_peak": products * 2 * n ** 3 / (gemm_ms * 1e-3) /
                     1e12 / bf16_peak,
                     "sampled_rows": elementwise_report(
                         C.view(n, n)[torch.from_numpy(rows).to(dev)].cpu().numpy(), r16, ex16)}
        del b1
    out["mm_8192"] = big
    return out


# ----------------------------------------------------------------- c5
P99_BOUND_MS = 20.0  # capacity = the highest served rate with p99 under this


def extra_c5(dev, n_requests, rates):
    """Serving the seeded trace with the native request loop (ltb_server_*,
    C++: no Python per request).  Warm: each server compiles the trace's
    distinct programs (or buckets) once, untimed, reserves its slot
    workspaces and serves an untimed warm-up trace (first launches load
    kernel modules), then serves the trace at every offered rate of the
    sweep.  Cold: a fresh server serves the trace at one rate with its
    kernel cache empty (every first use of a program compiles inside that
    request's latency), exact-size keys and shape buckets.  One arm of the
    Python loop (serve.Server) at one rate shows the host loop's share."""
    from loop_tool_b200.serve import NativeServer, Server, make_trace, padding_overhead

    trace0 = make_trace(n_requests, rate=1e9, seed=501)
    warmup = make_trace(2000, rate=1e9, seed=777)
    out = {"workload": f"{n_requests} requests, Poisson arrivals, 50% matmul (c4 shapes), "
                       f"30% conv (batch U[1,64]), 20% softmax (rows U[1,8192] x 4096)",
           "loop": "native (C++ ltb_server): admission, slots, kernel cache, device-side inputs",
           "workspaces": "reserved per slot before serving",
           "distinct_programs": len({(r.kind, r.params) for r in trace0}),
           "bucket_padding_work_ratio": padding_overhead(trace0),
           "capacity_rule": f"highest offered rate served at >= 95% with p99 <= {P99_BOUND_MS} ms"}
    configs = [("b200_bf16x3_8slots", dict(slots=8, precision="bf16x3")),
               ("b200_bf16x3_8slots_buckets", dict(slots=8, precision="bf16x3", buckets=True)),
               ("plain_fp32_1slot", dict(slots=1, precision="fp32"))]
    keys = ("req_per_s", "p50_ms", "p99_ms", "mean_ms", "peak_inflight", "compiles", "compile_s")
    for name, kw in configs:
        srv = NativeServer(hbm_budget=24 << 30, **kw)
        w0 = time.perf_counter()
        srv.prepare(trace0)  # every program compiled, workspaces sized, before the clock
        warm_s = time.perf_counter() - w0
        srv.serve(warmup)
        sweep, capacity = {}, None
        for rate in rates:
            stats, _ = srv.serve(make_trace(n_requests, rate=rate, seed=501))
            sweep[f"rate_{int(rate)}"] = {k: stats[k] for k in keys}
            if stats["req_per_s"] >= 0.95 * rate and stats["p99_ms"] <= P99_BOUND_MS:
                capacity = max(capacity or 0, rate)
        out[name] = {"kernel_cache": "warm", "warm_compile_s": warm_s,
                     "compiled_programs": stats["compiles"], "sweep": sweep,
                     "capacity_req_per_s": capacity,
                     "saturation_req_per_s": max(v["req_per_s"] for v in sweep.values())}
        del srv
    cold_rate = 4000.0
    for name, kw in configs[:2]:
        srv = NativeServer(hbm_budget=24 << 30, **kw)
        stats, _ = srv.serve(make_trace(n_requests, rate=cold_rate, seed=501))
        out[name + "_cold"] = dict({k: stats[k] for k in keys}, offered_req_per_s=cold_rate,
                                   kernel_cache="cold (compiles inside latency)")
        del srv
    # the Python request loop, same configuration, warm, at the native arm's
    # saturation point (offered 16k req/s)
    py = Server(slots=8, hbm_budget=24 << 30, precision="bf16x3")
    for r in trace0:
        py.bytes_of(r)
    py.reserve(trace0)
    py.serve(make_trace(2000, rate=1e9, seed=777))
    stats, _ = py.serve(make_trace(n_requests, rate=16000.0, seed=501))
    out["python_loop_bf16x3_8slots_rate_16000"] = {k: stats[k] for k in keys}
    del py
    return out


# ------------------------------------------------------- profiling cases
NCU_CASES = ("add", "add_2p28", "softmax", "maxpool", "mm_bf16", "mm_bf16x3", "mm_fp32", "conv_bf16",
             "conv_fp32", "batch_bf16", "mm_bf16_batch")


def ncu_case(name, reps, tune=True, schedules=None, variant=0):
    """One workload at a profiling size (inputs above L2, about 1 GB on the
    device), autotuned as in the benchmark, then run `reps` times inside the
    NVTX range "profile" (capture with ncu --nvtx --nvtx-include profile/).
    With `schedules` (a file path): if the file exists its schedules are
    loaded and nothing is tuned, else the tuned schedules are written there,
    so a capture under ncu runs what the plain run before it chose.  With
    `variant`, single-program cases run that launch variant on their first
    stage instead of tuning (e.g. 133: halo tiles on CTA pairs)."""
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
    elif name == "add_2p28":  # the headline's add at its own size (3.2 GB per launch)
        ir = reference_ir("add_2p28")
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
    if variant:
        c.set_schedule(0, variant=variant)
        tune = False
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
    ap.add_argument("--serve-rates", default="2000,4000,8000,16000")
    ap.add_argument("--ncu-case", choices=NCU_CASES,
                    help="run one workload at a profiling size and exit")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--variant", type=int, default=0,
                    help="--ncu-case: run this launch variant on the first stage (no tuning)")
    ap.add_argument("--schedules",
                    help="with --ncu-case: schedule file written by a tuning run and loaded "
                         "(no tuning) by a later run, e.g. the same case under ncu")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu_case:
        return ncu_case(args.ncu_case, args.reps, args.tune, args.schedules, args.variant)

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
        line["e2e_via_reference_frontend"] = reference_frontend(line["nests_bytes"])
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
