#!/usr/bin/env python
"""Benchmark of the B200 "cuda" backend for loop_tool.

Workload (one step): the bandwidth-bound FP32 nests of the reference's
headline configuration, each a loop tree built by the lazy frontend and run
through the backend's Compiled::run entry point (the C ABI):
  (i)   C = A + B over 2^28 elements
  (ii)  row softmax of x[8192, 4096] (max, subtract, exp, sum, divide)
  (iii) 2x2 stride-2 max-pool of X[64, 128, 112, 112]
Metric: HBM GB/s of algorithmic traffic (every input element read once,
every output element written once) for the whole step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's own CPU backend ("cpp": generated C
compiled by cc -O3, single-threaded like the reference) on the host cores, on
a bounded sample of the same workload.
"""
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

NESTS = [
    # name, IR fixture, input element counts, output element count
    ("add_2p28", "add_2p28.txt"),
    ("softmax_8192x4096", "softmax_8192x4096.txt"),
    ("maxpool_64x128x112x112", "maxpool_64x128x112x112.txt"),
]
IR_DIR = os.path.join(ROOT, "tests", "golden", "ir")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def read_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

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
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_time(nests, budget_s=20.0):
    """Times the reference CPU backend on a bounded sample of each nest:
    the same loop tree at reduced size, scaled by bytes."""
    samples = {
        "add_2p28": ("add", [1 << 24]),
        "softmax_8192x4096": ("softmax", [512, 4096]),
        "maxpool_64x128x112x112": ("maxpool", [4, 128, 112, 112, 2, 2]),
    }
    total_bytes = 0.0
    total_s = 0.0
    desc = []
    for name in nests:
        prog, params = samples[name]
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
            r = subprocess.run(["taskset", "-c", "0", HARNESS, "run", irf, "cpp", td, td, "3"],
                               capture_output=True, text=True)
            if r.returncode != 0:
                r = subprocess.run([HARNESS, "run", irf, "cpp", td, td, "3"],
                                   capture_output=True, text=True, check=True)
            secs = json.loads(r.stdout.strip().splitlines()[-1])["seconds"]
            t = min(secs)
            b = 4 * (sum(sizes["inputs"]) + sum(sizes["outputs"]))
            total_bytes += b
            total_s += t
            desc.append(f"{prog}{params}")
    return total_bytes / total_s / 1e9, "; ".join(desc)


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    if not os.path.exists(HARNESS):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref not built (make -C oracle)"}))
        return
    vals = []
    desc = ""
    for _ in range(args.warmup):
        reference_time([n for n, _ in NESTS])
    for _ in range(args.steps):
        v, desc = reference_time([n for n, _ in NESTS])
        vals.append(v)
    v = min(vals)
    print(json.dumps({
        "impl": "reference", "metric": "hbm_gbs_bandwidth_nests", "value": v, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
        "config": {"workload": "bandwidth nests: add 2^28, softmax 8192x4096, maxpool 64x128x112x112",
                   "parallelism": "cpu"},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": 1, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    import loop_tool_b200 as lt

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.init()

    comps, bufs, bytes_per = [], [], []
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    for name, fn in NESTS:
        ir = open(os.path.join(IR_DIR, fn)).read()
        c = lt.cuda(ir)
        ins = [torch.randn(n, device=dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
        if name.startswith("softmax"):
            ins = [4.0 * x for x in ins]
        outs = [torch.empty(n, device=dev) for n in c.io_sizes[c.n_inputs:]]
        comps.append(c)
        bufs.append(ins + outs)
        bytes_per.append(4 * sum(c.io_sizes))
    stream = torch.cuda.current_stream()

    def step(times=None):
        for i, (c, b) in enumerate(zip(comps, bufs)):
            if times is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            c.run(b, sync=False)
            if times is not None:
                e1.record(stream)
                times[i].append((e0, e1))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    per = [[] for _ in NESTS]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        step(per)
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = t0.elapsed_time(t1)
    nest_ms = [statistics.mean(a.elapsed_time(b) for a, b in lst) for lst in per]
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = tt.item()
    step_bytes = sum(bytes_per)
    value = world * step_bytes * args.steps / (ms / 1e3) / 1e9

    # e2e: same step through the C ABI with pinned host buffers; host->device
    # copies of the inputs and device->host copies of the outputs are inside
    # the timed region (the backend stages host pointers through HBM).
    hbufs = []
    for c, b in zip(comps, bufs):
        hb = [x.cpu().pin_memory() for x in b[:c.n_inputs]]
        hb += [torch.empty(n, pin_memory=True) for n in c.io_sizes[c.n_inputs:]]
        hbufs.append(hb)
    e2e_steps = max(1, min(args.steps, 3))
    for c, hb in zip(comps, hbufs):
        c.run(hb, sync=True)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        for c, hb in zip(comps, hbufs):
            c.run(hb, sync=True)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - w0) / e2e_steps
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_s = tt.item()
    h2d = sum(4 * sum(c.io_sizes[:c.n_inputs]) for c in comps)
    d2h = sum(4 * sum(c.io_sizes[c.n_inputs:]) for c in comps)

    peak, peak_kind = load_peaks()
    dom = int(np.argmax(nest_ms))
    achieved = bytes_per[dom] / (nest_ms[dom] / 1e3) / 1e9
    traffic = read_traffic().get(NESTS[dom][0])
    launches = sum(c.int_property("launches") for c in comps) * args.steps

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and os.path.exists(HARNESS):
        try:
            v, desc = reference_time([n for n, _ in NESTS])
            cpu = {"value": v, "unit": "GB/s", "cores": 1, "kind": "reference", "sample": desc}
        except Exception as e:  # reported, never fatal to the GPU number
            cpu = {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps({
            "metric": "hbm_gbs_bandwidth_nests", "value": value, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "bandwidth nests: add 2^28, softmax 8192x4096, "
                                   "maxpool 64x128x112x112 (FP32, lazy-frontend loop trees)",
                       "l2": "inputs larger than L2 (126 MB)",
                       "parallelism": f"replicas{world}"},
            "nests_ms": {n: t for (n, _), t in zip(NESTS, nest_ms)},
            "nests_gbs": {n: b / (t / 1e3) / 1e9 for (n, _), b, t in zip(NESTS, bytes_per, nest_ms)},
            "roofline": {"bound": "hbm", "kernel": NESTS[dom][0], "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic},
            "e2e": {"value": world * step_bytes / e2e_s / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
