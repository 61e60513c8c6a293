"""Continuous-batching request loop over the B200 backend.

Requests are lazy-tensor programs (this package's lazy frontend) of varying
symbolic sizes.  The loop:
  * admits a request as soon as a slot (a CUDA stream) is free and its bytes
    (inputs + output + scratch, from the compiled plan) fit the HBM budget;
    requests that arrive while others run are admitted in arrival order as
    slots and memory free up, so their kernels overlap on the device;
  * reuses compiled loop trees through its kernel cache, one entry per
    distinct program + sizes (the reference's lazy cache is keyed the same
    way, lazy.h:82-115), applying any autotuned schedule cached for the IR;
  * keeps every buffer device-resident: inputs are produced on the device,
    buffers come from torch's stream-ordered caching allocator, and each run
    gets its own scratch (ltb_run_with_scratch), so concurrent runs of one
    compiled object never share scratch;
  * reports throughput and p50 / p99 latency (arrival -> completion).

The reference has no serving loop; its lazy frontend runs one program at a
time, synchronously (lazy.h:255-258).
"""
import math
import time
from collections import deque

import numpy as np

from . import lazy as lt
from . import nn
from .backend import Compiled

KINDS = ("matmul", "conv", "softmax")


def make_trace(n, rate, seed=501, mix=(0.5, 0.3, 0.2), mm_range=(64, 4096),
               conv_batch=(1, 64), softmax_rows=(1, 8192)):
    """Seeded request trace with Poisson arrivals at `rate` requests/s:
    matmuls with M, N, K log-uniform in mm_range rounded to multiples of 16,
    3x3 pad-1 convolutions [b,64,56,56] * [128,64,3,3] with b uniform in
    conv_batch, row softmaxes [rows, 4096] with rows uniform in softmax_rows."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    kinds = rng.choice(3, size=n, p=list(mix))
    out = []
    lo, hi = math.log(mm_range[0]), math.log(mm_range[1])
    for i in range(n):
        k = KINDS[kinds[i]]
        if k == "matmul":
            m, nn_, kk = (int(max(16, 16 * round(math.exp(rng.uniform(lo, hi)) / 16)))
                          for _ in range(3))
            params = (m, kk, nn_)
        elif k == "conv":
            params = (int(rng.integers(conv_batch[0], conv_batch[1] + 1)),)
        else:
            params = (int(rng.integers(softmax_rows[0], softmax_rows[1] + 1)),)
        out.append(Request(i, k, params, float(t[i]), seed * 1000003 + i))
    return out


class Request:
    __slots__ = ("rid", "kind", "params", "arrival", "seed", "admitted", "done", "out",
                 "bytes", "event", "hold")

    def __init__(self, rid, kind, params, arrival, seed):
        self.rid, self.kind, self.params, self.arrival, self.seed = rid, kind, params, arrival, seed
        self.admitted = self.done = None
        self.out = None
        self.bytes = 0
        self.event = None
        self.hold = None


def _program(kind, params):
    """The request's loop tree, built with the lazy frontend."""
    if kind == "matmul":
        M, K, N = params
        A, B = lt.Tensor(M, K), lt.Tensor(K, N)
        m, k, n = lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
        return (A.to(m, k) * B.to(k, n)).sum(k)
    if kind == "conv":
        (b,) = params
        X, W = lt.Tensor(b, 64, 56, 56), lt.Tensor(128, 64, 3, 3)
        n_, c, h, w, co, kh, kw = (lt.Symbol(x) for x in ("n", "c", "h", "w", "co", "kh", "kw"))
        x = X.to(n_, c, h, w).pad(h, 1)
        x = x.pad(x.shape[3], 1)
        return nn.conv(x, W.to(co, c, kh, kw), [x.shape[2], x.shape[3]], [kh, kw])
    (rows,) = params
    X = lt.Tensor(rows, 4096)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    x = X.to(r, n)
    e = (x - x.max_reduce(n)).exp()
    return e / e.sum(n)


# Shape buckets (the reference keys its compile cache by exact sizes,
# lazy.h:82-115, so every new size is a new compile): a bucketed server
# compiles one loop tree per bucket and runs each request in it, its inputs
# zero-padded into the bucket's layout and its output read back at the
# request's own size.  Zero padding only adds exact zeros to sums (and
# computes rows / columns / images that are dropped), so values stay within
# the contraction's tolerance.  Ladder: multiples of 16, about 1.25x apart.
LADDER = sorted({16 * round(16 * 1.25 ** i / 16) for i in range(0, 40)
                 if 16 * 1.25 ** i <= 1 << 15} | {1, 2, 4, 8})


def _bucket(x):
    for b in LADDER:
        if b >= x:
            return b
    return x


def bucket_params(kind, params):
    """The bucket a request runs in: matmul M, K, N and softmax rows up the
    ladder, convolution batch to the next power of two."""
    if kind == "matmul":
        return tuple(_bucket(v) for v in params)
    if kind == "conv":
        (b,) = params
        return (1 << (b - 1).bit_length(),)
    (rows,) = params
    return (_bucket(rows),)


def work_of(kind, params):
    """FLOP (contractions) or bytes (softmax) of a request, for the padding
    overhead of buckets."""
    if kind == "matmul":
        M, K, N = params
        return 2.0 * M * K * N
    if kind == "conv":
        return 2.0 * params[0] * 128 * 56 * 56 * 64 * 9
    return 8.0 * params[0] * 4096


_ALIGN = 64  # floats (256 bytes) between the regions of a slot workspace


def _up(n):
    return (n + _ALIGN - 1) // _ALIGN * _ALIGN


class Server:
    """slots: concurrent requests (one CUDA stream each); hbm_budget: bytes of
    request buffers admitted at once; precision: contraction mode.

    Each slot owns one device workspace (grown on demand, never per request)
    that holds its request's inputs, output and run scratch, so the steady
    state makes no allocator calls; a slot that must grow first releases the
    workspaces of idle slots when the sum would pass the budget."""

    def __init__(self, slots=8, hbm_budget=16 << 30, precision="bf16x3", device=0,
                 keep_outputs=False, buckets=False):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(slots)]
        self.gens = [torch.Generator(device=self.dev) for _ in range(slots)]
        self.events = [torch.cuda.Event() for _ in range(slots)]
        self.ws = [None] * slots
        self.free = list(range(slots))
        self.budget = hbm_budget
        self.used = 0
        self.precision = precision
        self.keep = keep_outputs
        self._kernels = {}
        self.compiles = 0
        self.compile_s = 0.0
        self.buckets = buckets

    def _shape(self, req):
        return bucket_params(req.kind, req.params) if self.buckets else req.params

    def _compiled(self, req):
        """The request's compiled loop tree from the server's own kernel
        cache: one entry per distinct program and sizes (or per bucket),
        never evicted (a trace of 20,000 requests holds ~14,000 distinct
        programs, ~1,800 buckets)."""
        key = (req.kind, self._shape(req))
        c = self._kernels.get(key)
        if c is None:
            t0 = time.perf_counter()
            c = Compiled(_program(req.kind, key[1]).ir, precision=self.precision)
            self.compile_s += time.perf_counter() - t0
            self._kernels[key] = c
            self.compiles += 1
        return c

    def _workspace(self, slot, floats):
        torch = self.torch
        ws = self.ws[slot]
        if ws is not None and ws.numel() >= floats:
            return ws
        want = max(floats, int(1.25 * ws.numel()) if ws is not None else 0)
        held = sum(w.numel() for w in self.ws if w is not None) - (ws.numel() if ws is not None else 0)
        if 4 * (held + want) > self.budget:
            for s in self.free:
                if s != slot:
                    self.ws[s] = None
            want = floats
        self.ws[slot] = None
        self.ws[slot] = torch.empty(want, device=self.dev)
        return self.ws[slot]

    def _need(self, req):
        """Floats of a slot workspace for this request (regions 256-byte
        aligned: inputs, output, run scratch)."""
        c = self._compiled(req)
        return sum(_up(n) for n in c.io_sizes) + _up((c.int_property("scratch_bytes") + 3) // 4)

    def reserve(self, trace):
        """Size every slot's workspace for the largest request of `trace`
        (within the HBM budget) before serving, so no allocation, and no
        allocator synchronisation, happens while requests are in flight."""
        need = max((self._need(r) for r in trace), default=0)
        per_slot = min(need, self.budget // (4 * len(self.streams)))
        for slot in range(len(self.streams)):
            with self.torch.cuda.stream(self.streams[slot]):
                self._workspace(slot, per_slot)
        self.torch.cuda.synchronize()
        return 4 * per_slot * len(self.streams)

    def _launch(self, req, slot, now):
        torch = self.torch
        c = self._compiled(req)
        st = self.streams[slot]
        sizes = c.io_sizes
        sb = (c.int_property("scratch_bytes") + 3) // 4
        offs, o = [], 0
        for n in sizes:
            offs.append(o)
            o += _up(n)
        with torch.cuda.stream(st):
            ws = self._workspace(slot, o + _up(sb))
            gen = self.gens[slot]
            gen.manual_seed(req.seed)
            views = [ws[a:a + n] for a, n in zip(offs, sizes)]
            for i, x in enumerate(views[:c.n_inputs]):
                dst = self._true_view(req, x, i)
                if dst is not x:
                    x.zero_()  # bucket padding
                v = torch.randn(dst.numel(), generator=gen, device=self.dev).view(dst.shape)
                if req.kind == "matmul":
                    v /= math.sqrt(req.params[1])  # N(0,1)/sqrt(K)
                elif req.kind == "conv" and i == 1:
                    v *= math.sqrt(6.0 / 576) / math.sqrt(3.0)  # Kaiming-uniform scale
                elif req.kind == "softmax":
                    v *= 4.0
                dst.copy_(v)
            c.run(views, sync=False, stream=st.cuda_stream,
                  scratch=ws[o:].data_ptr() if sb else None)
            ev = self.events[slot]
            ev.record(st)
        req.event, req.hold, req.admitted = ev, self._true_view(req, views[-1], -1), now

    def _true_view(self, req, buf, i):
        """The request's own part of one of its (possibly bucket-padded)
        buffers: input i, or the output for i = -1."""
        if not self.buckets:
            return buf
        p, q = req.params, self._shape(req)
        if p == q:
            return buf
        if req.kind == "matmul":
            (M, K, N), (Mp, Kp, Np) = p, q
            shape, want = {0: ((Mp, Kp), (M, K)), 1: ((Kp, Np), (K, N)),
                           -1: ((Mp, Np), (M, N))}[i]
            return buf.view(shape)[:want[0], :want[1]]
        if req.kind == "conv":
            if i == 1:  # weights: no batch dim
                return buf
            return buf.view(q[0], -1)[:p[0]]
        return buf.view(q[0], 4096)[:p[0]]

    def bytes_of(self, req):
        c = self._compiled(req)
        return 4 * sum(c.io_sizes) + c.int_property("scratch_bytes")

    def serve(self, trace, time_scale=1.0, poll_sleep=0.0):
        """Run a trace against the wall clock.  Returns per-request latencies
        (seconds) and summary statistics."""
        torch = self.torch
        pending = deque()
        inflight = {}
        arrivals = deque(sorted(trace, key=lambda r: r.arrival))
        done = []
        self.peak_used = self.peak_inflight = 0
        t0 = time.perf_counter()
        while arrivals or pending or inflight:
            now = time.perf_counter() - t0
            while arrivals and arrivals[0].arrival * time_scale <= now:
                r = arrivals.popleft()
                r.bytes = self.bytes_of(r)
                if r.bytes > self.budget:
                    raise ValueError(f"request {r.rid} needs {r.bytes} B > budget {self.budget} B")
                pending.append(r)
            for slot, r in list(inflight.items()):
                if r.event.query():
                    r.done = time.perf_counter() - t0
                    if self.keep:
                        r.out = r.hold.cpu().numpy().ravel()
                    r.hold = None
                    self.used -= r.bytes
                    self.free.append(slot)
                    del inflight[slot]
                    done.append(r)
            while pending and self.free and self.used + pending[0].bytes <= self.budget:
                r = pending.popleft()
                slot = self.free.pop()
                self.used += r.bytes
                self._launch(r, slot, time.perf_counter() - t0)
                inflight[slot] = r
                self.peak_used = max(self.peak_used, self.used)
                self.peak_inflight = max(self.peak_inflight, len(inflight))
            if not pending and not inflight and arrivals:
                wait = arrivals[0].arrival * time_scale - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            elif poll_sleep:
                time.sleep(poll_sleep)
        torch.cuda.synchronize()
        lat = np.array([r.done - r.arrival * time_scale for r in done])
        span = max(r.done for r in done) - min(r.arrival * time_scale for r in done)
        return {
            "requests": len(done),
            "req_per_s": len(done) / span if span > 0 else float("nan"),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3),
            "span_s": span,
            "compiles": self.compiles,
            "compile_s": self.compile_s,
            "peak_inflight": self.peak_inflight,
            "peak_bytes": self.peak_used,
            "slots": len(self.streams),
            "precision": self.precision,
        }, done


_IR_TEXT = {}  # (kind, shape) -> IR bytes, built once per distinct program


def _ir_bytes(kind, shape):
    key = (kind, shape)
    t = _IR_TEXT.get(key)
    if t is None:
        t = _IR_TEXT[key] = _program(kind, shape).ir.encode()
    return t


def _blocks(kind, params, shape):
    """(rows, cols, true_rows, true_cols, scale) of each buffer of a request
    whose program runs at `shape` (its bucket, or its own sizes): inputs
    first, then the output; the true block holds the request's own data."""
    if kind == "matmul":
        (M, K, N), (Mp, Kp, Np) = params, shape
        return [(Mp, Kp, M, K, 1.0 / math.sqrt(K)), (Kp, Np, K, N, 1.0), (Mp, Np, M, N, 0.0)]
    if kind == "conv":
        (b,), (bp,) = params, shape
        img, out = 64 * 56 * 56, 56 * 56 * 128
        return [(bp, img, b, img, 1.0), (128, 64 * 9, 128, 64 * 9, math.sqrt(6.0 / 576) / math.sqrt(3.0)),
                (bp, out, b, out, 0.0)]
    (rows,), (rp,) = params, shape
    return [(rp, 4096, rows, 4096, 4.0), (rp, 4096, rows, 4096, 0.0)]


class NativeServer:
    """The same request loop in C++ (ltb_server_*, csrc/serve.cpp): slots
    as streams, HBM budget admission, a kernel cache per distinct loop tree,
    inputs generated on the device from each request's seed (zero-padded
    into its bucket's layout when `buckets`), per-slot workspaces.  The
    Python side only describes the trace; no Python runs per request."""

    def __init__(self, slots=8, hbm_budget=16 << 30, precision="bf16x3", buckets=False):
        import ctypes

        from . import _lib

        self._c, self._L = ctypes, _lib
        self.buckets = buckets
        self.precision = precision
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ltb_server_create(int(slots), int(hbm_budget),
                                                f"precision={precision}".encode(),
                                                ctypes.byref(h)))
        self._h = h
        self.slots = slots

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and self._L._lib is not None:
            self._L.lib().ltb_server_release(h)
            self._h = None

    def _requests(self, trace, keep_outputs=False):
        c, L = self._c, self._L
        arr = (L.LtbRequest * len(trace))()
        outs = []
        for i, r in enumerate(trace):
            shape = bucket_params(r.kind, r.params) if self.buckets else r.params
            q = arr[i]
            q.ir_text = _ir_bytes(r.kind, shape)
            q.arrival_s = r.arrival
            q.seed = r.seed
            bl = _blocks(r.kind, r.params, shape)
            q.n_io = len(bl)
            for j, (R, C, tr, tc, sc) in enumerate(bl):
                q.io[j] = L.LtbBlock(R, C, tr, tc, sc)
            if keep_outputs:
                R, C, tr, tc, _ = bl[-1]
                o = np.empty(tr * tc, np.float32)
                outs.append(o)
                q.host_out = o.ctypes.data_as(c.POINTER(c.c_float))
            else:
                outs.append(None)
        return arr, outs

    def prepare(self, trace):
        """Compile every distinct program of the trace and size the slot
        workspaces for its largest request; returns the bytes reserved."""
        arr, _ = self._requests(trace)
        got = self._c.c_int64()
        self._L.check(self._L.lib().ltb_server_prepare(self._h, arr, len(trace),
                                                       self._c.byref(got)))
        return got.value

    def serve(self, trace, time_scale=1.0, keep_outputs=False):
        """Serve the trace against the wall clock; returns (stats, outputs),
        outputs[i] the true output of trace[i] when keep_outputs."""
        c, L = self._c, self._L
        arr, outs = self._requests(trace, keep_outputs)
        st = L.LtbServeStats()
        lat = (c.c_double * len(trace))()
        L.check(L.lib().ltb_server_serve(self._h, arr, len(trace), float(time_scale),
                                         c.byref(st), lat))
        stats = {k: getattr(st, k) for k, _ in L.LtbServeStats._fields_}
        stats.update(slots=self.slots, precision=self.precision, buckets=self.buckets)
        return stats, outs


def padding_overhead(trace):
    """Work of the trace run in its buckets over its own work."""
    own = sum(work_of(r.kind, r.params) for r in trace)
    return sum(work_of(r.kind, bucket_params(r.kind, r.params)) for r in trace) / own


def run_alone(req, precision="bf16x3", device=0, buckets=False):
    """One request by itself on a fresh stream: the reference point for
    "same result alone and in the mix"."""
    s = Server(slots=1, precision=precision, device=device, keep_outputs=True, buckets=buckets)
    r = Request(req.rid, req.kind, req.params, 0.0, req.seed)
    s.serve([r])
    return r.out
