"""Host-side mirror of the reference's backend plugin surface.

Reference: include/loop_tool/backend.h (Backend::compile -> Compiled,
Compiled::run(memory, sync)), and the Python binding src/frontends/python.cpp
where each registered backend becomes ``lt.<name>(loop_tree)`` (:208-218) and
``Compiled.__call__`` runs it on a list of tensors (:182-196).

Here the loop tree crosses the C ABI as serialized IR text; ``cuda`` accepts
that text, an object with ``serialize()`` (this package's IR / LoopTree) or
a lazy Tensor.
"""
import ctypes

import numpy as np

from . import _lib

_OPT_KEYS = ("precision", "fuse_rows", "tensor_cores", "kahan_threshold")


def _options(opts):
    parts = []
    for k, v in opts.items():
        if k not in _OPT_KEYS:
            raise ValueError(f"unknown option {k}")
        if isinstance(v, bool):
            v = int(v)
        parts.append(f"{k}={v}")
    return ";".join(parts).encode()


def _ir_text(obj):
    if isinstance(obj, str):
        return obj
    if isinstance(obj, bytes):
        return obj.decode()
    if hasattr(obj, "serialize"):
        return obj.serialize()
    raise TypeError(f"cannot take a loop tree from {type(obj).__name__}")


def plan(loop_tree, **opts):
    """The kernel plan for a loop tree, computed on the host (no device)."""
    buf = ctypes.create_string_buffer(1 << 20)
    _lib.check(_lib.lib().ltb_plan(_ir_text(loop_tree).encode(), _options(opts), buf, len(buf)))
    return buf.value.decode()


def device_count():
    return _lib.lib().ltb_device_count()


_TORCH_F32 = []  # torch.float32, looked up once (torch is optional)


def _is_f32(dtype):
    if not _TORCH_F32:
        import torch

        _TORCH_F32.append(torch.float32)
    return dtype is _TORCH_F32[0]


def _ptr_and_keep(t):
    """Raw pointer of a buffer-like; returns (ptr, keepalive, host_array)."""
    if hasattr(t, "data_ptr"):  # torch.Tensor
        if not _is_f32(t.dtype):
            raise TypeError("loop_tool buffers are float32")
        if not t.is_contiguous():
            raise ValueError("buffers must be contiguous")
        return t.data_ptr(), t, None
    if isinstance(t, RawTensor):
        return t.ptr, t, None
    if isinstance(t, np.ndarray):
        if t.dtype != np.float32 or not t.flags.c_contiguous:
            raise TypeError("numpy buffers must be contiguous float32")
        return t.ctypes.data, t, t
    if isinstance(t, int):
        return t, None, None
    raise TypeError(f"unsupported buffer type {type(t).__name__}")


class Compiled:
    """A loop tree compiled for the B200 (CudaCompiled, cuda.cpp:818-851)."""

    def __init__(self, loop_tree, **opts):
        self.ir_text = _ir_text(loop_tree)
        self.options = dict(opts)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ltb_compile(self.ir_text.encode(), _options(opts), ctypes.byref(h)))
        self._h = h
        n_in, n_out = ctypes.c_int(), ctypes.c_int()
        elems = (ctypes.c_int64 * 256)()
        _lib.check(_lib.lib().ltb_io_sizes(h, ctypes.byref(n_in), ctypes.byref(n_out), elems, 256))
        self.n_inputs, self.n_outputs = n_in.value, n_out.value
        self.io_sizes = [elems[i] for i in range(self.n_inputs + self.n_outputs)]
        self.name = "cuda"

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib._lib is not None:
            _lib.lib().ltb_release(h)
            self._h = None

    # Compiled::run(memory, sync)
    def run(self, memory, sync=True, stream=None, scratch=None):
        ptrs, keep = [], []
        for t in memory:
            p, k, _ = _ptr_and_keep(t)
            ptrs.append(p)
            keep.append(k)
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        if stream is None:
            stream = _current_stream()
        if scratch is None:
            rc = _lib.lib().ltb_run(self._h, arr, len(ptrs), int(bool(sync)), stream)
        else:
            rc = _lib.lib().ltb_run_with_scratch(self._h, arr, len(ptrs), int(bool(sync)),
                                                 stream, scratch)
        _lib.check(rc)

    def __call__(self, tensors, sync=True):
        self.run(tensors, sync)

    def schedule_ir(self):
        """The current launch schedule as an annotated loop tree (IR text
        the reference's deserialize reads; ltb_schedule_ir)."""
        buf = ctypes.create_string_buffer(1 << 22)
        _lib.check(_lib.lib().ltb_schedule_ir(self._h, buf, len(buf)))
        return buf.value.decode()

    def run_plan(self, memory):
        """How run() would treat each buffer (in place, staged, rejected),
        decided on the host without launching anything."""
        ptrs, keep = [], []
        for t in memory:
            p, k, _ = _ptr_and_keep(t)
            ptrs.append(p)
            keep.append(k)
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        buf = ctypes.create_string_buffer(1 << 16)
        _lib.check(_lib.lib().ltb_run_plan(self._h, arr, len(ptrs), buf, len(buf)))
        return buf.value.decode().splitlines()

    def int_property(self, name):
        v = ctypes.c_int64()
        _lib.check(_lib.lib().ltb_int_property(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    @property
    def int_properties(self):
        keys = ("bandwidth", "stages", "launches", "scratch_bytes", "inputs", "outputs",
                "algorithmic_bytes", "flops", "tuned", "implicit_conv", "tma_store_output")
        return {k: self.int_property(k) for k in keys}

    def capture(self, memory, stream=None, scratch=None):
        """One run on these device buffers captured as a CUDA graph: every
        launch of the loop tree replayed with one graph launch."""
        return CapturedRun(self, memory, stream, scratch)

    # ------------------------------------------------------------ autotuner
    def tune(self, memory, reps=10, stream=None):
        """Time every candidate schedule of every stage on `memory` (device
        buffers in run order), keep the fastest, record it in the schedule
        cache; returns the per-stage report.  The outputs in `memory` are
        left computed with the chosen schedules."""
        ptrs = [_ptr_and_keep(t)[0] for t in memory]
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        if stream is None:
            stream = _current_stream()
        buf = ctypes.create_string_buffer(1 << 16)
        _lib.check(_lib.lib().ltb_tune(self._h, arr, len(ptrs), stream, int(reps), buf, len(buf)))
        return buf.value.decode()

    def schedule(self, stage):
        """(cta_per_sm, threads, variant) of a stage; zeros = heuristic."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().ltb_get_schedule(self._h, int(stage), ctypes.byref(a),
                                                ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def set_schedule(self, stage, cta_per_sm=0, threads=0, variant=0):
        _lib.check(_lib.lib().ltb_set_schedule(self._h, int(stage), int(cta_per_sm),
                                                int(threads), int(variant)))

    def record_schedule(self):
        """Store the current schedules in the cache (keyed by IR + options)."""
        _lib.check(_lib.lib().ltb_tune_record(self._h))

    @property
    def string_properties(self):
        return {"code": self.code}

    @property
    def code(self):
        buf = ctypes.create_string_buffer(1 << 20)
        _lib.check(_lib.lib().ltb_dump(self._h, buf, len(buf)))
        return buf.value.decode()

    def dump(self):
        return self.code

    def __getattr__(self, name):  # python.cpp:197-207 exposes properties
        if name.startswith("_"):
            raise AttributeError(name)
        if name in ("bandwidth", "stages", "launches", "scratch_bytes", "flops",
                    "algorithmic_bytes"):
            return self.int_property(name)
        raise AttributeError(name)


class CapturedRun:
    """A compiled loop tree's launches on fixed device buffers, captured
    once into a CUDA graph (ltb_graph_create) and replayed by run()."""

    def __init__(self, compiled, memory, stream=None, scratch=None):
        self._compiled = compiled
        self._keep = list(memory)
        ptrs = [_ptr_and_keep(t)[0] for t in memory]
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        if stream is None:
            stream = _current_stream()
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ltb_graph_create(compiled._h, arr, len(ptrs), scratch, stream,
                                               ctypes.byref(h)))
        self._h = h

    def run(self, sync=True, stream=None):
        if stream is None:
            stream = _current_stream()
        _lib.check(_lib.lib().ltb_graph_run(self._h, int(bool(sync)), stream))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib._lib is not None:
            _lib.lib().ltb_graph_release(h)
            self._h = None


_TORCH = []  # the torch module, or None without torch (looked up once)


def _current_stream():
    if not _TORCH:
        try:
            import torch

            _TORCH.append(torch)
        except Exception:
            _TORCH.append(None)
    torch = _TORCH[0]
    if torch is not None and torch.cuda.is_initialized():
        return torch.cuda.current_stream().cuda_stream
    return None


def tune_batch(members, capture_stream=None, reps=3):
    """Tile widths for a batch of contractions, chosen by timing the grouped
    launch (operand packing + persistent GEMMs) under each policy: the
    members' current schedules, every problem at one variant (128 or 256
    columns, each with either epilogue), and each member's own tuned
    variant.  The best policy is left on the members and recorded in the
    schedule cache; the grouped packing's launch shape is then timed the
    same way.  Returns the Batch (captured on capture_stream if given), the
    tile policy and a report."""
    policies = {"current": [c.schedule(0) for c, _ in members]}
    # tile width | form (1: transposed epilogue, 2: 2 CTAs/SM); 258: 256 x 256
    # tiles on CTA pairs
    for v in (128, 129, 130, 256, 257, 258):
        policies[f"all_{v}"] = [(0, 0, v)] * len(members)
    tuned = []
    for c, bufs in members:
        c.tune(bufs, reps=2)
        tuned.append(c.schedule(0))
    policies["member_tuned"] = tuned
    times = {}
    for name, sched in policies.items():
        for (c, _), sc in zip(members, sched):
            c.set_schedule(0, *sc)
        b = Batch(members)
        b.run_timed()
        ms = min(sum(b.run_timed()) for _ in range(reps))
        times[name] = ms
        del b
    best = min(times, key=times.get)
    for (c, _), sc in zip(members, policies[best]):
        c.set_schedule(0, *sc)
        c.record_schedule()
    report = "; ".join(f"{k} {v:.3f} ms" for k, v in times.items()) + f" -> {best}"
    # then the grouped packing's launch shape (chunk of tiles, CTAs per SM)
    b = Batch(members)
    pack = {}
    for chunk, per_sm in ((4, 4), (1, 4), (16, 4), (64, 4), (16, 2), (4, 6), (16, 6), (64, 8)):
        b.set_schedule(chunk, per_sm)
        b.run_timed()
        pack[(chunk, per_sm)] = min(b.run_timed()[0] for _ in range(reps))
    del b
    pbest = min(pack, key=pack.get)
    report += "; pack " + ", ".join(f"{k[0]}x{k[1]} {v:.3f} ms" for k, v in pack.items()) + \
        f" -> chunk {pbest[0]}, {pbest[1]}/SM"
    out = Batch(members)
    out.set_schedule(*pbest)
    if capture_stream is not None:
        out._capture_stream = capture_stream
        _lib.check(_lib.lib().ltb_batch_capture(out._h, capture_stream))
    return out, best, report


def tune_save(path):
    """Write the schedule cache (IR text + options + per-stage schedule)."""
    _lib.check(_lib.lib().ltb_tune_save(str(path).encode()))


def tune_load(path):
    """Merge a schedule file into the cache; later compiles of the same IR
    and options start from the stored schedules."""
    _lib.check(_lib.lib().ltb_tune_load(str(path).encode()))


def tune_clear():
    _lib.check(_lib.lib().ltb_tune_clear())


def tune_entries():
    return int(_lib.lib().ltb_tune_entries())


def cuda(loop_tree, **opts):
    """lt.cuda(loop_tree) -> Compiled (python.cpp:208-218)."""
    return Compiled(loop_tree, **opts)


class RawTensor:
    """Buffer from the backend's "cuda" hardware allocator
    (CudaGPUHardware::alloc/free, cuda.cpp:800-816): device memory, managed
    memory (managed=True) or pinned host memory (pinned=True)."""

    def __init__(self, size, managed=False, pinned=False):
        self.size = int(size)
        p = ctypes.c_void_p()
        kind = 2 if pinned else int(bool(managed))
        _lib.check(_lib.lib().ltb_alloc(max(self.size, 1) * 4, kind, ctypes.byref(p)))
        self.ptr = p.value
        self.managed = managed

    def __del__(self):
        if getattr(self, "ptr", None) and _lib._lib is not None:
            _lib.lib().ltb_free(self.ptr)
            self.ptr = None


class Batch:
    """Many compiled contractions run as one grouped launch (optionally a
    captured CUDA graph): the batched-uneven-matmul form of family (c).
    `members` is a list of (Compiled, [device buffers in run order])."""

    def __init__(self, members, capture_stream=None):
        n = len(members)
        self._keep = members
        hs = (ctypes.c_void_p * n)(*[c._h.value for c, _ in members])
        rows = []
        for c, bufs in members:
            ptrs = [_ptr_and_keep(t)[0] for t in bufs]
            rows.append((ctypes.c_void_p * len(ptrs))(*ptrs))
        self._rows = rows
        mem = (ctypes.POINTER(ctypes.c_void_p) * n)(
            *[ctypes.cast(r, ctypes.POINTER(ctypes.c_void_p)) for r in rows])
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ltb_batch_create(hs, mem, n, ctypes.byref(h)))
        self._h = h
        self._capture_stream = capture_stream
        if capture_stream is not None:
            _lib.check(_lib.lib().ltb_batch_capture(h, capture_stream))

    def set_schedule(self, pack_chunk=0, pack_cta_per_sm=0):
        """Launch shape of the grouped operand packing (0: defaults); a
        captured graph is captured again."""
        _lib.check(_lib.lib().ltb_batch_set_schedule(self._h, int(pack_chunk),
                                                      int(pack_cta_per_sm)))
        if self._capture_stream is not None:
            _lib.check(_lib.lib().ltb_batch_capture(self._h, self._capture_stream))

    def run(self, sync=True, stream=None):
        if stream is None:
            stream = _current_stream()
        _lib.check(_lib.lib().ltb_batch_run(self._h, int(bool(sync)), stream))

    def int_property(self, name):
        v = ctypes.c_int64()
        _lib.check(_lib.lib().ltb_batch_int_property(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def run_timed(self, stream=None):
        """(pack_ms, gemm_ms) of one eager run, CUDA-event timed."""
        if stream is None:
            stream = _current_stream()
        a, b = ctypes.c_float(), ctypes.c_float()
        _lib.check(_lib.lib().ltb_batch_run_timed(self._h, stream, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib._lib is not None:
            _lib.lib().ltb_batch_release(h)
            self._h = None
