"""ctypes binding of libloop_tool_b200.so (the C ABI in include/loop_tool_b200.h).

The shared library is built in-tree (loop_tool_b200/_lib/) by
``python -m loop_tool_b200.build``.  Importing this module without it raises:
there is no CPU fallback for the CUDA path.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libloop_tool_b200.so")

OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_NO_DEVICE = 4
ERR_TIMEOUT = 5

# The serving structures of include/loop_tool_b200.h ("serving").
LTB_SERVE_MAX_IO = 8


class LtbBlock(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
                ("true_rows", ctypes.c_int64), ("true_cols", ctypes.c_int64),
                ("scale", ctypes.c_float)]


class LtbRequest(ctypes.Structure):
    _fields_ = [("ir_text", ctypes.c_char_p), ("arrival_s", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("n_io", ctypes.c_int),
                ("io", LtbBlock * LTB_SERVE_MAX_IO), ("host_out", ctypes.POINTER(ctypes.c_float))]


class LtbServeStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_int64), ("compiles", ctypes.c_int64),
                ("peak_inflight", ctypes.c_int64), ("peak_bytes", ctypes.c_int64),
                ("span_s", ctypes.c_double), ("req_per_s", ctypes.c_double),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("compile_s", ctypes.c_double)]


# every symbol include/loop_tool_b200.h declares, with its ctypes signature
SIGNATURES = {
    "ltb_abi_version": (ctypes.c_int, []),
    "ltb_last_error": (ctypes.c_char_p, []),
    "ltb_device_count": (ctypes.c_int, []),
    "ltb_plan": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ltb_compile": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "ltb_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                               ctypes.c_int, ctypes.c_void_p]),
    "ltb_run_with_scratch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "ltb_run_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "ltb_release": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_dump": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ltb_int_property": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                        ctypes.POINTER(ctypes.c_int64)]),
    "ltb_io_sizes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64),
                                    ctypes.c_int]),
    "ltb_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "ltb_free": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_check_bounded_wait": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    "ltb_row_sum_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ltb_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.POINTER(ctypes.c_void_p)),
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "ltb_batch_capture": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ltb_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "ltb_batch_int_property": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p,
                                              ctypes.POINTER(ctypes.c_int64)]),
    "ltb_batch_release": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_batch_run_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_float)]),
    "ltb_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "ltb_get_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]),
    "ltb_set_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]),
    "ltb_tune_record": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_schedule_ir": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "ltb_batch_set_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "ltb_graph_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "ltb_graph_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "ltb_graph_release": (ctypes.c_int, [ctypes.c_void_p]),
    "ltb_tune_save": (ctypes.c_int, [ctypes.c_char_p]),
    "ltb_tune_load": (ctypes.c_int, [ctypes.c_char_p]),
    "ltb_tune_clear": (ctypes.c_int, []),
    "ltb_tune_entries": (ctypes.c_int64, []),
    "ltb_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_char_p,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "ltb_server_prepare": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LtbRequest), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int64)]),
    "ltb_server_serve": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LtbRequest), ctypes.c_int,
                                        ctypes.c_double, ctypes.POINTER(LtbServeStats),
                                        ctypes.POINTER(ctypes.c_double)]),
    "ltb_server_release": (ctypes.c_int, [ctypes.c_void_p]),
}


class LoopToolError(RuntimeError):
    """Raised for every failed call, like the reference's ASSERT throwing
    std::runtime_error (include/loop_tool/error.h:47-61)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA extension with "
                "`python -m loop_tool_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != OK:
        msg = lib().ltb_last_error().decode(errors="replace")
        raise LoopToolError(rc, msg)
    return rc
