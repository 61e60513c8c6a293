"""loop_tool_b200: a B200 (sm_100a) "cuda" backend for loop_tool.

Drop-in for the reference's deprecated NVRTC backend
(src/backends/cuda/cuda.cpp): same plugin surface (Backend -> Compiled,
Compiled.run(memory, sync)), with loop trees passed as serialized IR.
"""
from ._lib import LoopToolError  # noqa: F401
from .backend import (Batch, Compiled, RawTensor, cuda, device_count, plan,  # noqa: F401
                      tune_batch, tune_clear, tune_entries, tune_load, tune_save)

__all__ = ["Batch", "Compiled", "RawTensor", "cuda", "device_count", "plan", "LoopToolError",
           "tune_save", "tune_load", "tune_clear", "tune_entries", "tune_batch"]
