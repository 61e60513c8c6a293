"""Captured runs (one CUDA graph per compiled loop tree on fixed buffers) and
concurrent runs of one compiled object from several host threads."""
import threading

import numpy as np
import pytest

from programs import conv, mm, softmax


def _fullsum():
    import loop_tool_b200.lazy as lt

    X = lt.Tensor(2, 300000)
    a, b = lt.Symbol("a"), lt.Symbol("b")
    return X.to(a, b).sum(a, b)


CASES = {
    "softmax": lambda: (softmax(256, 4096)[0], {}),
    "mm_bf16x3": lambda: (mm(200, 130, 70)[0], {"precision": "bf16x3"}),
    "mm_fp32": lambda: (mm(64, 96, 80)[0], {}),
    "conv_implicit": lambda: (conv(2, 64, 16, 16, 40, 3, 1, 1)[0], {"precision": "bf16"}),
    "fullsum_splitk": lambda: (_fullsum(), {}),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_captured_run_matches_plain_run(name, cuda_dev):
    import torch

    import loop_tool_b200 as ltb

    T, opts = CASES[name]()
    c = ltb.Compiled(T.ir, **opts)
    g = torch.Generator(device=cuda_dev).manual_seed(3)
    ins = [torch.randn(n, device=cuda_dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
    out = torch.empty(c.io_sizes[-1], device=cuda_dev)
    stream = torch.cuda.Stream()
    graph = c.capture(ins + [out], stream=stream.cuda_stream)
    for trial in range(2):  # the replay reads the buffers' current contents
        for x in ins:
            x.normal_(generator=g)
        out.fill_(float("nan"))
        graph.run(stream=stream.cuda_stream)
        torch.cuda.synchronize()
        got = out.clone()
        ref = torch.empty_like(out)
        c(ins + [ref])
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (name, trial)


@pytest.mark.gpu
def test_threads_share_one_compiled_object(cuda_dev):
    """Four host threads run the same compiled loop tree on their own streams
    with their own scratch; every result equals the single-thread one."""
    import torch

    import loop_tool_b200 as ltb

    T, _ = mm(256, 192, 320)
    c = ltb.Compiled(T.ir, precision="bf16x3")
    g = torch.Generator(device=cuda_dev).manual_seed(8)
    jobs = []
    for _ in range(4):
        ins = [torch.randn(n, device=cuda_dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
        ref = torch.empty(c.io_sizes[-1], device=cuda_dev)
        c(ins + [ref])
        jobs.append((ins, ref))
    torch.cuda.synchronize()
    errors = []

    def worker(ins, ref):
        try:
            st = torch.cuda.Stream()
            sb = c.int_property("scratch_bytes")
            scratch = torch.empty(max(sb // 4, 1), device=cuda_dev)
            out = torch.empty_like(ref)
            for _ in range(20):
                with torch.cuda.stream(st):
                    c.run(ins + [out], sync=True, stream=st.cuda_stream,
                          scratch=scratch.data_ptr())
                if not torch.equal(out, ref):
                    errors.append("mismatch")
                    return
        except Exception as e:  # reported in the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=j) for j in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


@pytest.mark.gpu
def test_kernel_cache_is_thread_safe(cuda_dev):
    """Concurrent lookups of one IR text get one compiled object."""
    import loop_tool_b200.lazy as lt

    T, _ = mm(48, 32, 16)
    ir = T.ir
    lt.clear_cache()
    got = []
    threads = [threading.Thread(target=lambda: got.append(lt.compiled(ir))) for _ in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert len({id(c) for c in got}) == 1 and lt.cache_info()["entries"] == 1
