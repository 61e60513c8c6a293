"""Device-side robustness: bounded waits that give up cleanly, buffers off a
16-byte boundary, and runs of one compiled object on its own (default)
scratch from several threads and streams at once.  None of these tests
faults or hangs the GPU: the wait that runs out is a bounded wait on a
barrier nothing arrives at, and misaligned buffers are staged on the host
side's decision (checked through run_plan before anything runs)."""
import ctypes
import threading

import numpy as np
import pytest

from golden_util import bits_equal, fp64_oracle, load
from programs import mm

LTB_ERR_TIMEOUT = 5


def _stream_ptr(st):
    return ctypes.c_void_p(st.cuda_stream)


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_the_device_stays_usable(cuda_dev):
    import torch

    import loop_tool_b200 as lt
    from loop_tool_b200 import _lib

    L = _lib.lib()
    st = torch.cuda.Stream()
    for _ in range(2):  # the flag is cleared by the report: the check repeats
        done, drained = ctypes.c_int(-1), ctypes.c_int(-1)
        rc = L.ltb_check_bounded_wait(2000, _stream_ptr(st), ctypes.byref(done),
                                      ctypes.byref(drained))
        assert rc == LTB_ERR_TIMEOUT, (rc, L.ltb_last_error())
        assert done.value == 0 and drained.value == 1
    # reported once: the stream's next synchronisation is clean
    assert L.ltb_synchronize(_stream_ptr(st)) == 0
    # the TMEM was freed and the context is intact: a tensor-core run on the
    # same stream allocates TMEM on the SMs and computes the right result
    case = load("mm_128")
    c = lt.cuda(case["ir"], precision="bf16")
    ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    out = torch.full((c.io_sizes[-1],), float("nan"), device=cuda_dev)
    with torch.cuda.stream(st):
        c.run(ins + [out], sync=True, stream=st.cuda_stream)
    got = out.cpu().numpy().astype(np.float64)
    exact = fp64_oracle(case).ravel()
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < 1.5e-2


@pytest.mark.gpu
@pytest.mark.parametrize("name,precision", [("add_4099", None), ("softmax_16x4096", None),
                                            ("maxpool_2x3x8x8", None), ("mm_128", "bf16x3"),
                                            ("conv_2x4x8x8_pad1", None), ("pad2d_128x16", None)])
def test_misaligned_buffers_are_staged(name, precision, cuda_dev):
    """Views one element into a tensor (4-byte offset) give the same bits
    as aligned buffers: run_plan shows them staged, nothing reads them with
    16-byte vectors in place."""
    import torch

    import loop_tool_b200 as lt

    case = load(name)
    opts = {"precision": precision} if precision else {}
    c = lt.cuda(case["ir"], **opts)
    aligned = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    ref = torch.full((c.io_sizes[-1],), 1337.0, device=cuda_dev)
    c(aligned + [ref])
    backing = [torch.zeros(a.numel() + 1, device=cuda_dev) for a in aligned]
    views = []
    for b, a in zip(backing, aligned):
        b[1:].copy_(a)
        views.append(b[1:])
    out_backing = torch.full((c.io_sizes[-1] + 1,), 1337.0, device=cuda_dev)
    out = out_backing[1:]
    assert all(v.data_ptr() % 16 == 4 for v in views + [out])
    plan = c.run_plan(views + [out])
    assert all("off a 16-byte boundary" in line for line in plan), plan
    c(views + [out])
    torch.cuda.synchronize()
    assert bits_equal(out.cpu().numpy(), ref.cpu().numpy())
    assert out_backing[0].item() == 1337.0  # nothing written before the view


@pytest.mark.gpu
def test_foreign_and_aligned_buffers_in_run_plan(cuda_dev):
    import torch

    import loop_tool_b200 as lt

    case = load("add_1000")
    c = lt.cuda(case["ir"])
    dev = [torch.zeros(1000, device=cuda_dev) for _ in range(3)]
    host = np.zeros(1000, np.float32)
    plan = c.run_plan([dev[0], host, dev[2]])
    assert "in place" in plan[0] and "host memory" in plan[1] and "in place" in plan[2]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", None])
def test_threads_and_streams_share_the_default_scratch(precision, cuda_dev):
    """4 threads x 20 asynchronous runs on 4 streams of one compiled object
    that needs scratch (packed tensor-core operands, or the intermediates of
    a layer norm), none bringing caller scratch: each result equals the
    single-thread result bit for bit."""
    import torch

    import loop_tool_b200 as lt

    if precision:
        T, _ = mm(256, 192, 320)
        c = lt.Compiled(T.ir, precision=precision)
    else:
        c = lt.Compiled(load("layernorm_8x256")["ir"])
    assert c.int_property("scratch_bytes") > 0
    g = torch.Generator(device=cuda_dev).manual_seed(9)
    jobs = []
    for _ in range(4):
        ins = [torch.randn(n, device=cuda_dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
        if not precision:  # element count and eps of the layer norm
            ins[1].fill_(256.0)
            ins[2].fill_(1e-5)
        ref = torch.empty(c.io_sizes[-1], device=cuda_dev)
        c(ins + [ref])
        jobs.append((ins, ref))
    torch.cuda.synchronize()
    errors = []
    barrier = threading.Barrier(4)

    def worker(ins, ref):
        try:
            st = torch.cuda.Stream()
            outs = [torch.empty_like(ref) for _ in range(20)]
            barrier.wait()
            for o in outs:
                c.run(ins + [o], sync=False, stream=st.cuda_stream)
            st.synchronize()
            if not all(torch.equal(o, ref) for o in outs):
                errors.append("mismatch")
        except Exception as e:  # reported in the main thread
            errors.append(repr(e))

    threads = [threading.Thread(target=worker, args=j) for j in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
