"""Parity of the B200 path with the reference on its own IR.

Each fixture holds the IR text the reference lazy frontend produced, seeded
inputs, and the reference's output (tests/golden/make_golden.py).  The IR
goes through the C ABI (ltb_compile / ltb_run) on cuda:0.
"""
import numpy as np
import pytest

from golden_util import EXACT_PROGRAMS, assert_accuracy, assert_parity, fp64_oracle, load, manifest


def check(got, case, name):
    """Bit-exact against the reference where its arithmetic is exact, else
    measured against the FP64 oracle (and never worse than the reference)."""
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)

CASES = [m["name"] for m in manifest()]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_golden_device_buffers(name, cuda_dev):
    import torch

    import loop_tool_b200 as lt

    case = load(name)
    c = lt.cuda(case["ir"])
    ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    out = torch.full((c.io_sizes[-1],), 1337.0, device=cuda_dev)
    c(ins + [out])
    torch.cuda.synchronize()
    check(out.cpu().numpy(), case, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["add_4099", "softmax_16x32", "maxpool_specials",
                                  "conv_2x4x8x8_pad1", "concat2d_kat"])
def test_golden_host_buffers(name, cuda_dev):
    """numpy-bound (host) buffers are staged through HBM, like the
    reference's Tensor.numpy() path (python.cpp:548-559)."""
    import loop_tool_b200 as lt

    case = load(name)
    c = lt.cuda(case["ir"])
    out = np.full(c.io_sizes[-1], 1337.0, np.float32)
    c([np.ascontiguousarray(a) for a in case["inputs"]] + [out])
    check(out, case, name)
