"""Annotated loop trees on the GPU: "[cuda]" sub-trees (the reference's
route to a backend for one sub-tree, compile.cpp:404-417) run as device
launches with the rest of the tree, through the C ABI and through the
reference's own Backend registry with the plugin; "parallel" pins give the
same values; a tuned schedule written back as annotations
(ltb_schedule_ir) compiles to the same launch choices and the same bits."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from golden_util import (GOLDEN, EXACT_PROGRAMS, assert_accuracy, assert_parity, bits_equal,
                         fp64_oracle, load)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "libloop_tool_cuda_b200.so")
ANNOTATED = json.load(open(os.path.join(GOLDEN, "annotated_cuda.json")))


def check(got, case, name):
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(ANNOTATED))
def test_cuda_subtree_through_the_abi(name, cuda_dev):
    import torch

    import loop_tool_b200 as lt

    case = load(name)
    for depth, ir in sorted(ANNOTATED[name].items()):
        c = lt.cuda(ir)
        assert "[cuda] sub-tree" in c.code
        ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
        out = torch.full((c.io_sizes[-1],), 1337.0, device=cuda_dev)
        c(ins + [out])
        torch.cuda.synchronize()
        check(out.cpu().numpy(), case, f"{name} [cuda]@{depth}")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["add_4099", "softmax_16x4096", "mm_200x130x70",
                                  "conv_2x4x8x8_pad1", "colsum_300x37", "maxpool_specials"])
def test_cuda_subtree_through_the_reference_registry(name, cuda_dev):
    """The reference deserializes the annotated tree and hands it to the
    backend registered as "cuda" (the plugin): Backend::compile + run."""
    if not (os.path.exists(HARNESS) and os.path.exists(PLUGIN)):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    case = load(name)
    for depth, ir in sorted(ANNOTATED[name].items()):
        with tempfile.TemporaryDirectory() as td:
            for i, a in enumerate(case["inputs"]):
                a.tofile(os.path.join(td, f"in{i}.f32"))
            irf = os.path.join(td, "ir.txt")
            open(irf, "w").write(ir)
            env = dict(os.environ, LT_PLUGIN=PLUGIN)
            r = subprocess.run([HARNESS, "run", irf, "cuda", td, td], env=env,
                               capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
            got = np.fromfile(os.path.join(td, "out0.f32"), dtype=np.float32)
        check(got, case, f"{name} [cuda]@{depth} via plugin")


@pytest.mark.gpu
def test_parallel_pins_keep_values(cuda_dev):
    import torch

    import loop_tool_b200 as lt
    from test_cpu_annotations import tutorial_add

    ir = tutorial_add(n=(1 << 20) + 37)
    c = lt.cuda(ir)
    assert "pinned{ parallel=8192 }" in c.code
    n = c.io_sizes[-1]
    g = torch.Generator(device=cuda_dev).manual_seed(3)
    a, b = (torch.randn(n, device=cuda_dev, generator=g) for _ in range(2))
    out = torch.empty(n, device=cuda_dev)
    c([a, b, out])
    torch.cuda.synchronize()
    assert torch.equal(out, a + b)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["add_4099", "rowsum_37x300", "colsum_300x37", "maxpool_2x3x8x8",
                                  "layernorm_8x256"])
def test_tuned_schedule_round_trips_as_annotations(name, cuda_dev):
    import torch

    import loop_tool_b200 as lt

    case = load(name)
    c = lt.Compiled(case["ir"])
    ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    out = torch.empty(c.io_sizes[-1], device=cuda_dev)
    c.tune(ins + [out], reps=3)
    ref = out.clone()
    text = c.schedule_ir()
    c2 = lt.Compiled(text)
    for i in range(c2.int_property("stages")):
        s1, s2 = c.schedule(i), c2.schedule(i)
        if s1[1] > 0 and "pinned" in c2.code.splitlines()[1 + i]:
            assert s2[1] == s1[1], (i, s1, s2)  # the tuned CTA size, now pinned
    out2 = torch.empty_like(out)
    c2(ins + [out2])
    torch.cuda.synchronize()
    assert bits_equal(out2.cpu().numpy(), ref.cpu().numpy())
    check(out2.cpu().numpy(), case, name + " (schedule from annotations)")
