"""The configurations at their full sizes, checked through properties that do
not need the CPU oracle to finish: elementwise add and max-pool are exact
operations, so the B200 result must equal the same operation done by torch
bit for bit; softmax, convolution and the 8192^3 matmul are compared with
FP64 results (softmax on every element, the contractions normwise on sampled
outputs).  The loop trees are built with the lazy frontend exactly as the
benchmark builds them, and run with autotuned schedules."""
import math

import numpy as np
import pytest


def _run(ir, bufs, tune=True, **opts):
    import torch

    import loop_tool_b200 as ltb

    c = ltb.Compiled(ir, **opts)
    if tune:
        c.tune(bufs, reps=2)
    for t in bufs[c.n_inputs:]:
        t.fill_(float("nan"))
    c(bufs)
    torch.cuda.synchronize()
    return c


@pytest.mark.gpu
def test_add_2p28_bit_exact(cuda_dev):
    import torch

    import loop_tool_b200.lazy as lt

    n = 1 << 28
    A, B = lt.Tensor(n), lt.Tensor(n)
    N = lt.Symbol("N")
    g = torch.Generator(device=cuda_dev).manual_seed(201)
    a = torch.randn(n, device=cuda_dev, generator=g)
    b = torch.randn(n, device=cuda_dev, generator=g)
    c = torch.empty(n, device=cuda_dev)
    _run((A.to(N) + B.to(N)).ir, [a, b, c])
    assert torch.equal(c, a + b)


@pytest.mark.gpu
def test_maxpool_64x128x112x112_bit_exact(cuda_dev):
    import torch

    import loop_tool_b200.lazy as lt
    import loop_tool_b200.nn as nn

    P = lt.Tensor(64, 128, 112, 112)
    b, ch, h, w = (lt.Symbol(s) for s in "nchw")
    ir = nn.maxpool(P.to(b, ch, h, w), [h, w], 2, 2).ir
    g = torch.Generator(device=cuda_dev).manual_seed(221)
    x = torch.randn(64 * 128 * 112 * 112, device=cuda_dev, generator=g)
    y = torch.empty(64 * 128 * 56 * 56, device=cuda_dev)
    _run(ir, [x, y])
    ref = torch.nn.functional.max_pool2d(x.view(64, 128, 112, 112), 2, 2)
    assert torch.equal(y.view(64, 128, 56, 56), ref)


@pytest.mark.gpu
def test_softmax_8192x4096_vs_fp64(cuda_dev):
    import torch

    import loop_tool_b200.lazy as lt

    X = lt.Tensor(8192, 4096)
    r, n = lt.Symbol("r"), lt.Symbol("n")
    x = X.to(r, n)
    e = (x - x.max_reduce(n)).exp()
    g = torch.Generator(device=cuda_dev).manual_seed(211)
    xs = 4 * torch.randn(8192 * 4096, device=cuda_dev, generator=g)
    y = torch.empty_like(xs)
    _run((e / e.sum(n)).ir, [xs, y])
    ref = torch.softmax(xs.view(8192, 4096).double(), dim=1)
    err = (y.view(8192, 4096).double() - ref).abs()
    # every element within FP32 rounding of its FP64 value (relative)
    assert float((err / ref.clamp_min(1e-30)).max()) < 1e-5
    assert float(y.view(8192, 4096).double().sum(1).sub(1).abs().max()) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp32", 1e-6), ("bf16x3", 1.5e-5), ("bf16", 1.5e-2)])
def test_conv_32x64x56x56_vs_fp64(precision, tol, cuda_dev):
    import torch

    from loop_tool_b200.serve import _program

    ir = _program("conv", (32,)).ir
    g = torch.Generator(device=cuda_dev).manual_seed(301)
    x = torch.randn(32 * 64 * 56 * 56, device=cuda_dev, generator=g)
    bound = math.sqrt(6.0 / 576)
    w = (torch.rand(128 * 64 * 9, device=cuda_dev, generator=g) * 2 - 1) * bound
    y = torch.empty(32 * 56 * 56 * 128, device=cuda_dev)
    _run(ir, [x, w, y], precision=precision)
    ref = torch.nn.functional.conv2d(x.view(32, 64, 56, 56).double(),
                                     w.view(128, 64, 3, 3).double(), padding=1)
    got = y.view(32, 56, 56, 128).permute(0, 3, 1, 2).double()  # output is [n, ho, wo, co]
    err = float((got - ref).norm() / ref.norm())
    assert err <= tol, f"{precision}: normwise error {err:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("bf16x3", 1.5e-5), ("bf16", 1.5e-2)])
def test_mm_8192_sampled_vs_fp64(precision, tol, cuda_dev):
    import torch

    import loop_tool_b200.lazy as lt

    n = 8192
    A, B = lt.Tensor(n, n), lt.Tensor(n, n)
    m, k, j = lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
    ir = (A.to(m, k) * B.to(k, j)).sum(k).ir
    g = torch.Generator(device=cuda_dev).manual_seed(402)
    a = torch.randn(n * n, device=cuda_dev, generator=g) / math.sqrt(n)
    b = torch.randn(n * n, device=cuda_dev, generator=g)
    c = torch.empty(n * n, device=cuda_dev)
    _run(ir, [a, b, c], precision=precision)
    rng = np.random.default_rng(3)
    rows = torch.from_numpy(rng.integers(0, n, 256)).to(cuda_dev)
    cols = torch.from_numpy(rng.integers(0, n, 256)).to(cuda_dev)
    A2, B2, C2 = a.view(n, n), b.view(n, n), c.view(n, n)
    ref = (A2[rows].double() @ B2[:, cols].double())
    got = C2[rows][:, cols].double()
    err = float((got - ref).norm() / ref.norm())
    assert err <= tol, f"{precision}: sampled normwise error {err:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["add", "exp"])
def test_host_buffers_pipelined(op, cuda_dev):
    """Host-buffer runs of a linear map large enough to be staged chunk by
    chunk on two streams (and asynchronous with sync=False): the result is
    bit-identical to the same loop tree run on device buffers, for pinned
    and pageable host memory."""
    import torch

    import loop_tool_b200 as ltb
    import loop_tool_b200.lazy as lt

    n = (1 << 25) + 12344  # two full 2^24 chunks and a ragged third
    A, B = lt.Tensor(n), lt.Tensor(n)
    N = lt.Symbol("N")
    T = A.to(N) + B.to(N) if op == "add" else A.to(N).exp()
    c = ltb.Compiled(T.ir)
    g = torch.Generator(device=cuda_dev).manual_seed(5)
    dev_in = [torch.randn(n, device=cuda_dev, generator=g) for _ in range(c.n_inputs)]
    dev_out = torch.empty(n, device=cuda_dev)
    c(dev_in + [dev_out])
    ref = dev_out.cpu()
    pinned = [x.cpu().pin_memory() for x in dev_in] + [torch.full((n,), float("nan")).pin_memory()]
    c.run(pinned, sync=False)
    torch.cuda.synchronize()
    assert torch.equal(pinned[-1], ref)
    pageable = [x.cpu().numpy() for x in dev_in] + [np.full(n, np.nan, np.float32)]
    c(pageable)
    assert np.array_equal(pageable[-1], ref.numpy())
