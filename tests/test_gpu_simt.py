"""The FP32 CUDA-core contraction (the default precision) through each of its
operand tile loader forms: 16-byte loads along k (row-major A, k-contiguous
transposed B), 16-byte loads along rows (row-major B, transposed A) and the
gather form (tables, guards, ragged or unaligned operands).  Every layout is
checked against the FP64 oracle; and since every output is one FP32 FMA
chain over k in order, the same product read through a vector form and
through the gather form (an operand buffer offset by one element, which
rules out 16-byte loads) must agree bit for bit.  Problems with few
128 x 128 tiles run 64 x 64 tiles by default; the large shapes below take
the 128-wide loader forms."""
import numpy as np
import pytest

# (layout, M, K, N): "n" = operand stored as in C = A[M,K] B[K,N], "t" =
# stored transposed.  Sizes cross the 128-row tiles and the 16-k steps, and
# include K, M, N not multiples of 4 (no vector form).
LAYOUTS = [("nn", 130, 68, 20), ("nn", 65, 37, 50), ("nn", 200, 36, 132), ("nn", 1, 300, 8),
           ("tn", 132, 36, 68), ("tn", 67, 20, 30), ("nt", 130, 68, 20), ("nt", 33, 19, 129),
           ("tt", 64, 40, 100), ("tt", 9, 7, 5), ("nn", 257, 1000, 260),
           ("nn", 1664, 36, 1540), ("tn", 1540, 20, 1664), ("nt", 1500, 37, 1500)]


def _program(layout, M, K, N):
    import loop_tool_b200.lazy as lt

    A = lt.Tensor(M, K) if layout[0] == "n" else lt.Tensor(K, M)
    B = lt.Tensor(K, N) if layout[1] == "n" else lt.Tensor(N, K)
    m, k, n = lt.Symbol("m"), lt.Symbol("k"), lt.Symbol("n")
    a = A.to(m, k) if layout[0] == "n" else A.to(k, m)
    b = B.to(k, n) if layout[1] == "n" else B.to(n, k)
    return (a * b).sum(k).ir


def _oracle(ir, ins):
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
    import np_oracle

    return np_oracle.evaluate(ir, [a.astype(np.float64) for a in ins], dtype=np.float64)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("case", LAYOUTS, ids=lambda c: "%s_%dx%dx%d" % c)
def test_fp32_layouts_vs_oracle_and_forms(case, cuda_dev):
    import torch

    import loop_tool_b200 as ltb

    layout, M, K, N = case
    ir = _program(layout, M, K, N)
    c = ltb.Compiled(ir)
    assert "contraction" in c.code
    g = torch.Generator(device=cuda_dev).manual_seed(M * 31 + K * 7 + N)
    a = torch.randn(M * K + 1, device=cuda_dev, generator=g)
    b = torch.randn(K * N + 1, device=cuda_dev, generator=g)
    outs = []
    # aligned buffers (vector forms where the layout allows them), then the
    # same values one element into a larger buffer (gather form only)
    for off in (0, 1):
        if off:
            a2, b2 = torch.empty_like(a), torch.empty_like(b)
            a2[1:] = a[:-1]
            b2[1:] = b[:-1]
            ins = [a2[1:], b2[1:]]
        else:
            ins = [a[:-1], b[:-1]]
        out = torch.full((M * N,), float("nan"), device=cuda_dev)
        c(ins + [out])
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    assert np.isfinite(outs[0]).all()
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32)), \
        "vector and gather tile loaders disagree"
    exact = _oracle(ir, [a[:-1].cpu().numpy(), b[:-1].cpu().numpy()]).ravel()
    err = float(np.linalg.norm(outs[0] - exact) / np.linalg.norm(exact))
    assert err <= 1e-6, f"normwise error {err:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("case", [("nn", 130, 68, 20), ("nt", 33, 19, 129), ("tn", 67, 20, 30),
                                  ("nn", 1500, 70, 1300), ("tt", 200, 33, 1400)],
                         ids=lambda c: "%s_%dx%dx%d" % c)
def test_fp32_tile_sizes_same_bits(case, cuda_dev):
    """64 x 64 and 128 x 128 CUDA-core tiles (a tuned choice; small problems
    default to 64) run the same FMA chain per output: identical bits."""
    import torch

    import loop_tool_b200 as ltb

    layout, M, K, N = case
    c = ltb.Compiled(_program(layout, M, K, N))
    g = torch.Generator(device=cuda_dev).manual_seed(M + K + N)
    a = torch.randn(M * K, device=cuda_dev, generator=g)
    b = torch.randn(K * N, device=cuda_dev, generator=g)
    outs = []
    for tile in (64, 128):
        c.set_schedule(0, variant=tile)
        assert c.schedule(0)[2] == tile
        out = torch.full((M * N,), float("nan"), device=cuda_dev)
        c([a, b, out])
        torch.cuda.synchronize()
        outs.append(out)
    assert torch.isfinite(outs[0]).all()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(2, 4, 8, 8, 6, 3, 1), (1, 3, 7, 9, 5, 3, 0),
                                   (2, 64, 16, 16, 40, 3, 1), (4, 16, 33, 35, 24, 5, 2),
                                   (1, 160, 12, 12, 8, 3, 1)])
def test_fp32_conv_gather(shape, cuda_dev):
    """Padded convolution: the image operand is gathered with its guards
    (zero outside the image), the weights through 16-byte loads along k; on
    64-wide tiles element by element, on 128-wide tiles through the shared
    per-k table.  Both give the same bits."""
    import torch

    import loop_tool_b200 as ltb
    from programs import conv

    N, C, H, W, CO, K, pad = shape
    T, _ = conv(N, C, H, W, CO, K, pad, 1)
    c = ltb.Compiled(T.ir)
    g = torch.Generator(device=cuda_dev).manual_seed(sum(shape))
    x = torch.randn(N * C * H * W, device=cuda_dev, generator=g)
    w = torch.randn(CO * C * K * K, device=cuda_dev, generator=g)
    Ho, Wo = H + 2 * pad - K + 1, W + 2 * pad - K + 1
    ref = torch.nn.functional.conv2d(x.view(N, C, H, W).double(),
                                     w.view(CO, C, K, K).double(), padding=pad)
    outs = []
    for tile in (64, 128):
        c.set_schedule(0, variant=tile)
        y = torch.full((N * Ho * Wo * CO,), float("nan"), device=cuda_dev)
        c([x, w, y])
        torch.cuda.synchronize()
        got = y.view(N, Ho, Wo, CO).permute(0, 3, 1, 2).double()
        err = float((got - ref).norm() / ref.norm())
        assert err <= 1e-6, f"tile {tile}: normwise error {err:.3g}"
        outs.append(y)
    assert torch.equal(outs[0], outs[1])


@pytest.mark.gpu
def test_fp32_batch_mixed_forms(cuda_dev):
    """A grouped FP32 launch whose members allow different loader forms runs
    every member through the gather form; one whose members all allow the
    vector forms uses those; both give each member's single-launch bits."""
    import torch

    import loop_tool_b200 as ltb

    g = torch.Generator(device=cuda_dev).manual_seed(23)
    shapes = [("nn", 130, 68, 20), ("nn", 64, 32, 96), ("nt", 33, 19, 129), ("tn", 67, 20, 30)]
    members, singles = [], []
    for layout, M, K, N in shapes:
        c = ltb.Compiled(_program(layout, M, K, N))
        bufs = [torch.randn(M * K, device=cuda_dev, generator=g),
                torch.randn(K * N, device=cuda_dev, generator=g),
                torch.full((M * N,), float("nan"), device=cuda_dev)]
        ref = torch.empty(M * N, device=cuda_dev)
        c(bufs[:2] + [ref])
        members.append((c, bufs))
        singles.append(ref)
    for group in (members[:2], members):  # all vector-capable; mixed
        b = ltb.Batch(group)
        b.run()
        torch.cuda.synchronize()
        for (c, bufs), ref in zip(group, singles):
            assert torch.equal(bufs[2], ref)
        del b
