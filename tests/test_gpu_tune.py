"""The autotuner: every candidate schedule computes the same loop tree, the
chosen one is cached by IR text + options and reapplied at compile time,
and the cache survives a save / clear / load round trip."""
import numpy as np
import pytest

from golden_util import fp64_oracle, load
from programs import mm, softmax

TOL = {"bf16x3": 1.5e-5, "bf16": 1.5e-2}


def _bufs(c, dev, seed):
    import torch

    g = torch.Generator(device=dev).manual_seed(seed)
    ins = [torch.randn(n, device=dev, generator=g) for n in c.io_sizes[:c.n_inputs]]
    return ins + [torch.full((n,), float("nan"), device=dev) for n in c.io_sizes[c.n_inputs:]]


@pytest.mark.gpu
def test_tune_elementwise_exact_and_cached(cuda_dev, tmp_path):
    import torch

    import loop_tool_b200 as ltb
    import loop_tool_b200.lazy as lt

    ltb.tune_clear()
    A, B = lt.Tensor(1 << 20), lt.Tensor(1 << 20)
    n = lt.Symbol("n")
    ir = (A.to(n) + B.to(n)).ir
    c = ltb.Compiled(ir)
    assert c.int_property("tuned") == 0
    bufs = _bufs(c, cuda_dev, 1)
    report = c.tune(bufs, reps=3)
    assert "stage 0" in report and "parallel(" in report
    torch.cuda.synchronize()
    assert torch.equal(bufs[2], bufs[0] + bufs[1])  # bit-exact under the tuned schedule
    sched = c.schedule(0)
    assert ltb.tune_entries() == 1
    c2 = ltb.Compiled(ir)  # the cache applies the schedule at compile time
    assert c2.int_property("tuned") == 1 and c2.schedule(0) == sched
    assert ltb.Compiled(ir, precision="bf16").int_property("tuned") == 0  # options are in the key
    path = tmp_path / "schedules.txt"
    ltb.tune_save(path)
    ltb.tune_clear()
    assert ltb.Compiled(ir).int_property("tuned") == 0
    ltb.tune_load(path)
    c3 = ltb.Compiled(ir)
    assert c3.int_property("tuned") == 1 and c3.schedule(0) == sched
    ltb.tune_clear()


@pytest.mark.gpu
@pytest.mark.parametrize("cols", [4096, 4094, 1000])
def test_every_softmax_schedule_agrees(cols, cuda_dev):
    """Each candidate (elements x threads, register or bulk-copy staging,
    grid) of the row-softmax chain, set by hand, gives results within FP32
    rounding of the FP64 oracle; bulk variants on rows that are not 16-byte
    aligned (4094 columns) fall back to the register form."""
    import torch

    import loop_tool_b200 as ltb

    T, _ = softmax(300, cols)
    c = ltb.Compiled(T.ir)
    bufs = _bufs(c, cuda_dev, 2)
    x = bufs[0].cpu().numpy().reshape(300, cols).astype(np.float64)
    e = np.exp(x - x.max(1, keepdims=True))
    exact = e / e.sum(1, keepdims=True)
    for variant in range(1, 18):
        for w in (0, 2, 8):
            c.set_schedule(0, cta_per_sm=w, variant=variant)
            bufs[1].fill_(float("nan"))
            c(bufs)
            torch.cuda.synchronize()
            got = bufs[1].cpu().numpy().reshape(300, cols)
            err = np.abs(got - exact).max() / np.abs(exact).max()
            assert err < 1e-6, (variant, w, err)
    ltb.tune_clear()


@pytest.mark.gpu
@pytest.mark.parametrize("shape,k,st", [((3, 5, 112, 112), 2, 2), ((2, 3, 37, 42), 2, 2),
                                        ((2, 4, 30, 30), 3, 3), ((1, 2, 17, 21), 3, 2)])
def test_every_pool_schedule_exact(shape, k, st, cuda_dev):
    """Max-pool through the window kernel with 2 and 4 work items per thread
    (variant 0 / 4), every grid and CTA size: bit-identical to torch's
    max_pool2d, ragged rows and partial vectors included."""
    import torch

    import loop_tool_b200 as ltb
    from programs import maxpool

    N, C, H, W = shape
    T, _ = maxpool(N, C, H, W, k, st)
    c = ltb.Compiled(T.ir)
    g = torch.Generator(device=cuda_dev).manual_seed(H * W + k)
    x = torch.randn(N * C * H * W, device=cuda_dev, generator=g)
    ref = torch.nn.functional.max_pool2d(x.view(N, C, H, W), k, st).flatten()
    y = torch.empty(c.io_sizes[-1], device=cuda_dev)
    assert y.numel() == ref.numel()
    for variant in (0, 4):
        for w in (0, 1, 8):
            for t in (128, 256):
                c.set_schedule(0, cta_per_sm=w, threads=t, variant=variant)
                y.fill_(float("nan"))
                c([x, y])
                torch.cuda.synchronize()
                assert torch.equal(y, ref), (variant, w, t)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
@pytest.mark.parametrize("name", ["mm_200x130x70", "conv_2x4x8x8_pad1", "bmm_3x16x8x24"])
def test_tile_widths_agree(name, precision, cuda_dev):
    import torch

    import loop_tool_b200 as ltb

    case = load(name)
    exact = fp64_oracle(case)
    c = ltb.cuda(case["ir"], precision=precision)
    ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    stage = [i for i in range(c.int_property("stages")) if c.schedule(i)[2] in (128, 256)][0]
    # tile width (+1: shared-memory transposed epilogue) x raster group
    for bn, gm in ((128, 0), (129, 8), (130, 0), (130, 16), (256, 32), (257, 0), (256, 1),
                   (258, 0), (258, 4)):
        c.set_schedule(stage, cta_per_sm=gm, variant=bn)
        assert c.schedule(stage) == (gm, 0, bn)
        out = torch.full((c.io_sizes[-1],), float("nan"), device=cuda_dev)
        c(ins + [out])
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
        assert err <= TOL[precision], (bn, err)


@pytest.mark.gpu
def test_tuned_batch_matches_fp64(cuda_dev):
    import torch

    import loop_tool_b200 as ltb

    sizes = [(64, 96, 48), (300, 128, 64), (128, 700, 80), (16, 16, 16), (512, 257 // 16 * 16, 32)]
    g = torch.Generator(device=cuda_dev).manual_seed(11)
    members = []
    for M, N, K in sizes:
        T, _ = mm(M, K, N)
        c = ltb.Compiled(T.ir, precision="bf16x3")
        members.append((c, [torch.randn(M * K, device=cuda_dev, generator=g),
                            torch.randn(K * N, device=cuda_dev, generator=g),
                            torch.full((M * N,), float("nan"), device=cuda_dev)]))
    stream = torch.cuda.Stream()
    b, best, report = ltb.tune_batch(members, capture_stream=stream.cuda_stream)
    assert best in report
    b.run(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    for (c, (A, B, C)), (M, N, K) in zip(members, sizes):
        exact = (A.cpu().numpy().reshape(M, K).astype(np.float64) @
                 B.cpu().numpy().reshape(K, N).astype(np.float64))
        err = np.linalg.norm(C.cpu().numpy().reshape(M, N) - exact) / np.linalg.norm(exact)
        assert err <= TOL["bf16x3"], ((M, N, K), err)
    ltb.tune_clear()
