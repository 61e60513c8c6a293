"""Batches of uneven matmuls in one grouped launch captured into a CUDA
graph (the batched form of the contraction family): every problem's result
is checked against FP64, in each precision mode."""
import numpy as np
import pytest

from programs import mm

TOL = {"bf16x3": 1.5e-5, "bf16": 1.5e-2, "fp32": 1e-5}


def uneven_sizes(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    v = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(n, 3)))
    return [tuple(int(max(16, 16 * round(x / 16))) for x in row) for row in v]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "bf16", "fp32"])
def test_batch_of_uneven_matmuls(precision, cuda_dev):
    import torch

    import loop_tool_b200 as ltb

    sizes = uneven_sizes(24, 16, 600, seed=401)
    sizes[0] = (17 * 16, 5 * 16, 3 * 16)  # tails in M, N and K tiles
    g = torch.Generator(device=cuda_dev).manual_seed(5)
    members, host = [], []
    for M, N, K in sizes:
        T, _ = mm(M, K, N)
        c = ltb.Compiled(T.ir, precision=precision)
        A = torch.randn(M * K, device=cuda_dev, generator=g) / K ** 0.5
        B = torch.randn(K * N, device=cuda_dev, generator=g)
        C = torch.full((M * N,), float("nan"), device=cuda_dev)
        members.append((c, [A, B, C]))
        host.append((M, N, K))
    stream = torch.cuda.Stream()
    b = ltb.Batch(members, capture_stream=stream.cuda_stream)
    assert b.int_property("graph") == 1 and b.int_property("problems") == len(sizes)
    for _ in range(2):  # replay twice: results must not depend on the replay
        b.run(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    for (c, (A, B, C)), (M, N, K) in zip(members, host):
        a = A.cpu().numpy().reshape(M, K).astype(np.float64)
        bb = B.cpu().numpy().reshape(K, N).astype(np.float64)
        exact = a @ bb
        got = C.cpu().numpy().reshape(M, N)
        assert np.isfinite(got).all(), f"{(M, N, K)}: unwritten outputs"
        err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
        assert err <= TOL[precision], f"{(M, N, K)} {precision}: normwise error {err:.3g}"


@pytest.mark.gpu
def test_pack_schedules_agree_bit_for_bit(cuda_dev):
    """Every launch shape of the grouped operand packing (tile chunk dealt
    per CTA, CTAs per SM) packs the same bits: results are identical."""
    import torch

    import loop_tool_b200 as ltb

    sizes = uneven_sizes(12, 16, 700, seed=402)
    g = torch.Generator(device=cuda_dev).manual_seed(6)
    members = []
    for M, N, K in sizes:
        T, _ = mm(M, K, N)
        members.append((ltb.Compiled(T.ir, precision="bf16x3"),
                        [torch.randn(M * K, device=cuda_dev, generator=g),
                         torch.randn(K * N, device=cuda_dev, generator=g),
                         torch.empty(M * N, device=cuda_dev)]))
    stream = torch.cuda.Stream()
    b = ltb.Batch(members, capture_stream=stream.cuda_stream)
    b.run(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ref = [C.clone() for _, (_, _, C) in members]
    for chunk, per_sm in ((1, 4), (16, 2), (64, 8), (3, 1)):
        b.set_schedule(chunk, per_sm)
        assert b.int_property("graph") == 1 and b.int_property("pack_chunk") == chunk
        for _, (_, _, C) in members:
            C.fill_(float("nan"))
        b.run(stream=stream.cuda_stream)
        torch.cuda.synchronize()
        for r, (_, (_, _, C)) in zip(ref, members):
            assert torch.equal(r, C), (chunk, per_sm)
