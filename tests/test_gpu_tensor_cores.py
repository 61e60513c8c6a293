"""Contractions on the tcgen05 tensor-core path.

BF16 inputs with FP32 accumulation ("bf16") and the split-BF16 three-product
mode ("bf16x3") are measured against the FP64 oracle: normwise relative
error ||C - C64|| / ||C64||.  bf16x3 must reach FP32-level accuracy (the
1e-5 target); bf16 is bounded by BF16's 8-bit significand.
"""
import os

import numpy as np
import pytest

from golden_util import fp64_oracle, load

CONTRACTIONS = ["mm_16", "mm_128", "mm_17x33x9", "mm_200x130x70", "bmm_3x16x8x24",
                "conv_2x4x8x8_pad1", "conv_1x3x7x9_nopad", "conv_2x3x9x9_s2"]
# measured normwise errors (N(0,1) inputs): bf16x3 ~1.0e-5 (the dropped
# Al*Bl term and the 2^-17 residual of each hi/lo split), bf16x4 ~7e-6
TOL = {"bf16x6": 1e-6, "bf16x4": 1e-5, "bf16x3": 1.5e-5, "bf16": 1.5e-2}


def normwise(got, exact):
    return float(np.linalg.norm(got.astype(np.float64) - exact) / np.linalg.norm(exact))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x6", "bf16x4", "bf16x3", "bf16"])
@pytest.mark.parametrize("name", CONTRACTIONS)
def test_tensor_core_contraction(name, precision, cuda_dev):
    import torch

    import loop_tool_b200 as lt

    case = load(name)
    c = lt.cuda(case["ir"], precision=precision)
    assert "contraction" in c.code
    ins = [torch.from_numpy(a).to(cuda_dev) for a in case["inputs"]]
    out = torch.full((c.io_sizes[-1],), float("nan"), device=cuda_dev)
    c(ins + [out])
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isfinite(got).all(), f"{name}: unwritten or non-finite outputs"
    err = normwise(got, fp64_oracle(case))
    assert err <= TOL[precision], f"{name} {precision}: normwise error {err:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x4", "bf16x3", "bf16", "fp32"])
def test_mm_2048_sampled(precision, cuda_dev):
    """A multi-tile matmul (2048 x 2048 x 2048 from the reference's IR
    format) checked on sampled entries against FP64 dot products."""
    import torch

    import loop_tool_b200 as lt

    ir = open(os.path.join(os.path.dirname(__file__), "golden", "ir", "mm_128.txt")).read()
    ir = ir.replace(";128;", ";2048;")
    g = torch.Generator(device=cuda_dev).manual_seed(7)
    n = 2048
    A = torch.randn(n * n, device=cuda_dev, generator=g)
    B = torch.randn(n * n, device=cuda_dev, generator=g)
    C = torch.full((n * n,), float("nan"), device=cuda_dev)
    c = lt.cuda(ir, precision=precision)
    c([A, B, C])
    torch.cuda.synchronize()
    a, b, got = (t.cpu().numpy().reshape(n, n) for t in (A, B, C))
    rng = np.random.default_rng(0)
    rows, cols = rng.integers(0, n, 256), rng.integers(0, n, 256)
    exact = np.einsum("ik,ki->i", a[rows].astype(np.float64), b[:, cols].astype(np.float64))
    err = normwise(got[rows, cols], exact)
    tol = dict(TOL, fp32=1e-6)[precision]
    assert err <= tol, f"{precision}: sampled normwise error {err:.3g}"


# Operand-packing layouts: k-contiguous A with K % 8 == 4 (half-vector tail),
# row-contiguous B with rows % 4 == 0 (float4 transpose path) and % 4 != 0
# (gather path), split-BF16 segments starting at offsets that are not
# multiples of 8 (scalar stores), tiles straddling the 64 x 64 edges.
PACK_SHAPES = [(100, 68, 20), (64, 132, 36), (130, 256, 84), (65, 66, 67), (1, 300, 8),
               (300, 1, 12)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x6", "bf16x3", "bf16"])
@pytest.mark.parametrize("shape", PACK_SHAPES)
def test_pack_layouts(shape, precision, cuda_dev):
    import torch

    import loop_tool_b200 as lt
    from programs import mm

    M, N, K = shape
    T, _ = mm(M, K, N)
    c = lt.cuda(T.ir, precision=precision)
    g = torch.Generator(device=cuda_dev).manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M * K, device=cuda_dev, generator=g)
    B = torch.randn(K * N, device=cuda_dev, generator=g)
    C = torch.full((M * N,), float("nan"), device=cuda_dev)
    for _ in range(2):  # the second run reuses scratch: padding must stay zero
        c([A, B, C])
    torch.cuda.synchronize()
    exact = (A.cpu().numpy().reshape(M, K).astype(np.float64) @
             B.cpu().numpy().reshape(K, N).astype(np.float64))
    got = C.cpu().numpy().reshape(M, N)
    assert np.isfinite(got).all()
    err = normwise(got, exact)
    assert err <= TOL[precision], f"{shape} {precision}: normwise error {err:.3g}"


# Output tiles written by TMA stores: C rows one progression whose pitch
# is a multiple of 4 floats.  Ragged M and N edges (boxes clipped at the
# tensor), a single row, a 4-float pitch, and N % 4 != 0 (per-thread row
# stores); every tile form, so the two-CTA form's row stores and the
# transposed form's staging share the checks.  (M, K, N, TMA-stored)
TMA_STORE = [(300, 64, 200, 1), (1, 64, 36, 1), (70, 32, 4, 1), (130, 96, 66, 0),
             (256, 128, 512, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
@pytest.mark.parametrize("variant", [256, 257, 128, 129, 130, 258])
@pytest.mark.parametrize("shape", TMA_STORE)
def test_tma_store_epilogue(shape, variant, precision, cuda_dev):
    import torch

    import loop_tool_b200 as lt
    from programs import mm

    M, K, N, tma = shape
    T, _ = mm(M, K, N)
    c = lt.cuda(T.ir, precision=precision)
    assert c.int_property("tma_store_output") == tma
    c.set_schedule(0, variant=variant)
    g = torch.Generator(device=cuda_dev).manual_seed(M + 5 * N + 11 * K)
    A = torch.randn(M * K, device=cuda_dev, generator=g)
    B = torch.randn(K * N, device=cuda_dev, generator=g)
    # the output at a 16-byte offset into a larger buffer, guarded on both sides
    buf = torch.full((M * N + 8,), float("nan"), device=cuda_dev)
    C = buf[4:4 + M * N]
    for _ in range(2):
        c([A, B, C])
    torch.cuda.synchronize()
    exact = (A.cpu().numpy().reshape(M, K).astype(np.float64) @
             B.cpu().numpy().reshape(K, N).astype(np.float64))
    got = C.cpu().numpy().reshape(M, N)
    assert np.isfinite(got).all()
    assert np.isnan(buf[:4].cpu().numpy()).all() and np.isnan(buf[4 + M * N:].cpu().numpy()).all()
    err = normwise(got, exact)
    assert err <= TOL[precision], f"{shape} {precision} {variant}: normwise error {err:.3g}"


# 256 x 256 tiles on CTA pairs (variant 258, tcgen05 cta_group::2): each CTA
# of the pair loads half of A's and half of B's rows and receives its 128
# rows of the tile.  A tile whose second CTA has no rows (M <= 128), whose
# second B' half is out of range (N <= 128), a single k block, many
# accumulation chunks, a ragged edge everywhere, and N % 4 != 0 (row stores).
PAIR = [(100, 64, 90), (200, 64, 120), (256, 64, 256), (300, 2048, 520), (513, 200, 259),
        (1000, 96, 1030)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x6", "bf16x3", "bf16"])
@pytest.mark.parametrize("shape", PAIR)
def test_cta_pair_tiles(shape, precision, cuda_dev):
    import torch

    import loop_tool_b200 as lt
    from programs import mm

    M, K, N = shape
    T, _ = mm(M, K, N)
    c = lt.cuda(T.ir, precision=precision)
    c.set_schedule(0, variant=258)
    assert c.schedule(0)[2] == 258
    g = torch.Generator(device=cuda_dev).manual_seed(M * 3 + N + 7 * K)
    A = torch.randn(M * K, device=cuda_dev, generator=g)
    B = torch.randn(K * N, device=cuda_dev, generator=g)
    C = torch.full((M * N,), float("nan"), device=cuda_dev)
    for _ in range(2):
        c([A, B, C])
    torch.cuda.synchronize()
    exact = (A.cpu().numpy().reshape(M, K).astype(np.float64) @
             B.cpu().numpy().reshape(K, N).astype(np.float64))
    got = C.cpu().numpy().reshape(M, N)
    assert np.isfinite(got).all()
    err = normwise(got, exact)
    assert err <= TOL[precision], f"{shape} {precision}: normwise error {err:.3g}"
    # the same contraction on 128 x 256 single-CTA tiles: equal up to the
    # order the tensor core sums each K=16 step in (BF16 products are exact)
    c.set_schedule(0, variant=256)
    C2 = torch.full((M * N,), float("nan"), device=cuda_dev)
    c([A, B, C2])
    torch.cuda.synchronize()
    assert normwise(C2.cpu().numpy().reshape(M, N), got.astype(np.float64)) <= 1e-6


@pytest.mark.gpu
def test_cta_pair_tiles_in_batch(cuda_dev):
    """CTA-pair members beside single-CTA members in one grouped launch."""
    import torch

    import loop_tool_b200 as ltb
    from programs import mm

    g = torch.Generator(device=cuda_dev).manual_seed(23)
    members, shapes = [], [(300, 128, 520, 258), (96, 64, 48, 128), (700, 256, 300, 258),
                           (130, 96, 66, 256)]
    for M, K, N, v in shapes:
        T, _ = mm(M, K, N)
        c = ltb.Compiled(T.ir, precision="bf16x3")
        c.set_schedule(0, variant=v)
        members.append((c, [torch.randn(M * K, device=cuda_dev, generator=g) / K ** 0.5,
                            torch.randn(K * N, device=cuda_dev, generator=g),
                            torch.full((M * N,), float("nan"), device=cuda_dev)]))
    stream = torch.cuda.Stream()
    b = ltb.Batch(members, capture_stream=stream.cuda_stream)
    b.run(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    for (c, (A, B, C)), (M, K, N, v) in zip(members, shapes):
        exact = A.view(M, K).double() @ B.view(K, N).double()
        got = C.view(M, N).double()
        assert torch.isfinite(got).all()
        assert float((got - exact).norm() / exact.norm()) <= TOL["bf16x3"], (M, K, N, v)


# Convolution as implicit GEMM: NCHW inputs with 64-channel blocks and output
# widths that are multiples of 8 are read by the tensor-core kernel straight
# from a padded NHWC image (4-D TMA boxes per output image row); the other
# shapes take the gathered-operand path.  (N, C, H, W, CO, K, pad, implicit)
IMPLICIT = [(2, 64, 8, 8, 16, 3, 1, True), (2, 64, 16, 16, 40, 3, 1, True),
            (1, 128, 10, 10, 24, 3, 0, True), (3, 64, 24, 24, 64, 5, 2, True),
            (1, 64, 56, 56, 128, 3, 1, True), (1, 64, 14, 14, 32, 3, 1, False),
            (2, 32, 16, 16, 16, 3, 1, False)]


def _conv_check(c, N, C, H, W, CO, K, pad, dev, tol, batch=False):
    """Runs c twice (through a one-member Batch with batch=True) and checks
    the output against torch's FP64 convolution, normwise."""
    import torch

    import loop_tool_b200 as lt

    g = torch.Generator(device=dev).manual_seed(N * 1000 + C + H + CO + K)
    x = torch.randn(N * C * H * W, device=dev, generator=g)
    w = torch.randn(CO * C * K * K, device=dev, generator=g) / (C * K * K) ** 0.5
    Ho, Wo = H + 2 * pad - K + 1, W + 2 * pad - K + 1
    y = torch.full((N * Ho * Wo * CO,), float("nan"), device=dev)
    b = lt.Batch([(c, [x, w, y])]) if batch else None
    for _ in range(2):  # scratch reused: the padded image must be rewritten whole
        if b is not None:
            b.run()
        else:
            c([x, w, y])
    torch.cuda.synchronize()
    ref = torch.nn.functional.conv2d(x.view(N, C, H, W).double(),
                                     w.view(CO, C, K, K).double(), padding=pad)
    got = y.view(N, Ho, Wo, CO).permute(0, 3, 1, 2).double()
    assert torch.isfinite(got).all()
    err = float((got - ref).norm() / ref.norm())
    assert err <= tol, f"normwise error {err:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x6", "bf16x3", "bf16"])
@pytest.mark.parametrize("shape", IMPLICIT)
def test_conv_implicit_gemm(shape, precision, cuda_dev):
    import loop_tool_b200 as lt
    from programs import conv

    N, C, H, W, CO, K, pad, implicit = shape
    T, _ = conv(N, C, H, W, CO, K, pad, 1)
    c = lt.cuda(T.ir, precision=precision)
    assert c.int_property("implicit_conv") == (1 if implicit else 0)
    _conv_check(c, N, C, H, W, CO, K, pad, cuda_dev, TOL[precision])


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [128, 129, 130])
def test_conv_implicit_every_variant(variant, cuda_dev):
    """Every tile form of the implicit-GEMM convolution (row stores, shared
    memory transposed epilogue, two CTAs per SM) agrees with FP64."""
    import loop_tool_b200 as lt
    from programs import conv

    T, _ = conv(2, 64, 16, 16, 40, 3, 1, 1)
    c = lt.cuda(T.ir, precision="bf16x3")
    c.set_schedule(0, variant=variant)
    assert c.schedule(0)[2] == variant and c.int_property("implicit_conv") == 1
    _conv_check(c, 2, 64, 16, 16, 40, 3, 1, cuda_dev, TOL["bf16x3"])


# Halo image tiles (variant 131, BF16; 133 on CTA pairs): one TMA box per
# kernel row covers the tile's padded image rows; the kw shifts are read in
# place at row offsets inside the 128-byte swizzle atoms; the weights stay in
# shared memory (half of them in each CTA of a pair).
# Shapes: partial last row group, several images, a 2 x 2 kernel, two
# channel blocks, and the 56 x 56 image with 128 output channels.
# (N, C, H, W, CO, K, pad)
HALO = [(2, 64, 8, 8, 16, 3, 1), (2, 64, 16, 16, 40, 3, 1), (2, 64, 17, 17, 24, 2, 0),
        (2, 128, 15, 15, 32, 2, 1), (4, 64, 32, 32, 128, 3, 1), (1, 64, 56, 56, 128, 3, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", HALO)
def test_conv_halo_tiles(shape, cuda_dev):
    import loop_tool_b200 as lt
    from programs import conv

    N, C, H, W, CO, K, pad = shape
    T, _ = conv(N, C, H, W, CO, K, pad, 1)
    c = lt.cuda(T.ir, precision="bf16")
    c.set_schedule(0, variant=131)
    assert c.schedule(0)[2] == 131
    _conv_check(c, N, C, H, W, CO, K, pad, cuda_dev, TOL["bf16"])
    # the same tiles two to a CTA pair (M = 256, half the weights per CTA)
    c.set_schedule(0, variant=133)
    assert c.schedule(0)[2] == 133
    _conv_check(c, N, C, H, W, CO, K, pad, cuda_dev, TOL["bf16"])
    # a batch runs a halo-form member as per-row image tiles of its width
    _conv_check(c, N, C, H, W, CO, K, pad, cuda_dev, TOL["bf16"], batch=True)
    # and back to the per-row image tiles on the same compiled object
    c.set_schedule(0, variant=128)
    assert c.schedule(0)[2] == 128
    _conv_check(c, N, C, H, W, CO, K, pad, cuda_dev, TOL["bf16"])


@pytest.mark.gpu
def test_conv_halo_not_applicable(cuda_dev):
    """Weights too large for shared memory (C x KH x KW = 1152) or a split
    precision: variant 131 falls back to the per-row image tiles."""
    import loop_tool_b200 as lt
    from programs import conv

    T, _ = conv(1, 128, 10, 10, 24, 3, 0, 1)
    c = lt.cuda(T.ir, precision="bf16")
    c.set_schedule(0, variant=131)
    assert c.schedule(0)[2] == 128
    _conv_check(c, 1, 128, 10, 10, 24, 3, 0, cuda_dev, TOL["bf16"])
    c.set_schedule(0, variant=133)  # the CTA-pair form likewise
    assert c.schedule(0)[2] == 128
    T, _ = conv(2, 64, 16, 16, 40, 3, 1, 1)
    c = lt.cuda(T.ir, precision="bf16x3")
    c.set_schedule(0, variant=131)
    assert c.schedule(0)[2] == 128
    _conv_check(c, 2, 64, 16, 16, 40, 3, 1, cuda_dev, TOL["bf16x3"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x6", "bf16x3", "bf16"])
def test_conv_implicit_in_batch(precision, cuda_dev):
    """An implicit-GEMM convolution and plain matmuls in one grouped launch."""
    import torch

    import loop_tool_b200 as ltb
    from programs import conv, mm

    T, _ = conv(2, 64, 16, 16, 40, 3, 1, 1)
    cc = ltb.Compiled(T.ir, precision=precision)
    assert cc.int_property("implicit_conv") == 1
    g = torch.Generator(device=cuda_dev).manual_seed(17)
    x = torch.randn(2 * 64 * 16 * 16, device=cuda_dev, generator=g)
    w = torch.randn(40 * 64 * 9, device=cuda_dev, generator=g) / 24.0
    y = torch.full((2 * 16 * 16 * 40,), float("nan"), device=cuda_dev)
    members = [(cc, [x, w, y])]
    mms = []
    for M, K, N in ((96, 64, 48), (300, 128, 200)):
        Tm, _ = mm(M, K, N)
        cm = ltb.Compiled(Tm.ir, precision=precision)
        bufs = [torch.randn(M * K, device=cuda_dev, generator=g) / K ** 0.5,
                torch.randn(K * N, device=cuda_dev, generator=g),
                torch.full((M * N,), float("nan"), device=cuda_dev)]
        members.append((cm, bufs))
        mms.append((M, K, N, bufs))
    stream = torch.cuda.Stream()
    b = ltb.Batch(members, capture_stream=stream.cuda_stream)
    b.run(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ref = torch.nn.functional.conv2d(x.view(2, 64, 16, 16).double(),
                                     w.view(40, 64, 3, 3).double(), padding=1)
    got = y.view(2, 16, 16, 40).permute(0, 3, 1, 2).double()
    assert float((got - ref).norm() / ref.norm()) <= TOL[precision]
    for M, K, N, (A, B, C) in mms:
        exact = A.view(M, K).double() @ B.view(K, N).double()
        assert float((C.view(M, N).double() - exact).norm() / exact.norm()) <= TOL[precision]
