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
TOL = {"bf16x4": 1e-5, "bf16x3": 1.5e-5, "bf16": 1.5e-2}


def normwise(got, exact):
    return float(np.linalg.norm(got.astype(np.float64) - exact) / np.linalg.norm(exact))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x4", "bf16x3", "bf16"])
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
@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
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
