"""The configurations at their full sizes.  The loop trees are the ones the
reference's own lazy frontend emitted for them (tests/golden/ir/, the text
the drop-in backend receives), run with autotuned schedules.  Elementwise
add and max-pool are exact operations, so the B200 result must equal the
same operation done by torch bit for bit; the FP32 convolution and a 1024^3
matmul must equal the reference CPU backend's own output on the same tree
bit for bit; softmax is checked elementwise and the tensor-core modes
against FP64 (normwise and elementwise on sampled outputs)."""
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest

from bench import reference_ir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")


def reference_cpp(ir, inputs):
    """The reference "cpp" backend's output on the IR (oracle harness)."""
    with tempfile.TemporaryDirectory() as td:
        irf = os.path.join(td, "ir.txt")
        open(irf, "w").write(ir)
        for i, a in enumerate(inputs):
            np.asarray(a, np.float32).tofile(os.path.join(td, f"in{i}.f32"))
        r = subprocess.run([HARNESS, "run", irf, "cpp", td, td], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        return np.fromfile(os.path.join(td, "out0.f32"), np.float32)


def reference_lazy(program, params, inputs):
    """The reference's output for a program run through its own lazy
    frontend (oracle harness `lazyrun`: the in-memory loop tree, as the
    golden fixtures are made -- a serialize/deserialize round trip gives
    every node fresh symbols, and the reference's Compiler then misreads
    the padded convolution's view)."""
    with tempfile.TemporaryDirectory() as td:
        for i, a in enumerate(inputs):
            np.asarray(a, np.float32).tofile(os.path.join(td, f"in{i}.f32"))
        r = subprocess.run([HARNESS, "lazyrun", td, td, program, *map(str, params)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        return np.fromfile(os.path.join(td, "out0.f32"), np.float32)


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

    n = 1 << 28
    g = torch.Generator(device=cuda_dev).manual_seed(201)
    a = torch.randn(n, device=cuda_dev, generator=g)
    b = torch.randn(n, device=cuda_dev, generator=g)
    c = torch.empty(n, device=cuda_dev)
    _run(reference_ir("add_2p28"), [a, b, c])
    assert torch.equal(c, a + b)


@pytest.mark.gpu
def test_maxpool_64x128x112x112_bit_exact(cuda_dev):
    import torch

    ir = reference_ir("maxpool_64x128x112x112")
    g = torch.Generator(device=cuda_dev).manual_seed(221)
    x = torch.randn(64 * 128 * 112 * 112, device=cuda_dev, generator=g)
    y = torch.empty(64 * 128 * 56 * 56, device=cuda_dev)
    _run(ir, [x, y])
    ref = torch.nn.functional.max_pool2d(x.view(64, 128, 112, 112), 2, 2)
    assert torch.equal(y.view(64, 128, 56, 56), ref)


@pytest.mark.gpu
def test_softmax_8192x4096_vs_fp64(cuda_dev):
    import torch

    g = torch.Generator(device=cuda_dev).manual_seed(211)
    xs = 4 * torch.randn(8192 * 4096, device=cuda_dev, generator=g)
    y = torch.empty_like(xs)
    _run(reference_ir("softmax_8192x4096"), [xs, y])
    ref = torch.softmax(xs.view(8192, 4096).double(), dim=1)
    err = (y.view(8192, 4096).double() - ref).abs()
    # every element within FP32 rounding of its FP64 value (relative)
    assert float((err / ref.clamp_min(1e-30)).max()) < 1e-5
    assert float(y.view(8192, 4096).double().sum(1).sub(1).abs().max()) < 1e-5


@pytest.mark.gpu
def test_conv_32x64x56x56_fp32_bit_exact_with_reference(cuda_dev):
    """The plain FP32 convolution reproduces the reference C path's output
    on the same tree bit for bit (same fold order over c, kh, kw, each
    multiply and add rounded on its own)."""
    import torch

    if not os.path.exists(HARNESS):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    ir = reference_ir("conv_32x64x56x56_co128")
    rng = np.random.default_rng(301)
    x = rng.standard_normal(32 * 64 * 56 * 56).astype(np.float32)
    bound = math.sqrt(6.0 / 576)
    w = np.random.default_rng(302).uniform(-bound, bound, 128 * 64 * 9).astype(np.float32)
    y = torch.empty(32 * 56 * 56 * 128, device=cuda_dev)
    _run(ir, [torch.from_numpy(x).to(cuda_dev), torch.from_numpy(w).to(cuda_dev), y])
    ref = reference_lazy("conv", [32, 64, 56, 56, 128, 3, 1, 1], [x, w])
    got = y.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), \
        f"{int((got != ref).sum())} of {got.size} entries differ"


@pytest.mark.gpu
def test_mm_1024_fp32_bit_exact_with_reference(cuda_dev):
    import torch

    if not os.path.exists(HARNESS):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    n = 1024
    ir = reference_ir("mm_128", {0: n, 1: n, 2: n})
    rng = np.random.default_rng(7)
    a, b = (rng.standard_normal(n * n).astype(np.float32) for _ in range(2))
    c = torch.empty(n * n, device=cuda_dev)
    _run(ir, [torch.from_numpy(a).to(cuda_dev), torch.from_numpy(b).to(cuda_dev), c])
    ref = reference_cpp(ir, [a, b])
    assert np.array_equal(c.cpu().numpy().view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("bf16x6", 1e-6), ("bf16x3", 1e-5), ("bf16", 1.5e-2)])
def test_conv_32x64x56x56_vs_fp64(precision, tol, cuda_dev):
    import torch

    ir = reference_ir("conv_32x64x56x56_co128")
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
@pytest.mark.parametrize("precision,tol", [("bf16x6", 1e-6), ("bf16x3", 1e-5), ("bf16", 1.5e-2)])
def test_mm_8192_sampled_vs_fp64(precision, tol, cuda_dev):
    import torch

    n = 8192
    ir = reference_ir("mm_8192")
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

    n = (1 << 25) + 12344  # four full 2^23-element chunks and a ragged fifth
    A, B = lt.Tensor(n), lt.Tensor(n)
    N = lt.Symbol("N")
    T = A.to(N) + B.to(N) if op == "add" else A.to(N).exp()
    c = ltb.Compiled(reference_ir("add_2p28", {0: n}) if op == "add" else T.ir)
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
