"""The serving loop: continuous batching over CUDA streams with admission by
an HBM byte budget.  Each request's result in the concurrent mix equals the
same request run alone (bit for bit: the kernels are deterministic and no
state is shared between concurrent runs)."""
import numpy as np
import pytest


def small_trace(n, seed):
    from loop_tool_b200.serve import make_trace

    return make_trace(n, rate=1e6, seed=seed, mm_range=(16, 512), conv_batch=(1, 3),
                      softmax_rows=(1, 300))


def same(a, b):
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and \
        np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_mix_equals_alone(precision, cuda_dev):
    from loop_tool_b200.serve import Server, run_alone

    trace = small_trace(30, seed=11)
    srv = Server(slots=6, precision=precision, keep_outputs=True)
    stats, done = srv.serve(trace)
    assert stats["requests"] == len(trace)
    assert stats["peak_inflight"] > 1, "requests never overlapped"
    assert {r.kind for r in done} == {"matmul", "conv", "softmax"}
    for r in done:
        alone = run_alone(r, precision=precision)
        assert same(r.out, alone), f"request {r.rid} ({r.kind} {r.params}) differs alone vs mix"


@pytest.mark.gpu
def test_admission_respects_hbm_budget(cuda_dev):
    from loop_tool_b200.serve import Server

    trace = small_trace(20, seed=12)
    probe = Server(slots=8)
    need = max(probe.bytes_of(r) for r in trace)
    srv = Server(slots=8, hbm_budget=int(need * 1.5))
    stats, done = srv.serve(trace)
    assert stats["requests"] == len(trace)
    assert srv.peak_used <= int(need * 1.5)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0


@pytest.mark.gpu
def test_reserved_workspaces_serve_without_growth(cuda_dev):
    """Workspaces sized up front: serving allocates nothing more, and every
    result matches the unreserved server's."""
    from loop_tool_b200.serve import Server

    trace = small_trace(24, seed=13)
    ref = Server(slots=4, keep_outputs=True)
    _, base = ref.serve(small_trace(24, seed=13))
    srv = Server(slots=4, keep_outputs=True)
    reserved = srv.reserve(trace)
    sizes = [w.numel() for w in srv.ws]
    assert reserved == 4 * sum(sizes) and min(sizes) > 0
    _, done = srv.serve(trace)
    assert [w.numel() for w in srv.ws] == sizes, "a workspace grew while serving"
    by_id = {r.rid: r.out for r in base}
    for r in done:
        assert same(r.out, by_id[r.rid]), f"request {r.rid} differs"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_bucketed_server(precision, cuda_dev):
    """Shape-bucketed keys: fewer compiled programs than distinct shapes;
    each result equals the same request alone in the same bucket (bit for
    bit) and the exact-size server's result (bit for bit in FP32, whose sums
    only gain trailing zero terms; within the split-BF16 tolerance, whose
    K segments shift with the padded K)."""
    from loop_tool_b200.serve import Server, bucket_params, run_alone

    trace = small_trace(30, seed=14)
    exact = Server(slots=4, precision=precision, keep_outputs=True)
    _, base = exact.serve(small_trace(30, seed=14))
    srv = Server(slots=6, precision=precision, keep_outputs=True, buckets=True)
    stats, done = srv.serve(trace)
    assert stats["requests"] == len(trace)
    assert srv.compiles == len({(r.kind, bucket_params(r.kind, r.params)) for r in trace})
    assert srv.compiles < exact.compiles
    by_id = {r.rid: r.out for r in base}
    for r in done:
        alone = run_alone(r, precision=precision, buckets=True)
        assert same(r.out, alone), f"request {r.rid} differs alone vs mix"
        ref = by_id[r.rid]
        if precision == "fp32":
            assert np.array_equal(r.out, ref), f"request {r.rid} ({r.kind} {r.params})"
        else:
            d = np.linalg.norm(r.out.astype(np.float64) - ref) / np.linalg.norm(ref)
            assert d <= 2e-5, f"request {r.rid} ({r.kind} {r.params}): {d:.3g}"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_native_server_mix_equals_alone(precision, cuda_dev):
    """The C++ request loop (ltb_server_*): every result in the concurrent
    mix equals the same request served alone, bit for bit; requests
    overlapped; softmax rows sum to one."""
    from loop_tool_b200.serve import NativeServer

    trace = small_trace(30, seed=21)
    srv = NativeServer(slots=6, precision=precision)
    srv.prepare(trace)
    stats, outs = srv.serve(trace, keep_outputs=True)
    assert stats["requests"] == len(trace) and stats["peak_inflight"] > 1
    alone = NativeServer(slots=1, precision=precision)
    for r, o in zip(trace, outs):
        _, (a,) = alone.serve([r], keep_outputs=True)
        assert same(o, a), f"request {r.rid} ({r.kind} {r.params}) differs alone vs mix"
        assert np.isfinite(o).all()
        if r.kind == "softmax":
            assert np.abs(o.reshape(-1, 4096).astype(np.float64).sum(1) - 1).max() < 1e-5


@pytest.mark.gpu
def test_native_server_budget_and_buckets(cuda_dev):
    """Admission keeps the bytes in flight within the budget; a bucketed
    native server compiles fewer programs and, in FP32, gives the exact-key
    server's results bit for bit (inputs are seeded per element of the true
    block, so padding does not change them)."""
    from loop_tool_b200.serve import NativeServer, bucket_params

    trace = small_trace(24, seed=22)
    exact = NativeServer(slots=4, precision="fp32")
    _, base = exact.serve(trace, keep_outputs=True)
    need = max(4 * sum(r.params[0] * 4096 for r in trace if r.kind == "softmax"), 1)
    srv = NativeServer(slots=8, hbm_budget=64 << 20, precision="fp32", buckets=True)
    stats, outs = srv.serve(trace, keep_outputs=True)
    assert stats["peak_bytes"] <= 64 << 20 and need > 0
    assert stats["compiles"] == len({(r.kind, bucket_params(r.kind, r.params)) for r in trace})
    for r, o, b in zip(trace, outs, base):
        assert np.array_equal(o, b), f"request {r.rid} ({r.kind} {r.params})"
