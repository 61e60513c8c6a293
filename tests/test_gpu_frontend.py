"""Programs written with this package's lazy frontend run on the B200 backend
(Tensor.numpy(): compile through the IR-text cache, numpy-bound inputs and
output staged through HBM) and reproduce the reference's outputs."""
import pytest

from golden_util import EXACT_PROGRAMS, assert_accuracy, assert_parity, fp64_oracle, load, manifest
from programs import BUILDERS, build

CASES = [m["name"] for m in manifest() if m["program"] in BUILDERS]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_frontend_on_b200(name, cuda_dev):
    case = load(name)
    T, _ = build(case)
    got = T.numpy().ravel()
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)


@pytest.mark.gpu
def test_kernel_cache_reuse(cuda_dev):
    import numpy as np

    import loop_tool_b200.lazy as lt
    from programs import mm

    lt.clear_cache()
    for _ in range(3):
        T, (A, B) = mm(64, 32, 48)
        A.set(np.ones((64, 32), np.float32))
        B.set(np.ones((32, 48), np.float32))
        assert (T.numpy() == 32).all()
    assert lt.cache_info()["entries"] == 1
