"""This package's lazy frontend (loop_tool_b200.lazy) builds the same
programs as the reference's lazy frontend: its IR, evaluated by the pinned
CPU oracle on the golden inputs, reproduces the reference's outputs."""
import os
import sys

import pytest

from golden_util import EXACT_PROGRAMS, assert_accuracy, assert_parity, fp64_oracle, load, manifest
from programs import BUILDERS, build

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import np_oracle  # noqa: E402

CASES = [m["name"] for m in manifest() if m["program"] in BUILDERS]


@pytest.mark.parametrize("name", CASES)
def test_frontend_ir_matches_reference(name):
    case = load(name)
    T, leaves = build(case)
    text = T.ir
    assert len(leaves) == len(case["inputs"])
    got = np_oracle.evaluate(text, case["inputs"])[0]
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)


def test_frontend_cache_key_is_structural():
    """Identical programs built twice lower to identical IR text (one cache
    entry), different sizes to different text."""
    from programs import mm

    a, _ = mm(16, 8, 4)
    b, _ = mm(16, 8, 4)
    c, _ = mm(16, 8, 5)
    assert a.ir == b.ir and a.ir != c.ir


def test_frontend_size_inference():
    """test_lazy.py:58-70: Y = conv(X, W0) with |W0| = 3, Z = (Y * W1).sum,
    |W1| = 8 -> |X| = 10."""
    import loop_tool_b200.lazy as lt

    N, K = lt.Symbol("N"), lt.Symbol("K")
    X, W0, W1 = lt.Tensor(N), lt.Tensor(3), lt.Tensor(8)
    No, Kw = lt.Symbol("No"), lt.Symbol("Kw")
    Y = (X[lt.Expr(No) + Kw] * W0.to(Kw)).sum(Kw)
    Z = (Y.to(K) * W1.to(K)).sum(K)
    sizes = Z._unify()[4]
    assert sizes[N] == 10
