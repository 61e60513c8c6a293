"""The CPU oracle (oracle/np_oracle.py) is pinned against the reference:
it must reproduce the reference lazy frontend's output for every golden
fixture (bit-exact where the reference's arithmetic is exact, else within
1e-5 relative), and the reference's own known-answer assertions."""
import os
import sys

import numpy as np
import pytest

from golden_util import EXACT_PROGRAMS, assert_parity, load, manifest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import np_oracle  # noqa: E402

# the oracle evaluates exp/log/sqrt in double like the generated C, so it is
# bit-exact even where the B200 path is within tolerance
ORACLE_EXACT = EXACT_PROGRAMS | {"exp", "log", "softmax", "rowsum", "colsum", "mm", "bmm",
                                 "conv", "padconv1d", "mean_rows", "layernorm", "fullsum"}


@pytest.mark.parametrize("name", [m["name"] for m in manifest()])
def test_oracle_matches_reference(name):
    case = load(name)
    got = np_oracle.evaluate(case["ir"], case["inputs"])[0]
    assert_parity(got, case["expected"], case["program"] in ORACLE_EXACT, what=name)


def test_reference_kats():
    """Known-answer assertions of the reference's own tests."""
    g = lambda n: load(n)["expected"]
    assert g("concat1d_kat")[10] == 2  # test_lazy.cpp:384
    assert g("concat2d_kat")[6] == 7 and g("concat2d_kat")[8] == 11  # :412-413
    assert g("pad1d_kat")[2] == 1 and g("pad1d_kat")[6] == 0  # :432-433
    assert (g("transpose_flatten_kat") == np.arange(64)).all()  # :279-281
    assert (g("flatten_kat") == np.arange(64)).all()  # :297-299
    assert g("conv1d_kat")[3] == 3  # :329
    assert g("scale_kat")[7] == 14  # :240


def test_oracle_against_numpy_semantics():
    """Independent cross-checks of the restated semantics."""
    c = load("conv_2x4x8x8_pad1")
    x = c["inputs"][0].reshape(2, 4, 8, 8).astype(np.float64)
    w = c["inputs"][1].reshape(8, 4, 3, 3).astype(np.float64)
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    y = np.zeros((2, 8, 8, 8))  # [n, ho, wo, co]
    for kh in range(3):
        for kw in range(3):
            y += np.einsum("nchw,oc->nhwo", xp[:, :, kh:kh + 8, kw:kw + 8], w[:, :, kh, kw])
    got = np_oracle.evaluate(c["ir"], c["inputs"])[0].reshape(2, 8, 8, 8)
    assert np.abs(got - y).max() < 1e-4
    s = load("softmax_16x32")
    x = s["inputs"][0].reshape(16, 32).astype(np.float64)
    e = np.exp(x - x.max(1, keepdims=True))
    ref = e / e.sum(1, keepdims=True)
    assert np.abs(np_oracle.evaluate(s["ir"], s["inputs"])[0].reshape(16, 32) - ref).max() < 1e-6


@pytest.mark.parametrize("name", ["fullsum_2x40000", "softmax_16x4096", "mm_128",
                                  "conv_2x4x8x8_pad1", "layernorm_8x256"])
def test_reference_fp32_error_vs_fp64(name):
    """The FP64 oracle agrees with the reference's FP32 result to the FP32
    rounding error of the reference's sequential order."""
    from golden_util import assert_accuracy, fp64_oracle

    case = load(name)
    assert_accuracy(case["expected"], case["expected"], fp64_oracle(case), rtol=1e-3, what=name)
