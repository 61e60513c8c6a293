"""Loading of the reference golden fixtures and the parity comparison."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Programs whose values the reference computes with copies, comparisons and
# single correctly rounded operations only: the B200 path must be bit-exact.
EXACT_PROGRAMS = {
    "add", "sub", "mul", "div", "min", "max", "sqrt", "neg", "recip", "abs",
    "chain", "scale", "bcast_add", "pad1d", "pad2d", "concat1d", "concat2d",
    "transpose_flatten", "flatten", "transpose", "rowmax", "rowmin", "colmax",
    "maxpool", "conv1d",
}
# FP32 arithmetic whose rounding depends on evaluation order (sums,
# contractions, exp): within 1e-5 relative.
RTOL = 1e-5


def manifest():
    return json.load(open(os.path.join(GOLDEN, "manifest.json")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = {k: z[k] for k in z.files}
    case["ir"] = str(case["ir"])
    case["program"] = str(case["program"])
    case["inputs"] = [case[f"in{i}"] for i in range(sum(1 for k in z.files if k.startswith("in") and k[2:].isdigit()))]
    case["expected"] = case["out0_lazy"]
    return case


def bits_equal(a, b):
    """Bitwise equality, with every NaN equal to every NaN."""
    a = np.asarray(a, np.float32).ravel()
    b = np.asarray(b, np.float32).ravel()
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


def assert_parity(got, expected, exact, rtol=RTOL, what=""):
    got = np.asarray(got, np.float32).ravel()
    expected = np.asarray(expected, np.float32).ravel()
    assert got.shape == expected.shape, f"{what}: shape {got.shape} vs {expected.shape}"
    if exact:
        if not bits_equal(got, expected):
            bad = np.nonzero(~((got == expected) | (np.isnan(got) & np.isnan(expected))) |
                             (np.signbit(got) != np.signbit(expected)))[0]
            i = bad[0] if len(bad) else 0
            raise AssertionError(f"{what}: not bit-exact at {len(bad)} positions, first {i}: "
                                 f"got {got[i]!r} expected {expected[i]!r}")
        return
    fin = np.isfinite(expected)
    assert np.array_equal(np.isnan(got), np.isnan(expected)), f"{what}: NaN pattern differs"
    scale = float(np.sqrt(np.mean(expected[fin].astype(np.float64) ** 2))) if fin.any() else 1.0
    err = np.abs(got[fin].astype(np.float64) - expected[fin])
    tol = rtol * np.abs(expected[fin]).astype(np.float64) + rtol * scale
    if not (err <= tol).all():
        i = int(np.argmax(err - tol))
        raise AssertionError(f"{what}: |err| {err[i]:.3g} > tol {tol[i]:.3g} at {i} "
                             f"(got {got[fin][i]!r}, expected {expected[fin][i]!r})")
