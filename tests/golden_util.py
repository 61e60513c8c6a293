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
# contractions, exp): within 1e-5 relative, entry by entry.
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
    if case["program"] == "abs":
        # The reference's two CPU backends disagree on abs: the C path emits
        # C's integer abs() on a float (cpp.cpp:223-224 prints "abs", so
        # 0.4 -> 0), the interpreter uses std::abs(float) (compile.cpp:1066).
        # The B200 backend and the oracle follow the float definition.
        case["expected_c_path"] = case["expected"]
        case["expected"] = np.abs(case["inputs"][0])
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


def fp64_oracle(case):
    """The FP64 evaluation of the case's loop tree (oracle/np_oracle.py)."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "oracle"))
    import np_oracle

    return np_oracle.evaluate(case["ir"], [a.astype(np.float64) for a in case["inputs"]],
                              dtype=np.float64)[0]


def accuracy_report(got, ref32, exact64):
    """Elementwise error of `got` and of the reference's own FP32 result
    `ref32` against the FP64 oracle `exact64` (finite entries only)."""
    got = np.asarray(got, np.float64).ravel()
    ref32 = np.asarray(ref32, np.float64).ravel()
    exact64 = np.asarray(exact64, np.float64).ravel()
    fin = np.isfinite(exact64) & np.isfinite(ref32)
    e = exact64[fin]
    err = np.abs(got[fin] - e)
    ref_err = np.abs(ref32[fin] - e)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(e != 0, err / np.abs(e), np.where(err == 0, 0.0, np.inf))
    tol = np.maximum(RTOL * np.abs(e), ref_err * (1 + 1e-6))
    return {
        "entries": int(e.size),
        "bit_exact_with_reference": bool(bits_equal(got.astype(np.float32), ref32.astype(np.float32))),
        "max_elementwise_rel_err_vs_fp64": float(rel.max()) if rel.size else 0.0,
        "normwise_rel_err_vs_fp64": float(np.linalg.norm(got[fin] - e) / max(np.linalg.norm(e), 1e-300)),
        "entries_over_tolerance": int((err > tol).sum()),
    }


def assert_accuracy(got, ref32, exact64, rtol=RTOL, what=""):
    """Order-dependent FP32 results (sums, contractions, exp), elementwise:
    each entry's error against the FP64 oracle is within rtol of that
    entry (|got - e| <= rtol * |e|) or no larger than the reference's own
    FP32 error on that entry.  A result that is bit-exact with the
    reference passes by construction; the second clause is what lets an
    entry whose exact value cancels to near zero through."""
    got = np.asarray(got, np.float64).ravel()
    ref32 = np.asarray(ref32, np.float64).ravel()
    exact64 = np.asarray(exact64, np.float64).ravel()
    assert got.shape == exact64.shape, f"{what}: shape {got.shape} vs {exact64.shape}"
    assert np.array_equal(np.isnan(got), np.isnan(ref32)), f"{what}: NaN pattern differs"
    fin = np.isfinite(exact64) & np.isfinite(ref32)
    assert np.array_equal(got[~fin & ~np.isnan(got)], ref32[~fin & ~np.isnan(ref32)]), \
        f"{what}: non-finite entries differ"
    e = exact64[fin]
    err = np.abs(got[fin] - e)
    ref_err = np.abs(ref32[fin] - e)
    tol = np.maximum(rtol * np.abs(e), ref_err * (1 + 1e-6))
    if not (err <= tol).all():
        bad = int((err > tol).sum())
        i = int(np.argmax(err - tol))
        raise AssertionError(f"{what}: {bad} of {e.size} entries over tolerance; worst "
                             f"|err vs fp64| {err[i]:.3g} > tol {tol[i]:.3g} at {i} "
                             f"(got {got[fin][i]!r}, fp64 {e[i]!r}, reference {ref32[fin][i]!r})")
    scale = float(np.sqrt(np.mean(e ** 2))) if e.size else 1.0
    return float(err.max() / max(scale, 1e-30)) if err.size else 0.0


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
    raise AssertionError(f"{what}: order-dependent results are checked with assert_accuracy "
                         "against the FP64 oracle")
