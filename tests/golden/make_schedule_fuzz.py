"""Generates tests/golden/schedule_fuzz.npz: randomly scheduled loop trees of
the reference's own programs, with the reference's outputs on them.

The reference's randomized test (test/test.py:56-96 rand_split /
rand_sched, run over sizes 2^i, 2^i + 1 and primes at :289-313) splits
every loop var of every node into up to three loops with random factors
and tails and checks its backends against each other.  Here the same
schedules are drawn by the oracle harness (oracle/ref_harness.cpp `fuzz`:
the program is built by the reference's lazy frontend, every non-view node
gets a rand_sched-style order, half of the trees also have their var
groups shuffled), serialized, and run by both reference CPU backends on
the in-memory loop tree: "cpp" (generated C) and "cpu_interpreted".

Each case stores the serialized scheduled IR, the seeded inputs and both
outputs.  The two backends disagree on some trees (the generated C of
some split-with-tail schedules is wrong; the interpreter matches the FP64
value); the case records which.

Needs the reference built by oracle/Makefile (oracle/_ref/lt_ref_harness).

    python tests/golden/make_schedule_fuzz.py
"""
import os
import json
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import np_oracle  # noqa: E402
OUT = os.path.join(HERE, "schedule_fuzz.npz")

# test/test.py:290-295: powers of two, 2^i + 1, primes
SIZES = [2 ** i for i in range(1, 8)] + [2 ** i + 1 for i in range(1, 7)] + \
        [x for x in range(8, 30) if all(x % y for y in range(2, x))]


def programs(rng):
    """(program, params) pairs: pointwise, reductions, contractions, views."""
    out = []
    for s in SIZES:
        out += [("add", [s]), ("chain", [s]), ("exp", [s])]
        s2 = int(rng.choice(SIZES))
        out += [("rowsum", [s, s2]), ("rowmax", [s2, s]), ("colsum", [s, s2]),
                ("softmax", [s2, s]), ("fullsum", [s, s2])]
    for m in range(1, 17, 3):  # test/test.py:305-311 test_rand_mm
        for n in range(5, 7):
            for k in range(8, 11):
                out.append(("mm", [m, k, n]))
    for s in (3, 8, 17, 32):
        out += [("pad1d", [s, 2, 3]), ("pad2d", [s, 5, 2]), ("concat1d", [s, 7]),
                ("concat2d", [4, s, 5]), ("transpose", [s, 7]), ("bcast_add", [s, 9]),
                ("bmm", [2, s, 5, 3]), ("padconv1d", [s + 4, 3, 1]), ("conv1d", [s + 4, 3]),
                ("layernorm", [3, s]), ("mean_rows", [s, 6]),
                ("transpose_flatten", [s, 5]), ("flatten", [5, s])]
    out += [("maxpool", [2, 3, 8, 8, 2, 2]), ("maxpool", [1, 2, 9, 9, 3, 2]),
            ("conv", [2, 3, 8, 8, 4, 3, 1, 1]), ("conv", [1, 2, 7, 9, 3, 3, 0, 1]),
            ("conv", [2, 3, 9, 9, 4, 3, 0, 2]), ("conv", [1, 4, 6, 6, 2, 3, 1, 1])]
    return out


def harness(*args):
    r = subprocess.run([HARNESS, *map(str, args)], capture_output=True, text=True)
    return r.returncode, r.stdout, r.stderr


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build the oracle first: make -C oracle REF=<reference checkout>")
    rng = np.random.default_rng(1337)
    arrays = {}
    meta = []
    skipped = []
    with tempfile.TemporaryDirectory() as tmp:
        for idx, (prog, params) in enumerate(programs(rng) * 2):
            ind, outd = os.path.join(tmp, f"i{idx}"), os.path.join(tmp, f"o{idx}")
            os.makedirs(ind)
            os.makedirs(outd)
            rc, ir, err = harness("ir", prog, *params)
            assert rc == 0, err
            ir_path = os.path.join(ind, "default.txt")
            open(ir_path, "w").write(ir)
            rc, sizes, err = harness("sizes", ir_path)
            assert rc == 0, err
            ins = []
            for i, n in enumerate(json.loads(sizes)["inputs"]):
                a = rng.standard_normal(n).astype(np.float32)
                if prog in ("layernorm",) and i == 1:
                    a = np.full(n, float(params[1]), np.float32)  # element count
                if prog in ("layernorm",) and i == 2:
                    a = np.full(n, 1e-5, np.float32)  # eps
                if prog == "mean_rows" and i == 1:
                    a = np.ones(n, np.float32)
                a.tofile(os.path.join(ind, f"in{i}.f32"))
                ins.append(a)
            seed = int(rng.integers(1 << 31))
            permute = idx % 2
            rc, _, err = harness("fuzz", outd, ind, seed, permute, "none", prog, *params)
            if rc != 0:
                skipped.append((prog, params, "schedule: " + " ".join(err.split()[-8:])))
                continue
            ir_text = open(os.path.join(outd, "ir.txt")).read()
            got = {}
            for be in ("cpu_interpreted", "cpp"):  # one process each
                rc, _, err = harness("fuzz", outd, ind, seed, permute, be, prog, *params)
                path = os.path.join(outd, be + "0.f32")
                got[be] = np.fromfile(path, np.float32) if rc == 0 and os.path.exists(path) else None
            interp = got["cpu_interpreted"]
            if interp is None:
                skipped.append((prog, params, "cpu_interpreted failed"))
                continue
            # the dataflow value in FP64 (oracle/np_oracle.py): a tree whose
            # interpreter output is far from it is a reference defect, kept
            # out of the parity set and counted
            exact = np_oracle.evaluate(ir_text, [a.astype(np.float64) for a in ins],
                                       dtype=np.float64)[0].ravel()
            fin = np.isfinite(exact)
            scale = float(np.abs(exact[fin]).mean()) if fin.any() else 1.0
            dev = float(np.abs(interp.astype(np.float64)[fin] - exact[fin]).max()) if fin.any() else 0.0
            if interp.shape != exact.shape or dev > 1e-3 * max(scale, 1e-30):
                skipped.append((prog, params, f"interpreter off the FP64 value by {dev:.3g}"))
                continue
            k = len(meta)
            arrays[f"{k}_ir"] = np.array(ir_text)
            for i, a in enumerate(ins):
                arrays[f"{k}_in{i}"] = a
            arrays[f"{k}_interp"] = interp
            cpp = got["cpp"]
            cpp_state = "failed" if cpp is None else (
                "same" if np.array_equal(cpp.view(np.uint32), interp.view(np.uint32)) else "differs")
            if cpp is not None:
                arrays[f"{k}_cpp"] = cpp
            meta.append((prog, params, seed, permute, len(ins), cpp_state))
    arrays["meta"] = np.array([repr(m) for m in meta])
    np.savez_compressed(OUT, **arrays)
    from collections import Counter

    print(f"{len(meta)} trees written to {OUT}; the cpp backend on them: "
          f"{dict(Counter(m[5] for m in meta))}; {len(skipped)} trees left out")
    for s in skipped:
        print("  skipped", s)


if __name__ == "__main__":
    main()
