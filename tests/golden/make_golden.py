"""Generates the golden fixtures in tests/golden/ from the reference itself.

For every case the reference lazy frontend (built from the reference sources
by oracle/Makefile into oracle/_ref/) emits the serialized IR of the program
(serialization.cpp:175-237) at the given sizes; seeded inputs are drawn with
numpy; the reference's two CPU backends ("cpp", the default C-codegen
backend, and "cpu_interpreted") run that exact IR; IR text, inputs and both
outputs are stored in one .npz per case, next to the output of the same
program run through the lazy frontend directly (out0_lazy, the expected
value: a serialize/deserialize round trip re-creates symbols per node and
the reference's Compiler then misses some view constraints, e.g. the first
operand of a concatenation reads index 0).

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py [case names...]
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")
OUT = os.path.dirname(os.path.abspath(__file__))

# (name, program, params, seed, input kind)
CASES = [
    # elementwise / broadcast (family a)
    ("add_1000", "add", [1000], 201, "randn"),
    ("add_4099", "add", [4099], 202, "randn"),
    ("sub_257", "sub", [257], 203, "randn"),
    ("mul_129", "mul", [129], 204, "randn"),
    ("div_1000", "div", [1000], 205, "randn"),
    ("min_specials", "min", [1024], 206, "specials"),
    ("max_specials", "max", [1024], 207, "specials"),
    ("exp_1000", "exp", [1000], 208, "randn"),
    # log (compile.cpp:1036-1081, op 11): the lazy frontend has no log
    # (lazy.cpp:221-270), so its IR is the reference's exp IR with the op
    # replaced, run by both CPU backends
    ("log_1000", "log", [1000], 233, "log"),
    ("sqrt_1000", "sqrt", [1000], 209, "abs"),
    ("neg_specials", "neg", [512], 210, "specials"),
    ("recip_1000", "recip", [1000], 211, "randn"),
    ("abs_specials", "abs", [512], 212, "specials"),
    ("chain_513", "chain", [513], 213, "randn"),
    ("scale_kat", "scale", [8], 214, "scale_kat"),
    ("bcast_add_16x64", "bcast_add", [16, 64], 215, "randn"),
    # views: pad / concat / transpose / flatten (bit-exact index semantics)
    ("pad1d_kat", "pad1d", [5, 1, 1], 0, "arange"),
    ("pad2d_128x16", "pad2d", [128, 16, 3], 216, "randn"),
    ("concat1d_kat", "concat1d", [8, 5], 0, "arange"),
    ("concat2d_kat", "concat2d", [2, 5, 3], 0, "concat2d_kat"),
    ("concat2d_128", "concat2d", [128, 16, 5], 217, "randn"),
    ("transpose_flatten_kat", "transpose_flatten", [8, 8], 0, "transpose_kat"),
    ("flatten_kat", "flatten", [8, 8], 0, "arange"),
    ("transpose_33x17", "transpose", [33, 17], 218, "randn"),
    # reductions (family b)
    ("rowsum_37x300", "rowsum", [37, 300], 219, "randn"),
    ("rowmax_specials", "rowmax", [37, 300], 220, "specials"),
    ("rowmin_specials", "rowmin", [29, 1000], 221, "specials"),
    ("colsum_300x37", "colsum", [300, 37], 222, "randn"),
    ("colmax_specials", "colmax", [300, 37], 223, "specials"),
    ("fullsum_2x40000", "fullsum", [2, 40000], 224, "randn"),
    # compensated row sums (rows above 65536) meeting inf, -inf, inf + -inf
    # and overflow: the plain sequential loop's inf / -inf / NaN
    ("rowsum_specials_5x70000", "rowsum", [5, 70000], 234, "sum_specials"),
    ("softmax_16x32", "softmax", [16, 32], 225, "softmax"),
    ("softmax_16x4096", "softmax", [16, 4096], 226, "softmax"),
    ("mean_rows_4x8", "mean_rows", [4, 8], 227, "ones_last"),
    ("layernorm_8x256", "layernorm", [8, 256], 228, "layernorm"),
    ("maxpool_2x3x8x8", "maxpool", [2, 3, 8, 8, 2, 2], 229, "randn"),
    ("maxpool_specials", "maxpool", [2, 4, 12, 12, 2, 2], 230, "specials"),
    ("maxpool_k3s2", "maxpool", [1, 2, 11, 11, 3, 2], 231, "randn"),
    # contractions (family c)
    ("mm_16", "mm", [16, 16, 16], 101, "randn"),
    ("mm_128", "mm", [128, 128, 128], 102, "randn"),
    ("mm_17x33x9", "mm", [17, 33, 9], 103, "randn"),
    ("mm_200x130x70", "mm", [200, 130, 70], 104, "randn"),
    ("bmm_3x16x8x24", "bmm", [3, 16, 8, 24], 105, "randn"),
    ("conv1d_kat", "conv1d", [10, 3], 0, "ones"),
    ("padconv1d_16", "padconv1d", [16, 3, 1], 232, "randn"),
    ("conv_2x4x8x8_pad1", "conv", [2, 4, 8, 8, 8, 3, 1, 1], 301, "conv"),
    ("conv_1x3x7x9_nopad", "conv", [1, 3, 7, 9, 5, 3, 0, 1], 302, "conv"),
    ("conv_2x3x9x9_s2", "conv", [2, 3, 9, 9, 4, 3, 1, 2], 303, "conv"),
]


def harness(*args, check=True):
    r = subprocess.run([HARNESS, *map(str, args)], capture_output=True, text=True)
    if check and r.returncode != 0:
        raise RuntimeError(f"harness {args} failed: {r.stderr}")
    return r


def make_inputs(kind, sizes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        if kind == "randn":
            a = rng.standard_normal(n)
        elif kind == "abs":
            a = np.abs(rng.standard_normal(n))
        elif kind == "sum_specials":  # rows: +inf, -inf, both, overflow, plain
            a = rng.standard_normal(n).reshape(5, -1)
            a[0, 1234] = np.inf
            a[1, 40000] = -np.inf
            a[2, 10] = np.inf
            a[2, 69000] = -np.inf
            a[3, :] = 3e38
            a = a.ravel()
        elif kind == "log":  # positive values, plus log's special arguments
            a = np.abs(rng.standard_normal(n)) * 10.0 ** rng.integers(-30, 30, n)
            a[:6] = [0.0, -0.0, 1.0, np.inf, -1.0, np.nan]
        elif kind == "softmax":
            a = 4.0 * rng.standard_normal(n)
        elif kind == "specials":
            a = rng.standard_normal(n)
            a[rng.random(n) < 0.15] = 0.0
            a[rng.random(n) < 0.15] = -0.0
            a[rng.random(n) < 0.03] = np.inf
            a[rng.random(n) < 0.03] = -np.inf
            a[rng.random(n) < 0.02] = np.nan
        elif kind == "arange":
            a = np.arange(n, dtype=np.float64)
        elif kind == "ones":
            a = np.ones(n)
        elif kind == "ones_last":
            a = rng.standard_normal(n) if i == 0 else np.ones(n)
        elif kind == "transpose_kat":  # test_lazy.cpp:271-273
            idx = np.arange(n)
            a = (idx % 8 * 8 + idx // 8).astype(np.float64)
        elif kind == "concat2d_kat":  # test_lazy.cpp:397-403
            a = np.full(n, 11.0 if i == 0 else 7.0)
        elif kind == "scale_kat":  # test_lazy.cpp:227-240
            a = np.arange(n, dtype=np.float64) if i == 0 else np.full(n, 2.0)
        elif kind == "layernorm":
            a = rng.standard_normal(n) if i == 0 else (np.full(n, 256.0) if i == 1 else np.full(n, 1e-5))
        elif kind == "conv":
            if i == 0:
                a = rng.standard_normal(n)
            else:  # Kaiming-uniform weights
                fan_in = max(n // 8, 1)
                bound = np.sqrt(6.0 / fan_in)
                a = rng.uniform(-bound, bound, n)
        else:
            raise ValueError(kind)
        out.append(a.astype(np.float32))
    return out


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build the oracle first: make -C oracle")
    only = set(sys.argv[1:])  # case names to (re)generate; default all
    manifest = []
    if only:
        manifest = [m for m in json.load(open(os.path.join(OUT, "manifest.json")))
                    if m["name"] not in only]
    for name, prog, params, seed, kind in CASES:
        if only and name not in only:
            continue
        if prog == "log":
            ir = harness("ir", "exp", *params).stdout
            assert "\nn:12:" in ir
            ir = ir.replace("\nn:12:", "\nn:11:")
        else:
            ir = harness("ir", prog, *params).stdout
        with tempfile.TemporaryDirectory() as td:
            irf = os.path.join(td, "ir.txt")
            open(irf, "w").write(ir)
            sizes = json.loads(harness("sizes", irf).stdout)
            inputs = make_inputs(kind, sizes["inputs"], seed)
            for i, a in enumerate(inputs):
                a.tofile(os.path.join(td, f"in{i}.f32"))
            outs = {}
            for backend in ("cpp", "cpu_interpreted"):
                od = os.path.join(td, backend)
                os.makedirs(od)
                # the interpreter rejects some ops the C path handles
                # (compile.cpp:253-256 has no reset for abs/log)
                r = harness("run", irf, backend, td, od, check=backend == "cpp")
                if r.returncode != 0:
                    outs[backend] = []
                    continue
                outs[backend] = [
                    np.fromfile(os.path.join(od, f"out{j}.f32"), dtype=np.float32)
                    for j in range(len(sizes["outputs"]))
                ]
            # the lazy frontend's own run (no serialize round trip): the
            # expected values -- deserialize() gives every node fresh
            # symbols, which changes some view index equations
            if prog == "log":  # no view in the tree: the C path's output
                outs["lazy"] = outs["cpp"]
            else:
                ld = os.path.join(td, "lazy")
                os.makedirs(ld)
                harness("lazyrun", ld, td, prog, *params)
                outs["lazy"] = [np.fromfile(os.path.join(ld, "out0.f32"), dtype=np.float32)]
            tree = harness("tree", irf).stdout
        arrays = {f"in{i}": a for i, a in enumerate(inputs)}
        arrays["out0_lazy"] = outs["lazy"][0]
        for j, o in enumerate(outs["cpp"]):
            arrays[f"out{j}_cpp"] = o
        for j, o in enumerate(outs["cpu_interpreted"]):
            arrays[f"out{j}_interp"] = o
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            ir=np.array(ir),
            tree=np.array(tree),
            program=np.array(prog),
            params=np.array(params, dtype=np.int64),
            seed=np.array(seed),
            kind=np.array(kind),
            **arrays,
        )
        manifest.append({"name": name, "program": prog, "params": params,
                         "seed": seed, "kind": kind,
                         "n_in": len(inputs), "n_out": len(sizes["outputs"])})
        print(f"{name}: {len(inputs)} in, {len(sizes['outputs'])} out")
    order = [c[0] for c in CASES]
    manifest.sort(key=lambda m: order.index(m["name"]))
    json.dump(manifest, open(os.path.join(OUT, "manifest.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
