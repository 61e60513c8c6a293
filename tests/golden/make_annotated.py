"""Generates tests/golden/annotated_cuda.json: the IR of every golden
program with the first loop at depth 0, 1 and 2 annotated "[cuda]" by the
reference's own annotate() (mutate.cpp:694-712) -- the annotation that makes
the reference's interpreter hand that sub-tree to the "cuda" backend
(compile.cpp:404-417).  Values are unchanged by the annotation, so each
tree's expected output is its golden fixture's.

    python tests/golden/make_annotated.py   (after make -C oracle)
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "lt_ref_harness")


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build the oracle first: make -C oracle REF=<reference checkout>")
    manifest = json.load(open(os.path.join(HERE, "manifest.json")))
    out = {}
    for m in manifest:
        if m["program"] == "log":  # not a lazy-frontend program
            continue
        for depth in (0, 1, 2):
            r = subprocess.run([HARNESS, "annotate", str(depth), "[cuda]", m["program"],
                                *map(str, m["params"])], capture_output=True, text=True)
            if r.returncode == 0:
                out.setdefault(m["name"], {})[str(depth)] = r.stdout
    json.dump(out, open(os.path.join(HERE, "annotated_cuda.json"), "w"), indent=0, sort_keys=True)
    print(sum(len(v) for v in out.values()), "annotated trees over", len(out), "programs")


if __name__ == "__main__":
    main()
