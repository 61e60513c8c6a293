"""The randomly scheduled loop trees of tests/golden/schedule_fuzz.npz
(made by tests/golden/make_schedule_fuzz.py)."""
import ast
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "schedule_fuzz.npz")
_Z = []


def _z():
    if not _Z:
        _Z.append(np.load(PATH))
    return _Z[0]


def cases():
    """Indices of every tree, grouped ids for pytest."""
    return list(range(len(_z()["meta"])))


def load(k):
    z = _z()
    prog, params, seed, permute, n_in, cpp_state = ast.literal_eval(str(z["meta"][k]))
    return {
        "program": prog, "params": params, "seed": seed, "permute": permute,
        "ir": str(z[f"{k}_ir"]),
        "inputs": [z[f"{k}_in{i}"] for i in range(n_in)],
        # the reference interpreter's output on the scheduled tree (checked
        # against the FP64 dataflow value when the fixtures were made)
        "expected": z[f"{k}_interp"],
        "cpp": z[f"{k}_cpp"] if f"{k}_cpp" in z.files else None,
        "cpp_state": cpp_state,
    }


def case_id(k):
    c = load(k)
    return f"{k}-{c['program']}-{'x'.join(map(str, c['params']))}"
