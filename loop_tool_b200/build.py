"""Builds the in-tree CUDA extension (sm_100a): ``python -m loop_tool_b200.build``."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8, verbose=False):
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("CUDA extension build failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return os.path.join(HERE, "_lib", "libloop_tool_b200.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
