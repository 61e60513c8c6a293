"""Parity on randomly scheduled loop trees: the reference's own programs
given rand_sched-style schedules (test/test.py:56-96, 289-313: every var
split into up to three loops with random factors and tails, sizes 2^i,
2^i + 1 and primes; half of the trees also with their var groups
reordered), run through the C ABI and compared with the reference
interpreter on the same tree: bit-exact where the reference's arithmetic
is exact or follows one order, else elementwise against the FP64 oracle."""
import numpy as np
import pytest

from fuzz_util import case_id, cases, load
from golden_util import EXACT_PROGRAMS, assert_accuracy, assert_parity, fp64_oracle


@pytest.mark.gpu
@pytest.mark.parametrize("k", cases(), ids=case_id)
def test_fuzzed_schedule(k, cuda_dev):
    import torch

    import loop_tool_b200 as lt

    c = load(k)
    comp = lt.cuda(c["ir"])
    ins = [torch.from_numpy(a).to(cuda_dev) for a in c["inputs"]]
    out = torch.full((comp.io_sizes[-1],), 1337.0, device=cuda_dev)
    comp(ins + [out])
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    name = case_id(k)
    if c["program"] in EXACT_PROGRAMS:
        assert_parity(got, c["expected"], True, what=name)
    else:
        assert_accuracy(got, c["expected"], fp64_oracle(c), what=name)
