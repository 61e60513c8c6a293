"""Loop annotations of the LoopTree drive the lowering (ltb_plan, on the
host): "parallel" pins thread counts and parallel reductions, "unroll"
items per thread, "[cuda]" sub-trees run on the device with the rest of the
tree, and a sub-tree annotated for another backend is rejected."""
import json
import os

import pytest

import loop_tool_b200 as lt
from golden_util import GOLDEN, load
from ir_edit import get_order, nodes_with_loops, set_order


def tutorial_add(n=1 << 20, parallel=8 * 1024, inner=4):
    """The reference tutorial's CUDA schedule of a pointwise add
    (tutorial.ipynb: split N into (size, tail) x parallel x inner and
    annotate the middle loop "parallel")."""
    text = open(os.path.join(GOLDEN, "ir", "add_2p28.txt")).read().replace(";268435456;", f";{n};")
    size, tail = n // (parallel * inner), n % (parallel * inner)
    for k in nodes_with_loops(text):
        (v, _, _), = get_order(text, k)[0]
        text = set_order(text, k, [(v, size, tail), (v, parallel, 0), (v, inner, 0)],
                         ["", "parallel", ""])
    return text


def test_parallel_pins_thread_count():
    plain = open(os.path.join(GOLDEN, "ir", "add_2p28.txt")).read().replace(";268435456;", ";1048576;")
    assert "pinned" not in lt.plan(plain)
    p = lt.plan(tutorial_add())
    assert "pinned{ parallel=8192 }" in p, p


def test_two_parallel_loops_give_cta_size():
    text = tutorial_add()
    for k in nodes_with_loops(text):
        order, _ = get_order(text, k)
        text = set_order(text, k, order, ["parallel", "parallel", ""])
    p = lt.plan(text)
    assert "parallel=" + str(32 * 8192) in p and "cta=8192" in p, p


def test_parallel_reduced_var_makes_a_parallel_reduction():
    case = load("rowsum_37x300")
    ir = case["ir"]
    base = lt.plan(ir)
    # the sum node: order r, n -> r, n(3), n(100) with n(3) parallel
    k = [k for k in nodes_with_loops(ir) if len(get_order(ir, k)[0]) == 2 and
         ir.splitlines()[[i for i, l in enumerate(ir.splitlines()) if l.startswith("n:")][k]].startswith("n:5:")][0]
    (r, rs, _), (n, ns, _) = get_order(ir, k)[0]
    ann = set_order(ir, k, [(r, rs, 0), (n, 3, 0), (n, 100, 0)], ["", "parallel", ""])
    p = lt.plan(ann)
    assert "parallel_reduce=3" in p, p
    big = set_order(ir, k, [(r, rs, 0), (n, 300, 0)], ["", "parallel"])
    assert "reduce_split" in lt.plan(big).split("\n")[1] or "parallel_reduce=300" in lt.plan(big)
    assert base != p


def test_unroll_recorded():
    case = load("maxpool_2x3x8x8")
    ir = case["ir"]
    k = nodes_with_loops(ir)[-2]
    order, _ = get_order(ir, k)
    ann = set_order(ir, k, order, [""] * (len(order) - 1) + ["unroll"])
    assert "unroll=" in lt.plan(ann)


def test_other_backend_subtree_rejected():
    case = load("add_1000")
    ir = case["ir"]
    k = nodes_with_loops(ir)[0]
    order, _ = get_order(ir, k)
    with pytest.raises(lt.LoopToolError, match="annotated for backend 'cpp'"):
        lt.plan(set_order(ir, k, order, ["[cpp]"]))


ANNOTATED = json.load(open(os.path.join(GOLDEN, "annotated_cuda.json")))


@pytest.mark.parametrize("name", sorted(ANNOTATED))
def test_cuda_subtrees_plan(name):
    for depth, ir in ANNOTATED[name].items():
        p = lt.plan(ir)
        assert "[cuda] sub-tree" in p, (name, depth, p)


def test_annotated_set_size():
    assert sum(len(v) for v in ANNOTATED.values()) >= 80
