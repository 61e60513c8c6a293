"""The C ABI library loads, exports every declared symbol, and lowers every
golden loop tree on the host (no GPU needed)."""
import os
import re

import pytest

from golden_util import load, manifest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "loop_tool_b200.h")).read()
    return sorted(set(re.findall(r"\b(ltb_[a-z_]+)\s*\(", hdr)))


def test_header_symbols_exported():
    from loop_tool_b200 import _lib

    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/loop_tool_b200.h but not exported"
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_abi_version_and_no_device_compile():
    import loop_tool_b200 as lt
    from loop_tool_b200 import _lib

    assert _lib.lib().ltb_abi_version() == 1
    if lt.device_count() == 0:
        with pytest.raises(lt.LoopToolError) as e:
            lt.cuda(load("add_1000")["ir"])
        assert e.value.code == _lib.ERR_NO_DEVICE


@pytest.mark.parametrize("name", [m["name"] for m in manifest()])
def test_plan_every_golden_ir(name):
    import loop_tool_b200 as lt

    p = lt.plan(load(name)["ir"])
    assert "stage(s)" in p


def test_plan_families():
    import loop_tool_b200 as lt

    assert "contraction" in lt.plan(load("mm_128")["ir"])
    assert "row_chain" in lt.plan(load("softmax_16x4096")["ir"])
    assert "reduce_serial" in lt.plan(load("maxpool_2x3x8x8")["ir"])
    assert "reduce_split" in lt.plan(load("fullsum_2x40000")["ir"])
    conv = lt.plan(load("conv_2x4x8x8_pad1")["ir"])
    assert "contraction" in conv and "A-guarded" in conv


def test_bad_ir_raises():
    import loop_tool_b200 as lt

    with pytest.raises(lt.LoopToolError):
        lt.plan("n:99::::::::::\n")
    with pytest.raises(lt.LoopToolError):
        lt.plan("v:a\nn:2::0,:::0:::::\nn:5:0,7,:0,:::0:::::\ni:0,\no:1,\n")
