"""Drop-in check: the reference's own lazy frontend, LoopTree and Backend
registry drive the B200 backend through the reference-side plugin
(loop_tool_b200/plugin/cuda_backend_plugin.cpp loaded with loadLibrary and
made the default "cuda" backend/hardware).  The programs are the golden
cases; results must equal the reference's own CPU run of the same program.

Needs the reference CPU library built here (oracle/_ref, `make -C oracle
all plugin`); skipped when that build is absent.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from golden_util import EXACT_PROGRAMS, assert_accuracy, assert_parity, fp64_oracle, load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "lt_ref_harness")
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "libloop_tool_cuda_b200.so")
CASES = ["add_4099", "max_specials", "chain_513", "pad2d_128x16", "concat1d_kat",
         "concat2d_128", "transpose_flatten_kat", "rowmax_specials", "colsum_300x37",
         "fullsum_2x40000", "softmax_16x4096", "layernorm_8x256", "maxpool_specials",
         "mm_200x130x70", "bmm_3x16x8x24", "conv_2x4x8x8_pad1", "conv_2x3x9x9_s2",
         "padconv1d_16"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_reference_frontend_drives_b200(name, cuda_dev):
    if not (os.path.exists(HARNESS) and os.path.exists(PLUGIN)):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    case = load(name)
    with tempfile.TemporaryDirectory() as td:
        for i, a in enumerate(case["inputs"]):
            a.tofile(os.path.join(td, f"in{i}.f32"))
        env = dict(os.environ, LT_PLUGIN=PLUGIN)
        r = subprocess.run([HARNESS, "lazyrun", td, td, case["program"],
                            *map(str, case["params"])], env=env, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(os.path.join(td, "out0.f32"), dtype=np.float32)
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["softmax_16x4096", "add_4099", "maxpool_specials"])
def test_plugin_autotunes_and_persists_schedules(name, cuda_dev):
    """LOOP_TOOL_B200_AUTOTUNE=1: the first run of a loop tree through the
    reference frontend tunes it (outputs still exact / accurate) and writes
    the schedule file; a second process loads the file at registration."""
    if not (os.path.exists(HARNESS) and os.path.exists(PLUGIN)):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    case = load(name)
    with tempfile.TemporaryDirectory() as td:
        for i, a in enumerate(case["inputs"]):
            a.tofile(os.path.join(td, f"in{i}.f32"))
        sched = os.path.join(td, "schedules.txt")
        env = dict(os.environ, LT_PLUGIN=PLUGIN, LOOP_TOOL_B200_AUTOTUNE="1",
                   LOOP_TOOL_B200_SCHEDULES=sched)
        for _ in range(2):
            r = subprocess.run([HARNESS, "lazyrun", td, td, case["program"],
                                *map(str, case["params"])], env=env, capture_output=True,
                               text=True)
            assert r.returncode == 0, r.stderr
            got = np.fromfile(os.path.join(td, "out0.f32"), dtype=np.float32)
            if case["program"] in EXACT_PROGRAMS:
                assert_parity(got, case["expected"], True, what=name)
            else:
                assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)
            text = open(sched, "rb").read()
            assert text.startswith(b"loop_tool_b200 schedules 1\n") and b"\nentry " in text


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["add_4099", "softmax_16x4096", "mm_200x130x70",
                                  "conv_2x4x8x8_pad1"])
def test_plugin_pinned_host_memory(name, cuda_dev):
    """LOOP_TOOL_B200_HOST_MEMORY=pinned: the "cuda" hardware allocates the
    reference frontend's buffers as pinned host memory; results unchanged."""
    if not (os.path.exists(HARNESS) and os.path.exists(PLUGIN)):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    case = load(name)
    with tempfile.TemporaryDirectory() as td:
        for i, a in enumerate(case["inputs"]):
            a.tofile(os.path.join(td, f"in{i}.f32"))
        env = dict(os.environ, LT_PLUGIN=PLUGIN, LOOP_TOOL_B200_HOST_MEMORY="pinned")
        r = subprocess.run([HARNESS, "lazyrun", td, td, case["program"],
                            *map(str, case["params"])], env=env, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(os.path.join(td, "out0.f32"), dtype=np.float32)
    if case["program"] in EXACT_PROGRAMS:
        assert_parity(got, case["expected"], True, what=name)
    else:
        assert_accuracy(got, case["expected"], fp64_oracle(case), what=name)
