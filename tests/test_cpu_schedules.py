"""Schedule cache persistence (no device needed): the file format keeps the
serialized IR text, the options and one schedule line per stage."""
import pytest

import loop_tool_b200 as ltb
from loop_tool_b200._lib import LoopToolError

IR = open(__file__.replace("test_cpu_schedules.py", "golden/ir/mm_128.txt")).read()


def test_save_load_round_trip(tmp_path):
    ltb.tune_clear()
    opts = "precision=0;fuse_rows=1;tensor_cores=1;kahan_threshold=65536"
    body = (f"loop_tool_b200 schedules 1\n"
            f"entry 148 1 {len(IR.encode())} {len(opts)}\n{IR}{opts}\n"
            f"4 256 128 12.5\n")
    src = tmp_path / "in.txt"
    src.write_bytes(body.encode())
    ltb.tune_load(src)
    assert ltb.tune_entries() == 1
    out = tmp_path / "out.txt"
    ltb.tune_save(out)
    text = out.read_bytes()
    assert text.startswith(b"loop_tool_b200 schedules 1\n")
    assert IR.encode() in text and b"4 256 128 12.5" in text
    ltb.tune_clear()
    ltb.tune_load(out)
    assert ltb.tune_entries() == 1
    ltb.tune_clear()
    assert ltb.tune_entries() == 0


@pytest.mark.parametrize("body", [b"not a schedule file\n",
                                  b"loop_tool_b200 schedules 1\nentry x\n",
                                  b"loop_tool_b200 schedules 1\nentry 148 2 5 0\nabcde\n1 2 3 4\n"])
def test_malformed_files_rejected(tmp_path, body):
    ltb.tune_clear()
    p = tmp_path / "bad.txt"
    p.write_bytes(body)
    with pytest.raises(LoopToolError):
        ltb.tune_load(p)
    assert ltb.tune_entries() == 0


def test_missing_file_rejected(tmp_path):
    with pytest.raises(LoopToolError):
        ltb.tune_load(tmp_path / "absent.txt")
