"""The Viterbi shape tuner's C emitter: the table it writes compiles and
lists the ranges the tuner chose (CPU only; the timing itself needs a GPU)."""
import os
import subprocess
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "sentinel-x_b200"))
from sxhmm import tune  # noqa: E402

SHAPES = [(1, 8, 0), (4, 8, 1), (8, 16, 0), (32, 64, 0)]


def _compile_and_dump(tmp_path, src):
    (tmp_path / "t.inc").write_text(src)
    (tmp_path / "main.cpp").write_text(
        '#include <cstdio>\n#include "t.inc"\n'
        "int main() { for (const auto& r : kTunedVit) std::printf(\"%d %d %d %d %d\\n\", r[0], r[1], r[2], r[3], r[4]); }\n")
    exe = tmp_path / "dump"
    subprocess.run(["g++", "-std=c++17", "-o", str(exe), str(tmp_path / "main.cpp")], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return [tuple(int(v) for v in line.split()) for line in out.splitlines()]


def test_emit_inc_ranges(tmp_path):
    t = np.full(tune.MAX_M + 1, -1, np.int32)
    t[1:33] = 1
    t[33:129] = 2
    t[1537:2049] = 3
    rows = _compile_and_dump(tmp_path, tune.emit_inc(t, SHAPES))
    assert rows == [(1, 32, 4, 8, 1), (33, 128, 8, 16, 0), (1537, 2048, 32, 64, 0), (0, -1, 0, 0, 0)]


def test_emit_inc_empty(tmp_path):
    rows = _compile_and_dump(tmp_path, tune.emit_inc(np.full(tune.MAX_M + 1, -1, np.int32), SHAPES))
    assert rows == [(0, -1, 0, 0, 0)]
