"""Runs tests/cpp/reference_style_caller.cpp (a caller written like the
reference's gbench: src/bench/main.cpp:88-113, 218-249, 447-454, 539-553) against
include/graph_b200.hpp on the GPU: every BFS variant's depths through dist() equal
a serial BFS, traces arrive in a util::BfsLevel-shaped vector, and the PageRank
pulls meet L1 < 1e-4 against a double-precision PageRank with the reference's
result fields (iters, lastDelta, lastMaxRel, floorStop, gpuMs) filled in."""
import os
import subprocess

import pytest

from test_boundary import build_caller

pytestmark = pytest.mark.gpu


def test_reference_style_caller_runs(tmp_path):
    exe = str(tmp_path / "caller")
    build_caller(exe)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip().endswith("OK")
    for v in ("gpu_vertex", "gpu_naive", "gpu_binned", "gpu_edge", "gpu_do", "hybrid", "gpu_pull_adaptive"):
        assert f"{v} ok" in p.stdout
