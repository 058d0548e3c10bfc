"""The C++ boundary and gbench's command line, checked without a GPU.

* tests/cpp/reference_style_caller.cpp is written the way the reference's gbench
  drives gpu::GpuBfs / gpu::GpuPageRank (src/bench/main.cpp:88-113, 218-249,
  447-454, 539-553: the reference's option and result member names, GpuBfs(ctx, g)
  on a graph::CSR-shaped type, util::BfsLevel-shaped traces, dist() as the output
  buffer); it must compile against include/graph_b200.hpp with -Wall -Werror.
  tests/test_boundary_gpu.py runs it.
* gbench's CPU variants with --host-prep need no GPU: --schedule (cpu_omp's OpenMP
  schedule, src/bench/main.cpp:215, names as src/cpu/bfs_cpu.cpp:9-23), the
  PageRank CSV rows (src/bench/main.cpp:571-620) and the git_commit field
  (src/util/sysinfo.hpp:27-42)."""
import csv
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "graph_analytics_applesilicon_b200")
GBENCH = os.path.join(PKG, "bin", "gbench")
CALLER = os.path.join(ROOT, "tests", "cpp", "reference_style_caller.cpp")


def build_caller(out_path: str) -> None:
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), CALLER, "-o",
           out_path, "-L" + PKG, "-lgraphb200", "-Wl,-rpath," + PKG]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr


def test_reference_style_caller_compiles(tmp_path):
    if not os.path.exists(os.path.join(PKG, "libgraphb200.so")):
        pytest.fail("libgraphb200.so is not built")
    build_caller(str(tmp_path / "caller"))


def _gbench(args, cwd):
    if not os.path.exists(GBENCH):
        pytest.fail("gbench is not built")
    return subprocess.run([GBENCH, *args, "--host-prep"], capture_output=True, text=True, timeout=300, cwd=cwd)


@pytest.mark.parametrize("schedule,name", [("static", "static"), ("dynamic,64", "dynamic/64"),
                                           ("dynamic", "dynamic/64"), ("guided", "guided")])
def test_gbench_schedule(tmp_path, schedule, name):
    out = tmp_path / "r.csv"
    p = _gbench(["--graph", "synth:rmat12", "--algo", "bfs", "--variant", "cpu_omp", "--schedule", schedule,
                 "--validate", "--sources", "3", "--trials", "1", "--csv", str(out)], tmp_path)
    assert p.returncode == 0, p.stdout + p.stderr
    assert f"schedule={name}" in p.stdout and "validated OK" in p.stdout
    rows = list(csv.DictReader(open(out)))
    assert len(rows) == 3 and all(r["params"].endswith(f"schedule={name}") for r in rows)


def test_gbench_unknown_schedule_is_an_error(tmp_path):
    p = _gbench(["--graph", "synth:rmat12", "--algo", "bfs", "--variant", "cpu_omp", "--schedule", "bogus"],
                tmp_path)
    assert p.returncode == 1 and "unknown schedule 'bogus'" in p.stderr


def test_gbench_pagerank_csv_rows(tmp_path):
    out = tmp_path / "pr.csv"
    for tol, trials in (("0", "2"), ("1e-7", "3")):
        p = _gbench(["--graph", "synth:rmat12_directed", "--algo", "pr", "--variant", "cpu_omp", "--tol", tol,
                     "--validate", "--trials", trials, "--csv", str(out)], tmp_path)
        assert p.returncode == 0, p.stdout + p.stderr
    rows = list(csv.DictReader(open(out)))
    assert len(rows) == 5
    assert all(r["algo"] == "pr" and r["source"] == "" and r["validated"] == "1" for r in rows)
    assert [r["trial"] for r in rows] == ["0", "1", "0", "1", "2"]
    assert rows[0]["params"].startswith("iters=20") and rows[0]["iters"] == "20"
    assert rows[2]["params"].startswith("tol=1e-07 cap=1000")  # %g, not a fixed 6 decimals
    it = int(rows[2]["iters"])
    assert 5 < it < 1000
    m = int(rows[2]["m"])
    assert float(rows[2]["gteps"]) == pytest.approx(m * it / (float(rows[2]["time_ms_e2e"]) * 1e6), rel=1e-3)


def test_gbench_git_commit_field(tmp_path):
    """In a git checkout the field is the short hash of HEAD (+ when tracked
    files are modified); outside one it is 'unknown'."""
    out = tmp_path / "r.csv"
    args = ["--graph", "synth:path1000", "--algo", "bfs", "--variant", "cpu_serial", "--sources", "1",
            "--trials", "1", "--csv", str(out)]
    p = _gbench(args, ROOT)
    assert p.returncode == 0, p.stderr
    head = subprocess.run(["git", "rev-parse", "--short", "HEAD"], capture_output=True, text=True, cwd=ROOT)
    got = list(csv.DictReader(open(out)))[-1]["git_commit"]
    if head.returncode == 0 and head.stdout.strip():
        assert got.rstrip("+") == head.stdout.strip()
    else:
        assert got == "unknown"
    out2 = tmp_path / "r2.csv"
    p = _gbench(args[:-1] + [str(out2)], tmp_path)  # tmp_path is no checkout
    assert p.returncode == 0
    assert list(csv.DictReader(open(out2)))[-1]["git_commit"] == "unknown"
