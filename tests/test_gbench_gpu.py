"""gbench end to end on the GPU: graph preparation (and --ordering degree /
rcm) on the device (the default) against --host-prep on the same command line.  Both runs must validate against
the serial CPU BFS / FP64 PageRank and write byte-identical distances and ranks
with the same sources, the contract of the reference's gbench
(bench/gbench.cpp: prep, source picking, --validate)."""
import csv
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GBENCH = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "graph_analytics_applesilicon_b200", "bin", "gbench")


def _run(tmp_path, tag, args, host):
    out = tmp_path / f"{tag}_{'host' if host else 'gpu'}"
    out.mkdir()
    bfs = "bfs" in args
    cmd = [GBENCH, *args, "--validate", "--csv", str(out / "r.csv")]
    cmd += ["--dump-dist" if bfs else "--dump-ranks", str(out / "d.bin")]
    if host:
        cmd.append("--host-prep")
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    with open(out / "r.csv") as f:
        rows = list(csv.DictReader(f))
    return rows, (out / "d.bin").read_bytes()


CASES = {
    "rmat12_directed_bfs": ["--graph", "synth:rmat12_directed", "--algo", "bfs", "--variant", "gpu_do_persistent",
                            "--sources", "8", "--trials", "1"],
    "two_components_bfs": ["--graph", "synth:two_components", "--algo", "bfs", "--variant", "gpu_do",
                           "--sources", "4", "--trials", "1"],
    "rmat12_random_order_bfs": ["--graph", "synth:rmat12", "--algo", "bfs", "--variant", "gpu_do_persistent",
                                "--ordering", "random", "--order-seed", "5", "--sources", "8", "--trials", "1"],
    "grid_batch_bfs": ["--graph", "synth:grid100x100", "--algo", "bfs", "--variant", "gpu_do_persistent",
                       "--batch", "64", "--sources", "64", "--trials", "1"],
    "rmat12_directed_pr": ["--graph", "synth:rmat12_directed", "--algo", "pr", "--variant", "gpu_pull_scalar",
                           "--iters", "20", "--trials", "1"],
    "grid_pr": ["--graph", "synth:grid100x100", "--algo", "pr", "--variant", "gpu_pull_adaptive",
                "--iters", "20", "--trials", "1"],
    "rmat12_rcm_bfs": ["--graph", "synth:rmat12", "--algo", "bfs", "--variant", "gpu_do_persistent",
                       "--ordering", "rcm", "--sources", "8", "--trials", "1"],
    "grid_degree_bfs": ["--graph", "synth:grid100x100", "--algo", "bfs", "--variant", "gpu_do",
                        "--ordering", "degree", "--sources", "4", "--trials", "1"],
    "rmat12_directed_rcm_pr": ["--graph", "synth:rmat12_directed", "--algo", "pr", "--variant", "gpu_pull_adaptive",
                               "--ordering", "rcm", "--iters", "20", "--trials", "1"],
    "rmat12_directed_degree_gs": ["--graph", "synth:rmat12_directed", "--algo", "pr", "--variant", "gpu_pull_gs",
                                  "--ordering", "degree", "--tol", "1e-6", "--trials", "1"],
    # --ref-tol: Gauss-Seidel at a tighter tol judged against the Jacobi reference at 1e-6
    "rmat12_directed_gs_ref_tol": ["--graph", "synth:rmat12_directed", "--algo", "pr", "--variant", "gpu_pull_gs",
                                   "--tol", "1e-8", "--ref-tol", "1e-6", "--trials", "1"],
    # --T: the reference's hybrid threshold, accepted; hybrid runs the persistent kernel
    "rmat12_hybrid_T": ["--graph", "synth:rmat12", "--algo", "bfs", "--variant", "hybrid", "--T", "5000",
                        "--sources", "4", "--trials", "1"],
}


@pytest.mark.parametrize("tag", sorted(CASES))
def test_gbench_gpu_prep_matches_host_prep(tmp_path, tag):
    if not os.path.exists(GBENCH):
        pytest.fail("gbench is not built")
    rows_g, dump_g = _run(tmp_path, tag, CASES[tag], host=False)
    rows_h, dump_h = _run(tmp_path, tag, CASES[tag], host=True)
    assert len(rows_g) == len(rows_h) > 0
    assert all(r["validated"] == "1" for r in rows_g)
    assert [r["source"] for r in rows_g] == [r["source"] for r in rows_h]
    assert [(r["n"], r["m"]) for r in rows_g] == [(r["n"], r["m"]) for r in rows_h]
    if "bfs" in CASES[tag]:
        assert dump_g == dump_h  # distances: exact
        assert len(rows_g) > 0
        d = np.frombuffer(dump_g, np.uint32)
        assert (d == 0).sum() == 1  # the dumped source
    else:
        # ranks: FP32 sweeps whose block sums may combine in either order
        assert all(r["algo"] == "pr" and r["source"] == "" and int(r["iters"]) > 0 for r in rows_g)
        a, b = np.frombuffer(dump_g, np.float64), np.frombuffer(dump_h, np.float64)
        assert a.size == b.size > 0
        assert np.abs(a - b).sum() < 1e-6
