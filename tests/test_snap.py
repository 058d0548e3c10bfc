"""SNAP edge-list converter, CPU side: the oracle's restatement of
graph::convertSnap (src/graph/snap.cpp:17-149) against the reference's own
results recorded in tests/golden/snap_golden.json, and against the reference
build itself on an R-MAT dump (the property of the reference's
converter_matches_in_memory_build test, tests/test_main.cpp:240-275)."""
import hashlib
import os

import numpy as np
import pytest

import snap_cases as S


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _cases(golden):
    cases = dict(S.SMALL)
    cases.update(S.long_cases())
    for name, (lines, seed) in golden["random"].items():
        cases[name] = S.random_text(lines, seed)
    return cases


def _check(rec, path, run):
    """run() -> (graph, stats) or raises; compare with one golden record."""
    if "error" in rec:
        with pytest.raises(Exception) as e:
            run()
        assert rec["error"].format(path=path) in str(e.value)
        return None
    g, st = run()
    for k in ("lines", "raw_max_id", "n", "m_before", "m"):
        assert st[k] == rec[k], (path, k)
    assert (g.n, g.m, g.flags) == (rec["n"], rec["m"], rec["flags"])
    assert _sha(g.row_ptr) == rec["row_ptr"] and _sha(g.col_idx) == rec["col_idx"]
    return g


def test_oracle_converter_matches_reference_golden(oracle, snap_golden, tmp_path):
    cases = _cases(snap_golden)
    seen = 0
    for key, rec in sorted(snap_golden["cases"].items()):
        name, fmt, d = key.split("|")
        path = S.write_case(cases[name], str(tmp_path), name, fmt == "gz")
        _check(rec, path, lambda: oracle.convert_snap(path, d == "dir"))
        os.unlink(path)
        seen += 1
    assert seen == len(snap_golden["cases"]) >= 100


def test_oracle_converter_matches_reference_on_rmat_dump(oracle, tmp_path):
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    g = oracle.gen("rmat", 12, 16, 1, 7)
    path = S.write_case(S.rmat_dump(g), str(tmp_path), "rmat", gz=True)
    for directed in (True, False):
        h, st = oracle.convert_snap(path, directed)
        r, rst = oracle.ref_convert_snap(path, str(tmp_path / "out.bin"), directed)
        assert st == rst and h.equal(r.host())
    # the dump drops isolated vertices; relabelling keeps the order of the rest
    h, _ = oracle.convert_snap(path, True)
    present = np.zeros(g.n, bool)
    present[np.repeat(np.arange(g.n), np.diff(g.row_ptr.astype(np.int64)))] = True
    present[g.col_idx] = True
    keep = np.flatnonzero(present).astype(np.uint32)
    new = np.full(g.n, 0xFFFFFFFF, np.uint32)
    new[keep] = np.arange(keep.size, dtype=np.uint32)
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr.astype(np.int64)))
    want = oracle.from_edges(keep.size, new[rows], new[g.col_idx], True)
    assert h.equal(want)


def test_gconvert_usage_errors():
    """Usage errors exit 2 before any conversion (src/graph/convert.cpp:13-17)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "graph_analytics_applesilicon_b200", "bin", "gconvert")
    if not os.path.exists(exe):
        pytest.skip("gconvert not built")
    for argv in ([], ["a.txt", "b.bin"], ["a.txt", "b.bin", "--directed", "--undirected"], ["a.txt", "--directed"]):
        p = subprocess.run([exe, *argv], capture_output=True, text=True, timeout=60)
        assert p.returncode == 2 and "usage: gconvert" in p.stderr
