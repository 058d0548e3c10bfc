"""SNAP edge-list converter on the GPU (gb_csr_from_snap_gpu /
gb_convert_snap_gpu) against the reference's own results
(tests/golden/snap_golden.json: graph::convertSnap compiled from the
reference sources) and against the oracle: the line rules, every error with
the reference's message and first-failing-line order, the 4 MiB line limit
found on the device (inside a chunk) and on the host (a line longer than a
chunk), chunk boundaries, gzip, and an R-MAT round trip.  Integer work: every
comparison is exact."""
import hashlib
import os

import numpy as np
import pytest

import snap_cases as S

pytestmark = pytest.mark.gpu

MIN_CHUNK = (4 << 20) + 1


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _cases(golden):
    cases = dict(S.SMALL)
    cases.update(S.long_cases())
    for name, (lines, seed) in golden["random"].items():
        cases[name] = S.random_text(lines, seed)
    return cases


def _check(gb, rec, path, directed, chunk=0):
    if "error" in rec:
        with pytest.raises(gb.GraphError) as e:
            gb.from_snap_gpu(path, directed, chunk)
        assert rec["error"].format(path=path) in str(e.value), path
        assert e.value.status == 1  # GB_ERR_ARG
        return
    g, st = gb.from_snap_gpu(path, directed, chunk)
    for k in ("lines", "raw_max_id", "n", "m_before", "m"):
        assert st[k] == rec[k], (path, k)
    assert (g.n, g.m, g.flags) == (rec["n"], rec["m"], rec["flags"]), path
    assert _sha(g.row_ptr) == rec["row_ptr"] and _sha(g.col_idx) == rec["col_idx"], path


def test_snap_gpu_matches_reference_golden(gb, snap_golden, tmp_path):
    cases = _cases(snap_golden)
    for key, rec in sorted(snap_golden["cases"].items()):
        name, fmt, d = key.split("|")
        path = S.write_case(cases[name], str(tmp_path), name, fmt == "gz")
        _check(gb, rec, path, d == "dir")
        os.unlink(path)


def test_snap_gpu_long_lines_with_smallest_chunk(gb, snap_golden, tmp_path):
    """At 4 MiB + 1 bytes per chunk a 4 MiB line fills a chunk exactly (found
    by the device) and the 9 MiB comment overflows one (found by the host)."""
    cases = S.long_cases()
    for name, data in cases.items():
        path = S.write_case(data, str(tmp_path), name)
        for d in ("dir", "undir"):
            _check(gb, snap_golden["cases"][f"{name}|txt|{d}"], path, d == "dir", MIN_CHUNK)


@pytest.mark.parametrize("chunk", [MIN_CHUNK, 5_000_011, 0])
def test_snap_gpu_chunk_boundaries_match_oracle(gb, oracle, tmp_path, chunk):
    data = S.random_text(1_500_000, 11, max_id=3_000_000)  # ~24 MB: several chunks
    path = S.write_case(data, str(tmp_path), "rnd", gz=chunk == 0)
    for directed in (True, False):
        want, wst = oracle.convert_snap(path, directed)
        g, st = gb.from_snap_gpu(path, directed, chunk)
        assert {k: st[k] for k in wst} == wst
        assert g.equal(want)


def test_snap_gpu_rmat_round_trip(gb, oracle, tmp_path):
    g = oracle.gen("rmat_edges", 16, 16 << 16, 1, 9)
    path = S.write_case(S.rmat_dump(g), str(tmp_path), "rmat16", gz=True)
    for directed in (True, False):
        want, wst = oracle.convert_snap(path, directed)
        h, st = gb.from_snap_gpu(path, directed)
        assert {k: st[k] for k in wst} == wst
        assert h.equal(want)
    # the file converter writes the same graph as a .bin
    out = str(tmp_path / "rmat16.bin")
    st = gb.convert_snap_gpu(path, out, True)
    back = gb.load(out)
    want, _ = oracle.convert_snap(path, True)
    assert back.equal(want) and st["n"] == want.n and st["m"] == want.m


def test_snap_gpu_errors(gb, tmp_path):
    with pytest.raises(gb.GraphError) as e:
        gb.from_snap_gpu(str(tmp_path / "absent.txt"), True)
    assert e.value.status == 6 and "cannot open" in str(e.value)  # GB_ERR_IO
    path = S.write_case(b"1 2\n", str(tmp_path), "one")
    with pytest.raises(gb.GraphError) as e:
        gb.from_snap_gpu(path, True, 1 << 20)  # below the 4 MiB + 1 minimum
    assert e.value.status == 1
    # a corrupt gzip stream reports the read failure
    bad = tmp_path / "bad.txt.gz"
    good = S.write_case(b"1 2\n" * 100000, str(tmp_path), "good", gz=True)
    raw = open(good, "rb").read()
    bad.write_bytes(raw[: len(raw) // 2] + bytes(64) + raw[len(raw) // 2 + 64:])
    with pytest.raises(gb.GraphError) as e:
        gb.from_snap_gpu(str(bad), True)
    assert e.value.status == 6 and "gzread failed" in str(e.value)


def test_gconvert_cli(gb, oracle, tmp_path):
    """bin/gconvert: the reference's command line, output lines and CSV upsert."""
    import subprocess
    exe = os.path.join(os.path.dirname(gb.__file__), "bin", "gconvert")
    path = S.write_case(S.QUIRKS, str(tmp_path), "toy", gz=True)
    out, csv = str(tmp_path / "toy.bin"), str(tmp_path / "stats.csv")
    for _ in range(2):  # the second run replaces the CSV row
        p = subprocess.run([exe, path, out, "--undirected", "--csv", csv], capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
    assert "lines 9, raw max id 729, n 6" in p.stdout
    want, _ = oracle.convert_snap(path, False)
    assert gb.load(out).equal(want)
    rows = open(csv).read().splitlines()
    assert rows[0] == "dataset,directed,lines,n,m_before,m,seconds,peak_rss_mb"
    assert len(rows) == 2 and rows[1].startswith("toy,0,9,6,18,14,")
    bad = S.write_case(b"1 2\n3\n", str(tmp_path), "bad")
    p = subprocess.run([exe, bad, out, "--directed", "--csv", ""], capture_output=True, text=True, timeout=300)
    assert p.returncode == 1 and f"gconvert: {bad}: malformed line 2" in p.stderr
