"""The product's host graph layer (src/graph equivalents, built in parallel):
byte-identical to the reference's graphs (golden fixtures), transforms agree
with the oracle, .bin I/O round-trips and rejects bad files.  CPU only."""
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import ROOT, sha

SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]


def rec(g):
    return {"n": g.n, "m": g.m, "flags": g.flags, "row_ptr": sha(g.row_ptr), "col_idx": sha(g.col_idx)}


@pytest.fixture(scope="module")
def psuite(gb):
    return dict(gb.gen.suite())


def test_suite_generators_match_reference(psuite, golden, gb):
    for name in SUITE:
        g = psuite[name]
        assert gb.validate(g) == "", name
        assert rec(g) == golden["graphs"][name]["stored"], name
        assert rec(gb.symmetrize(g)) == golden["graphs"][name]["sym"], name
        assert rec(gb.transpose(g)) == golden["graphs"][name]["transpose"], name


def test_config_generators_match_reference(golden, gb):
    assert rec(gb.gen.star(100000)) == golden["graphs"]["star100000"]["stored"]
    assert rec(gb.gen.grid2d(1400, 1400)) == golden["graphs"]["grid1400x1400"]["stored"]
    assert rec(gb.gen.rmat(16, 16, False, 1)) == golden["graphs"]["rmat16_ef16_s1"]["stored"]


def test_rmat22_config_graph_matches_reference(golden, gb):
    """The R-MAT scale-22 benchmark graph (8.5 * 2^22 draws, seed 22, ids
    permuted by reorder "random" seed 1) equals the reference-built one."""
    want = golden["graphs"]["rmat22_c2"]
    g = gb.gen.rmat(22, edges=want["edges_drawn"], directed=False, seed=want["gen_seed"])
    perm = gb.random_perm(g.n, want["perm_seed"])
    assert sha(perm) == want["perm"]
    assert rec(gb.permute(g, perm)) == want["stored"]


def test_transforms_match_oracle(gb, oracle):
    rng = np.random.default_rng(11)
    for trial in range(8):
        n = int(rng.integers(1, 3000))
        k = int(rng.integers(0, 6 * n))
        eu = rng.integers(0, n, k).astype(np.uint32)
        ev = rng.integers(0, n, k).astype(np.uint32)
        directed = bool(trial % 2)
        g = gb.from_edges(n, eu, ev, directed)
        o = oracle.from_edges(n, eu, ev, directed)
        assert g.equal(o)
        assert gb.symmetrize(g).equal(oracle.symmetrize(o))
        assert gb.transpose(g).equal(oracle.transpose(o))
        p = gb.random_perm(n, trial + 1)
        assert np.array_equal(p, oracle.random_perm(n, trial + 1))
        assert gb.permute(g, p).equal(oracle.permute(o, p))


def test_pick_sources_matches_oracle(gb, oracle):
    for g0 in (gb.gen.rmat(12, 16, False, 42), gb.gen.two_components(), gb.gen.star(1000), gb.gen.path(10)):
        g = gb.symmetrize(g0)
        for count, seed in ((64, 1), (5, 7), (1000, 2)):
            a = gb.pick_sources(g, count, seed)
            b = oracle.pick_sources(g, count, seed)
            assert np.array_equal(a, b)
        assert np.array_equal(gb.pick_sources(g, 10, 3, True), oracle.pick_sources(g, 10, 3, True))


def test_bin_roundtrip_and_rejects(gb):
    with tempfile.TemporaryDirectory() as d:
        for name, g in gb.gen.suite():
            p = os.path.join(d, name + ".bin")
            gb.save(g, p)
            h = gb.load(p)
            assert g.equal(h) and gb.validate(h) == ""
        bad = os.path.join(d, "bad.bin")
        with open(bad, "wb") as f:
            f.write(b"definitely not a graph file, but longer than a header")
        with pytest.raises(gb.GraphError):
            gb.load(bad)
        with pytest.raises(gb.GraphError):
            gb.load(os.path.join(d, "missing.bin"))
        # a file whose size disagrees with its header, and a path that cannot be written
        g = gb.gen.grid2d(10, 10)
        p = os.path.join(d, "short.bin")
        gb.save(g, p)
        with open(p, "r+b") as f:
            f.truncate(os.path.getsize(p) - 4)
        with pytest.raises(gb.GraphError) as e:
            gb.load(p)
        assert e.value.status == 6 and "size does not match header" in str(e.value)
        with pytest.raises(gb.GraphError) as e:
            gb.save(g, os.path.join(d, "no_such_dir", "x.bin"))
        assert e.value.status == 6
        # a multi-slice graph (arrays larger than one 8 MiB read/write slice)
        big = gb.gen.rmat(18, 16, False, 4)
        p = os.path.join(d, "big.bin")
        gb.save(big, p)
        assert gb.load(p).equal(big)


def test_benchmark_generators_shapes(gb):
    # road: degree <= 8, roughly 4% of grid edges gone, symmetric and valid
    g = gb.gen.road(200, 200, 0.04, 0.005, 1400)
    deg = g.degrees()
    assert gb.validate(g) == "" and deg.max() <= 8
    full = 2 * (2 * 200 * 199)
    assert 0.94 * full < g.m < 0.98 * full + 4 * 200
    # web: directed, ~15% dangling, mean out-degree near 5.8
    w = gb.gen.web(50000, 5.8, 2.1, 875)
    od = w.degrees()
    assert w.directed and gb.validate(w) == ""
    assert 0.12 < (od == 0).mean() < 0.18
    assert 5.0 < od.mean() < 6.0
    # chung-lu: undirected, heavy tail, mean degree near the target
    c = gb.gen.chung_lu(20000, 2.2, 20.0, 307)
    cd = c.degrees()
    assert not c.directed and gb.validate(c) == ""
    assert 15 < cd.mean() < 21 and cd.max() > 10 * cd.mean()


def test_library_exports_every_declared_symbol(gb):
    """Every function declared in include/graph_b200.h is exported (no GPU calls)."""
    hdr = open(os.path.join(ROOT, "include", "graph_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(gb_[a-z0-9_]+)\s*\(", hdr))
    assert len(names) > 40
    L = gb.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_errors_are_reported_not_raised_across_abi(gb):
    with pytest.raises(gb.GraphError) as e:
        gb.permute(gb.gen.path(4), np.array([0, 0, 1, 2], np.uint32))
    assert "permutation" in str(e.value)
    with pytest.raises(gb.GraphError):
        gb.from_edges(3, [0, 5], [1, 1])
