"""The oracle pinned: its results must equal the golden fixtures written from
the reference's own CPU code (tests/golden/make_golden.py), the reference's
known-answer tests, and -- where the reference build is present -- that build.
CPU only."""
import hashlib
import json

import numpy as np
import pytest

from conftest import ref_test_sources, sha

SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]
DO_MODES = {"default": (15.0, 18.0), "all_td": (1e-12, 18.0), "all_bu": (1e12, 1e12), "flip_flop": (2.0, 4.0)}


def trace_record(tr):
    return {"levels": len(tr), "dirs": "".join(t[1] for t in tr),
            "frontier": sha(np.array([t[2] for t in tr], dtype=np.uint64)),
            "edges": sha(np.array([t[3] for t in tr], dtype=np.uint64))}


def rec(g):
    return {"n": g.n, "m": g.m, "flags": g.flags, "row_ptr": sha(g.row_ptr), "col_idx": sha(g.col_idx)}


@pytest.fixture(scope="module")
def suite(oracle):
    return dict(oracle.suite())


def test_suite_graphs_match_reference(suite, golden, oracle):
    for name in SUITE:
        g = suite[name]
        assert oracle.validate(g) == 0, name
        assert rec(g) == golden["graphs"][name]["stored"], name
        assert rec(oracle.symmetrize(g)) == golden["graphs"][name]["sym"], name
        assert rec(oracle.transpose(g)) == golden["graphs"][name]["transpose"], name


def test_larger_generators_match_reference(golden, oracle):
    assert rec(oracle.gen("star", 100000)) == golden["graphs"]["star100000"]["stored"]
    assert rec(oracle.gen("grid2d", 1400, 1400)) == golden["graphs"]["grid1400x1400"]["stored"]
    assert rec(oracle.gen("rmat", 16, 16, 0, 1)) == golden["graphs"]["rmat16_ef16_s1"]["stored"]


def test_bfs_serial_and_do_match_reference(suite, golden, oracle):
    for name in SUITE:
        s = oracle.symmetrize(suite[name])
        recs = golden["bfs"][name]
        srcs = ref_test_sources(s.n) + [int(np.argmax(s.degrees()))]
        assert [r["source"] for r in recs] == srcs
        for r in recs:
            d = oracle.bfs_serial(s, r["source"])
            assert sha(d) == r["dist"], (name, r["source"])
            assert int((d != oracle.UNREACHED).sum()) == r["reached"]
            assert oracle.component_edges(s, d) == r["comp_edges"]
            for mode, (a, b) in DO_MODES.items():
                dd, tr = oracle.bfs_do(s, r["source"], a, b)
                assert np.array_equal(dd, d)
                assert trace_record(tr) == r["do"][mode], (name, r["source"], mode)


def test_bfs_known_answers(oracle):
    """tests/test_main.cpp:268-279."""
    d = oracle.bfs_serial(oracle.gen("path", 1000), 0)
    assert np.array_equal(d, np.arange(1000, dtype=np.uint32))
    d = oracle.bfs_serial(oracle.gen("star", 100000), 7)
    assert d[7] == 0 and d[0] == 1 and d[8] == 2
    d = oracle.bfs_serial(oracle.gen("two_components"), 0)
    assert d[299] == 299 and d[300] == oracle.UNREACHED and d[399] == oracle.UNREACHED
    d = oracle.bfs_serial(oracle.gen("grid2d", 100, 100), 0)
    assert d[99 * 100 + 99] == 198
    d = oracle.bfs_serial(oracle.gen("empty", 1000), 3)
    assert d[3] == 0 and d[4] == oracle.UNREACHED


def test_pagerank_matches_reference(suite, golden, golden_ranks, oracle):
    for name in SUITE:
        g = suite[name]
        gin = oracle.transpose(g) if g.directed else g
        od = g.degrees()
        for key, iters, tol in (("fixed20", 20, 0.0), ("tol1e-6", 1000, 1e-6), ("conv1e-10", 1000, 1e-10)):
            r, it, last = oracle.pagerank_serial(gin, od, iters, tol)
            want = golden["pagerank"][name][key]
            assert it == want["iters"], (name, key)
            assert np.array_equal(r, golden_ranks[f"{name}/{key}"]), (name, key)
            assert last == want["last_delta"]


def test_pagerank_known_answers(oracle):
    """tests/test_main.cpp:630-652: hand-checked fixed points."""
    def solve(g):
        gin = oracle.transpose(g)
        r, _, _ = oracle.pagerank_serial(gin, g.degrees(), 1000, 1e-14)
        return r
    r = solve(oracle.from_edges(2, [0], [1], True))
    assert abs(r[0] - 0.5 / 1.425) < 1e-12 and abs(r[1] - (1 - 0.5 / 1.425)) < 1e-12
    r = solve(oracle.from_edges(3, [0, 1, 2], [1, 2, 0], True))
    assert np.all(np.abs(r - 1 / 3) < 1e-12)
    r = solve(oracle.gen("complete", 200))
    assert np.all(np.abs(r - 1 / 200) < 1e-12)
    r = solve(oracle.gen("empty", 1000))
    assert np.all(np.abs(r - 1 / 1000) < 1e-12)


def test_check_ranks_and_gs_rule(oracle):
    ref = np.array([0.5, 0.3, 0.2])
    c = oracle.check_ranks(ref, ref.astype(np.float32))
    assert c.ok() and c.l1 < 1e-7
    bad = oracle.check_ranks(ref, np.array([0.6, 0.2, 0.2], np.float32))
    assert not bad.ok()
    j = oracle.PrCheck(2e-4, 5e-4, 1.0)
    assert oracle.gs_no_worse(oracle.PrCheck(1.5e-4, 9e-4, 1.0001), j)
    assert not oracle.gs_no_worse(oracle.PrCheck(3e-4, 1e-4, 1.0), j)


def test_mlp_reference_gradient_is_consistent(oracle):
    """Finite differences of the oracle's own loss agree with its gradient."""
    rng = np.random.default_rng(0)
    nf, nh, no = 8, 32, 5
    npar = nh * nf + nh + nh * nh + nh + no * nh + no
    p = rng.normal(0, 0.3, npar).astype(np.float32)
    x = rng.random((16, nf), dtype=np.float32)
    y = rng.random((16, no), dtype=np.float32)
    mask = (rng.random((16, no)) > 0.2).astype(np.float32)
    loss, g = oracle.mlp_loss_grad(nf, nh, no, p, x, y, mask)
    for i in rng.choice(npar, 20, replace=False):
        e = 1e-2
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (oracle.mlp_loss_grad(nf, nh, no, pp, x, y, mask)[0] - oracle.mlp_loss_grad(nf, nh, no, pm, x, y, mask)[0]) / (2 * e)
        assert abs(fd - g[i]) < 2e-3 + 0.05 * abs(fd), (i, fd, g[i])


def test_pick_sources_restatement(oracle):
    """pickSources (src/bench/main.cpp:155-169): distinct, degree > 0, inside the
    largest component, deterministic for a seed."""
    g = oracle.symmetrize(oracle.gen("rmat", 12, 16, 0, 42))
    s1 = oracle.pick_sources(g, 64, 1)
    s2 = oracle.pick_sources(g, 64, 1)
    assert np.array_equal(s1, s2) and len(set(s1.tolist())) == 64
    d = oracle.bfs_serial(g, int(s1[0]))
    assert all(d[v] != oracle.UNREACHED and g.degrees()[v] > 0 for v in s1)
    two = oracle.gen("two_components")
    s = oracle.pick_sources(two, 1000, 1)
    assert len(s) == 299 + 1 and max(s) < 300  # the 300-vertex path is the largest component


@pytest.mark.skipif("not __import__('oracle_py').ref_available()")
def test_oracle_equals_reference_build_on_random_graphs(oracle):
    """Beyond the fixtures: random directed/undirected graphs, both builds."""
    ref = oracle.RefGraph
    rng = np.random.default_rng(5)
    for trial in range(6):
        n = int(rng.integers(1, 400))
        k = int(rng.integers(0, 3 * n))
        eu = rng.integers(0, n, k).astype(np.uint32)
        ev = rng.integers(0, n, k).astype(np.uint32)
        directed = bool(trial % 2)
        g = oracle.from_edges(n, eu, ev, directed)
        r = ref(oracle.ref().gref_from_edges(n, eu if k else np.zeros(1, np.uint32),
                                             ev if k else np.zeros(1, np.uint32), k, int(directed)))
        assert g.equal(r.host())
        s = oracle.symmetrize(g)
        rs = r.symmetrize()
        assert s.equal(rs.host())
        for src in {0, n // 2, n - 1}:
            assert np.array_equal(oracle.bfs_serial(s, src), rs.bfs_serial(src))
            d1, t1 = oracle.bfs_do(s, src, 2.0, 3.0)
            d2, t2 = rs.bfs_do(src, 2.0, 3.0, threads=1)
            assert t1 == t2
        gin = oracle.transpose(g)
        r1, i1, _ = oracle.pagerank_serial(gin, g.degrees(), 30)
        r2, i2, _ = r.transpose().pagerank(g.degrees(), 30)
        assert i1 == i2 and np.array_equal(r1, r2)
