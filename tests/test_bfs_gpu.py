"""GPU BFS parity through the C ABI against the oracle (the structure of the
reference's tests/test_main.cpp:467-623): every variant and parameter extreme
on every suite graph and source must give cpu_serial's depths bit for bit;
the trace must account for every reached vertex once; direction-optimizing
forms must take cpu_do's direction / frontier sequence level by level."""
import numpy as np
import pytest

from conftest import ref_test_sources

pytestmark = pytest.mark.gpu

SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]


@pytest.fixture(scope="module")
def cases(gb, oracle):
    out = []
    for name, g0 in gb.gen.suite():
        g = gb.symmetrize(g0)
        srcs = ref_test_sources(g.n) + [int(np.argmax(g.degrees()))]
        refs = {s: oracle.bfs_serial(g, s) for s in srcs}
        out.append((name, g, gb.GpuBfs(g), refs))
    return out


def reached(d):
    return int((d != 0xFFFFFFFF).sum())


CFGS = [
    ("gpu_vertex", {}), ("gpu_naive", {}),
    ("gpu_binned", dict(small_max=32, large_min=1024)), ("gpu_binned", dict(small_max=1 << 30, large_min=1 << 31)),
    ("gpu_binned", dict(small_max=0, large_min=0)), ("gpu_binned", dict(small_max=1, large_min=1 << 30)),
    ("gpu_binned", dict(small_max=2, large_min=3)),
    ("gpu_edge", dict(ept=1)), ("gpu_edge", dict(ept=4)), ("gpu_edge", dict(ept=16)),
]


@pytest.mark.parametrize("tg", [32, 256, 1024])
def test_level_variants_match_serial(cases, gb, tg):
    for name, g, bfs, refs in cases:
        deg = g.degrees().astype(np.uint64)
        for src, ref in refs.items():
            want_edges = int(deg[ref != 0xFFFFFFFF].sum())
            for variant, kw in CFGS:
                o = gb.BfsOptions(tg=tg, **kw)
                d, tr = bfs.run(variant, src, opts=o, trace=True)
                assert np.array_equal(d, ref), (name, src, variant, kw, tg)
                assert sum(L["frontier"] for L in tr) == reached(ref), (name, src, variant)
                assert sum(L["edges"] for L in tr) == want_edges, (name, src, variant)


MODES = [("default", 15.0, 18.0), ("force-bu", 1e9, 1e9), ("never-bu", 1e-9, 18.0), ("flip-flop", 2.0, 2.0)]


@pytest.mark.parametrize("variant", ["gpu_do", "gpu_do_persistent"])
def test_direction_optimizing_matches_cpu_do(cases, gb, oracle, variant):
    for name, g, bfs, refs in cases:
        for src, ref in refs.items():
            for mode, a, b in MODES:
                for tg in (32, 256):
                    o = gb.BfsOptions(tg=tg, alpha=a, beta=b, block=256 if tg == 32 else 512)
                    d, tr = bfs.run(variant, src, opts=o, trace=True)
                    assert np.array_equal(d, ref), (name, src, variant, mode)
                    _, ctr = oracle.bfs_do(g, src, a, b)
                    assert [L["direction"] for L in tr] == [t[1] for t in ctr], (name, src, variant, mode)
                    assert [L["frontier"] for L in tr] == [t[2] for t in ctr], (name, src, variant, mode)
                    if a > 1e6 and reached(ref) > 1:
                        assert any(L["direction"] == "B" for L in tr)
                    if a < 1e-6:
                        assert all(L["direction"] == "T" for L in tr)


@pytest.mark.parametrize("strategy", ["td_ept1", "td_ept2", "td_ept4", "td_warp", "bu"])
def test_persistent_forced_strategies_exact(cases, gb, strategy):
    for name, g, bfs, refs in cases:
        for src, ref in refs.items():
            for hub_min in (32, 4096):
                o = gb.BfsOptions(force_strategy=strategy, hub_min=hub_min)
                d, tr = bfs.run("gpu_do_persistent", src, opts=o, trace=True)
                assert np.array_equal(d, ref), (name, src, strategy, hub_min)
                assert sum(L["frontier"] for L in tr) == reached(ref)


def test_persistent_strategy_mixes_exact(gb, oracle):
    """Random per-level strategy switches are exercised by alternating forced
    runs over larger graphs (hubs split across blocks, BU<->TD conversions)."""
    graphs = [gb.gen.rmat(16, 16, False, 1), gb.gen.road(300, 300, 0.04, 0.005, 3), gb.gen.star(300000),
              gb.symmetrize(gb.gen.web(100000, 5.8, 2.1, 9))]
    for g in graphs:
        bfs = gb.GpuBfs(g)
        srcs = gb.pick_sources(g, 3, 5)
        for s in srcs:
            ref = oracle.bfs_serial(g, int(s))
            for mode, a, b in MODES:
                for hub_min in (64, 4096):
                    d = bfs.run("gpu_do_persistent", int(s), opts=gb.BfsOptions(alpha=a, beta=b, hub_min=hub_min))
                    assert np.array_equal(d, ref)
            d = bfs.run("gpu_do", int(s))
            assert np.array_equal(d, ref)


def test_persistent_small_heavy_queue_split_exact(gb, oracle):
    """A queue of fewer tiles than half the blocks, with many edges per tile,
    is expanded in edge-range parts spread over the grid.  With the hub list
    off (hub_min beyond every degree) every frontier goes through the tiles:
    each edge-balanced strategy and the rule, on the full grid and on one
    block per SM, must give the oracle's depths."""
    g = gb.gen.rmat(16, 16, False, 1)
    bfs = gb.GpuBfs(g)
    for s in gb.pick_sources(g, 4, 7):
        ref = oracle.bfs_serial(g, int(s))
        for strat in ("td_ept1", "td_ept2", "td_ept4", None):
            for grid in (0, 148):
                kw = dict(hub_min=1 << 30, grid_blocks=grid)
                if strat:
                    kw["force_strategy"] = strat
                d, tr = bfs.run("gpu_do_persistent", int(s), opts=gb.BfsOptions(**kw), trace=True)
                assert np.array_equal(d, ref), (int(s), strat, grid)
                assert sum(L["frontier"] for L in tr) == reached(ref)


def test_hybrid_is_the_persistent_kernel(cases, gb, oracle):
    name, g, bfs, refs = cases[6]
    for src, ref in refs.items():
        d, tr = bfs.runHybrid(src, trace=True)
        assert np.array_equal(d, ref)
        assert all(L["device"] == "G" for L in tr)


def test_invalid_options_raise(cases, gb):
    _, g, bfs, refs = cases[0]
    src = next(iter(refs))
    for bad in (dict(tg=48), dict(tg=0), dict(tg=2048), dict(ept=0)):
        with pytest.raises(gb.GraphError) as e:
            bfs.run("gpu_edge", src, opts=gb.BfsOptions(**bad))
        assert e.value.status == 1
    with pytest.raises(gb.GraphError):
        bfs.run("gpu_edge", g.n + 5)
    with pytest.raises(gb.GraphError):
        bfs.run(17, src)


def test_barrier_timeout_returns_status_and_context_survives(cases, gb):
    assert gb.barrier_timeout_selftest(2000) == 4
    name, g, bfs, refs = cases[1]
    src, ref = next(iter(refs.items()))
    assert np.array_equal(bfs.run("gpu_do_persistent", src), ref)


PRIM_SIZES = [0, 1, 2, 31, 32, 33, 255, 256, 257, 1023, 1024, 1025, 2047, 2048, 2049, 4097, 100003,
              1048575, 1048576, 1048577, 3000017]


def test_primitives_scan_reduce(gb):
    rng = np.random.default_rng(3)
    for n in PRIM_SIZES:
        v = rng.integers(0, 1000, n).astype(np.uint32)
        out, tot = gb.prim_scan(v)
        want = np.concatenate([[0], np.cumsum(v, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else v
        assert np.array_equal(out, want), n
        assert tot == int(v.sum(dtype=np.uint64)) & 0xFFFFFFFF
        w = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        s, m = gb.prim_reduce(w)
        assert s == int(w.sum(dtype=np.uint64)) & 0xFFFFFFFF
        assert m == (int(w.max()) if n else 0)


def test_primitives_queue_bitmap_roundtrip(gb):
    rng = np.random.default_rng(4)
    for n in (0, 1, 31, 32, 33, 1000, 100003):
        q = np.flatnonzero(rng.integers(0, 3, n) == 0).astype(np.uint32)
        rng.shuffle(q)
        bm, q2 = gb.prim_queue_bitmap(q, n)
        bits = np.zeros(n, bool)
        bits[q] = True
        got = ((bm[np.arange(n) >> 5] >> (np.arange(n) & 31)) & 1).astype(bool) if n else bits
        assert np.array_equal(got, bits)
        if n % 32:
            assert (int(bm[-1]) >> (n % 32)) == 0
        assert np.array_equal(np.sort(q2), np.sort(q))


@pytest.mark.parametrize("case", ["u4", "u8", "u16"])
def test_packed_depth_transfer(gb, oracle, case):
    """Depths returned to host memory travel packed (4 bits, 1 or 2 bytes per
    vertex) when the level count allows; arrays of at least 2^18 vertices with
    unreached vertices, single and batched runs: every depth must equal the
    oracle's."""
    if case == "u4":  # a power-law graph plus a separate path: few levels, unreached vertices
        a = gb.gen.rmat(18, 8, False, 21)
        n = a.n + 20000
        rows = np.repeat(np.arange(a.n, dtype=np.uint32), np.diff(a.row_ptr.astype(np.int64)))
        keep = rows < a.col_idx
        eu = np.concatenate([rows[keep], np.arange(a.n, n - 1, dtype=np.uint32)])
        ev = np.concatenate([a.col_idx[keep], np.arange(a.n + 1, n, dtype=np.uint32)])
        g = gb.from_edges(n, eu, ev, False)
    elif case == "u8":  # a sparse random graph: 20-30 levels
        g = gb.gen.chung_lu(300000, 2.8, 1.6, 24)
    else:  # a road grid: hundreds of levels
        g = gb.gen.road(560, 560, 0.04, 0.005, 22)
    og = oracle.HostGraph(g.n, g.m, g.flags, g.row_ptr, g.col_idx)
    bfs = gb.GpuBfs(g)
    srcs = gb.pick_sources(g, 4, 5)
    for s in srcs:
        want = oracle.bfs_serial(og, int(s))
        assert (want == 0xFFFFFFFF).any() or case == "u16"
        for variant in ("gpu_do_persistent", "gpu_do"):
            got = bfs.run(variant, int(s))
            assert np.array_equal(got, want), (case, variant, s)
        L = bfs.lastLevels()
        assert {"u4": L < 15, "u8": 15 <= L < 255, "u16": L >= 255}[case], (case, L)
    batch = bfs.run_batch(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(batch[i], oracle.bfs_serial(og, int(s)))
