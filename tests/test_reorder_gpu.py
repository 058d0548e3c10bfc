"""Vertex orderings on the GPU (gb_reorder_gpu "degree" / "rcm") against the
reference's own permutations (tests/golden/order_golden.json, from the
reference build) and against the oracle on graphs with thousands of BFS
levels (road grids), many components, isolated vertices and hubs.  Integer
work: permutations must be identical."""
import hashlib

import numpy as np
import pytest

from order_graphs import order_graphs

pytestmark = pytest.mark.gpu


def _sha(p):
    return hashlib.sha256(np.ascontiguousarray(p, np.uint32).tobytes()).hexdigest()


def _as_lib(gb, h):
    return gb.Graph(h.n, h.m, h.flags, h.row_ptr, h.col_idx)


def _as_oracle(oracle, g):
    return oracle.HostGraph(g.n, g.m, g.flags, g.row_ptr, g.col_idx)


def test_gpu_orderings_match_reference(gb, order_golden):
    for name, h in order_graphs():
        g = _as_lib(gb, h)
        for ordering in ("degree", "rcm"):
            assert _sha(gb.reorder_gpu(g, ordering)) == order_golden[name]["orderings"][ordering]["perm"], \
                (name, ordering)


@pytest.mark.parametrize("case", ["road600", "road_sparse", "chunglu", "forest", "rmat20"])
def test_gpu_orderings_match_oracle(gb, oracle, case):
    if case == "road600":  # ~1200 BFS levels per pass
        g = gb.gen.road(600, 600, 0.04, 0.005, 11)
    elif case == "road_sparse":  # many components from dropped edges
        g = gb.gen.road(300, 300, 0.45, 0.0, 12)
    elif case == "chunglu":
        g = gb.gen.chung_lu(200000, 2.2, 12.0, 13)
    elif case == "forest":  # stars, paths and isolated vertices side by side
        rng = np.random.default_rng(14)
        n = 50000
        u = rng.integers(0, n // 4, 30000).astype(np.uint32)
        v = rng.integers(0, n, 30000).astype(np.uint32)
        g = gb.from_edges(n, u, v, False)
    else:
        g = gb.gen.rmat(20, 8, False, 15)
    h = _as_oracle(oracle, g)
    for ordering in ("degree", "rcm"):
        assert np.array_equal(gb.reorder_gpu(g, ordering), oracle.reorder(h, ordering)), (case, ordering)


def test_gpu_orderings_errors(gb):
    with pytest.raises(gb.GraphError):
        gb.reorder_gpu(gb.gen.rmat(8, 8, True, 3), "rcm")
    with pytest.raises(gb.GraphError):
        gb.reorder_gpu(gb.gen.path(10), "sideways")
    g = gb.gen.path(10)
    assert np.array_equal(gb.reorder_gpu(g, "random", 4), gb.random_perm(10, 4))
    assert np.array_equal(gb.reorder_gpu(g, "original"), np.arange(10, dtype=np.uint32))


def _hub_first_numpy(g):
    deg = np.diff(g.row_ptr.astype(np.int64))
    rows = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    col = g.col_idx.astype(np.int64)
    return g.col_idx[np.lexsort((col, -deg[col], rows))]


@pytest.mark.parametrize("case", ["rmat16", "chunglu", "star", "road"])
def test_hub_first_layout_and_bfs(gb, oracle, case):
    """gb_csr_hub_first_gpu equals a numpy lexsort; a BFS handle with the
    hub-first layout returns the oracle's depths, and with the alpha/beta rule
    the oracle's per-level directions, frontier sizes and top-down edges."""
    g = {"rmat16": lambda: gb.gen.rmat(16, 16, False, 5), "chunglu": lambda: gb.gen.chung_lu(100000, 2.2, 20.0, 6),
         "star": lambda: gb.gen.star(5000), "road": lambda: gb.gen.road(120, 120, 0.04, 0.005, 7)}[case]()
    h = gb.hub_first_gpu(g)
    assert np.array_equal(h.row_ptr, g.row_ptr) and np.array_equal(h.col_idx, _hub_first_numpy(g))
    og = _as_oracle(oracle, g)
    bfs = gb.GpuBfs(g).hub_first()
    srcs = gb.pick_sources(g, 8, 3)
    rule = gb.BfsOptions(selector="rule")
    for s in srcs:
        want = oracle.bfs_serial(og, int(s))
        for variant in ("gpu_do", "gpu_do_persistent"):
            assert np.array_equal(bfs.run(variant, int(s), opts=rule), want), (case, variant, s)
        d, tr = bfs.run("gpu_do_persistent", int(s), opts=rule, trace=True)
        _, otr = oracle.bfs_do(og, int(s))
        assert [(t["direction"], t["frontier"]) for t in tr] == [(o[1], o[2]) for o in otr]
        assert [t["edges"] for t in tr if t["direction"] == "T"] == [o[3] for o in otr if o[1] == "T"]
    batch = bfs.run_batch(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(batch[i], oracle.bfs_serial(og, int(s)))
