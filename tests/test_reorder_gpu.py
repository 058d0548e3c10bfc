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
