"""Vertex orderings on the host: the oracle's restatement and the library's
host layer (gb_reorder, gb_locality) against the reference's own degree / RCM
permutations and locality metrics (src/graph/reorder.cpp:27-125), recorded in
tests/golden/order_golden.json.  Permutations are compared exactly (SHA-256);
the locality metrics exactly as well (the same integer sums, divided once)."""
import hashlib

import numpy as np

from order_graphs import order_graphs


def _sha(p):
    return hashlib.sha256(np.ascontiguousarray(p, np.uint32).tobytes()).hexdigest()


def _as_lib(gb, h):
    return gb.Graph(h.n, h.m, h.flags, h.row_ptr, h.col_idx)


def test_oracle_orderings_match_reference(oracle, order_golden):
    seen = set()
    for name, g in order_graphs():
        rec = order_golden[name]
        assert (g.n, g.m) == (rec["n"], rec["m"])
        for ordering in ("degree", "rcm"):
            perm = oracle.reorder(g, ordering)
            assert _sha(perm) == rec["orderings"][ordering]["perm"], (name, ordering)
        for ordering, want in rec["orderings"].items():
            h = oracle.permute(g, oracle.reorder(g, ordering)) if ordering != "original" else g
            assert oracle.locality(h) == (want["mean_gap"], want["same_block64"]), (name, ordering)
        seen.add(name)
    assert seen == set(order_golden)


def test_host_orderings_match_reference(gb, order_golden):
    for name, h in order_graphs():
        g = _as_lib(gb, h)
        rec = order_golden[name]
        for ordering in ("original", "degree", "rcm"):
            perm = gb.reorder(g, ordering)
            assert _sha(perm) == rec["orderings"][ordering]["perm"], (name, ordering)
            r = gb.permute(g, perm)
            assert gb.locality(r) == (rec["orderings"][ordering]["mean_gap"],
                                      rec["orderings"][ordering]["same_block64"])


def test_orderings_reject_bad_input(gb):
    import pytest
    g = gb.gen.rmat(8, 8, True, 3)  # directed: orderings need the symmetric graph
    with pytest.raises(gb.GraphError):
        gb.reorder(g, "rcm")
    with pytest.raises(gb.GraphError):
        gb.reorder(gb.gen.path(10), "sideways")
    assert np.array_equal(gb.reorder(g, "random", 5), gb.random_perm(g.n, 5))
