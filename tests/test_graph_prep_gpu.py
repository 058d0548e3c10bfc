"""Graph preparation on the GPU (gb_csr_*_gpu) against the host layer, whose
outputs are pinned byte for byte to the reference's own graph code by the
golden fixtures (tests/test_graph.py): fromEdgeList, transpose, symmetrize and
permute must return identical row_ptr, col_idx and flags, on the suite graphs,
random edge lists with duplicates and self-loops, and the 69M-entry R-MAT
scale-22 benchmark graph."""
import numpy as np
import pytest

from conftest import sha

pytestmark = pytest.mark.gpu


def same(a, b):
    return (a.n == b.n and a.m == b.m and a.flags == b.flags and np.array_equal(a.row_ptr, b.row_ptr)
            and np.array_equal(a.col_idx[: a.m], b.col_idx[: b.m]))


def test_suite_graph_ops_match_host(gb):
    for name, g in gb.gen.suite():
        assert same(gb.transpose_gpu(g), gb.transpose(g)), name
        assert same(gb.symmetrize_gpu(g), gb.symmetrize(g)), name
        perm = gb.random_perm(g.n, 5)
        assert same(gb.permute_gpu(g, perm), gb.permute(g, perm)), name


def test_from_edges_matches_host(gb):
    rng = np.random.default_rng(7)
    for n, k in ((1, 3), (2, 1), (1000, 5000), (70000, 400000), (1 << 20, 3 << 20)):
        eu = rng.integers(0, n, k, dtype=np.uint32)
        ev = rng.integers(0, n, k, dtype=np.uint32)
        ev[: k // 10] = eu[: k // 10]            # self-loops
        eu = np.concatenate([eu, eu[: k // 5]])  # repeated edges
        ev = np.concatenate([ev, ev[: k // 5]])
        for directed in (False, True):
            assert same(gb.from_edges_gpu(n, eu, ev, directed), gb.from_edges(n, eu, ev, directed)), (n, k, directed)
    assert same(gb.from_edges_gpu(10, [], [], False), gb.from_edges(10, [], [], False))


def test_directed_web_symmetrize_transpose(gb):
    g = gb.gen.web(200000, 5.8, 2.1, 11)
    assert same(gb.transpose_gpu(g), gb.transpose(g))
    assert same(gb.symmetrize_gpu(g), gb.symmetrize(g))


def test_benchmark_graph(gb, golden):
    """The C2 benchmark graph (R-MAT scale 22, 8.5 * 2^22 draws, seed 22) permuted
    on the GPU by the benchmark permutation equals the reference-built graph
    (pinned hashes); its transpose is itself (undirected)."""
    want = golden["graphs"]["rmat22_c2"]
    g0 = gb.gen.rmat(22, edges=want["edges_drawn"], directed=False, seed=want["gen_seed"])
    perm = gb.random_perm(g0.n, want["perm_seed"])
    g = gb.permute_gpu(g0, perm)
    st = want["stored"]
    assert (g.n, g.m, g.flags) == (st["n"], st["m"], st["flags"])
    assert sha(g.row_ptr[: g.n + 1]) == st["row_ptr"]
    assert sha(g.col_idx[: g.m]) == st["col_idx"]
    assert same(gb.transpose_gpu(g), g)


def test_pick_sources_gpu_matches_host(gb):
    """Sources from the largest component found on the GPU equal gb_pick_sources'
    (gbench's largestComponent + pickSources) on graphs with many components,
    equal-sized components, isolated vertices and long paths."""
    graphs = [g if not g.directed else gb.symmetrize(g) for _, g in gb.gen.suite()]
    graphs += [gb.gen.road(300, 300, 0.04, 0.005, 3), gb.gen.road(400, 400, 0.3, 0.0, 4),
               gb.from_edges(12, [0, 2, 4, 6], [1, 3, 5, 7]),          # equal components: the first wins
               gb.gen.path(200000), gb.gen.rmat(18, 4, False, 9)]
    for g in graphs:
        for count, seed in ((64, 1), (8, 7)):
            assert np.array_equal(gb.pick_sources_gpu(g, count, seed), gb.pick_sources(g, count, seed)), (g.n, g.m)
        assert np.array_equal(gb.pick_sources_gpu(g, 16, 3, True), gb.pick_sources(g, 16, 3, True))


def test_errors(gb):
    g = gb.gen.path(10)
    with pytest.raises(gb.GraphError):
        gb.permute_gpu(g, np.zeros(10, np.uint32))        # not a permutation
    with pytest.raises(gb.GraphError):
        gb.from_edges_gpu(5, [1, 7], [2, 3])              # endpoint >= n
    bad = gb.gen.path(10)
    bad.col_idx = bad.col_idx.copy()
    bad.col_idx[3] = 99                                   # column >= n
    with pytest.raises(gb.GraphError):
        gb.transpose_gpu(bad)
    assert same(gb.transpose_gpu(g), gb.transpose(g))     # the context is still usable
    with pytest.raises(gb.GraphError):
        gb.pick_sources_gpu(gb.gen.rmat(10, 8, True, 1))   # directed: not supported
