"""The oracle checked against an independent implementation, NetworkX, the way
the reference checks its own cpu_serial (tools/validate_networkx.py): BFS
distances on the symmetrized graph must match networkx's shortest path
lengths exactly for several sources per graph; PageRank of the stored
(directed) graph at d = 0.85, both sides run until the L1 change is below
1e-10, must agree at L1 < 1e-6 with relative error < 1e-4 on the 1000
highest-ranked vertices.  CPU only; skipped where NetworkX is absent."""
import numpy as np
import pytest

from conftest import ref_test_sources

nx = pytest.importorskip("networkx")

UNREACHED = 0xFFFFFFFF
SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]


def _graphs(oracle):
    g = dict(oracle.suite())
    g["rmat14_ef8"] = oracle.gen("rmat", 14, 8, 0, 5)
    g["rmat13_directed"] = oracle.gen("rmat", 13, 16, 1, 6)
    return g


def _nx(g, directed):
    G = nx.DiGraph() if directed else nx.Graph()
    G.add_nodes_from(range(g.n))
    rows = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.row_ptr.astype(np.int64)))
    G.add_edges_from(zip(rows.tolist(), g.col_idx[: g.m].tolist()))
    return G


@pytest.mark.parametrize("name", SUITE + ["rmat14_ef8", "rmat13_directed"])
def test_bfs_oracle_matches_networkx(oracle, name):
    s = oracle.symmetrize(_graphs(oracle)[name])
    G = _nx(s, directed=False)
    srcs = ref_test_sources(s.n) + [int(np.argmax(s.degrees()))]
    for src in srcs:
        want = np.full(s.n, UNREACHED, np.uint32)
        for v, d in nx.single_source_shortest_path_length(G, int(src)).items():
            want[v] = d
        assert np.array_equal(oracle.bfs_serial(s, int(src)), want), (name, src)


@pytest.mark.parametrize("name", SUITE + ["rmat14_ef8", "rmat13_directed"])
def test_pagerank_oracle_matches_networkx(oracle, name):
    g = _graphs(oracle)[name]
    r, it, last = oracle.pagerank_serial(oracle.transpose(g), oracle.out_degrees(g), iters=100000, tol=1e-10)
    assert last < 1e-10 or it == 100000
    G = _nx(g, directed=True)
    pr = nx.pagerank(G, alpha=0.85, tol=1e-10 / max(g.n, 1), max_iter=100000)
    want = np.array([pr[v] for v in range(g.n)])
    assert np.abs(r - want).sum() < 1e-6, name
    top = np.argsort(-want, kind="stable")[:1000]
    assert (np.abs(r[top] - want[top]) / want[top]).max() < 1e-4, name
    assert abs(r.sum() - 1.0) < 1e-9, name
