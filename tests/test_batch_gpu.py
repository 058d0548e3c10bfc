"""64-source batched BFS (one launch, per-vertex 64-bit masks) against the
oracle: every source's depths must equal cpu_serial's, whatever strategy runs
each level and whatever the batch size, including repeated sources."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def check_batch(gb, oracle, g, bfs, srcs, opts):
    d = bfs.run_batch(srcs, opts=opts)
    for i, s in enumerate(srcs):
        ref = oracle.bfs_serial(g, int(s))
        assert np.array_equal(d[i], ref), (i, int(s))
    return d


def test_batch_suite_all_strategies(gb, oracle):
    for name, g0 in gb.gen.suite():
        g = gb.symmetrize(g0)
        bfs = gb.GpuBfs(g)
        rng = np.random.default_rng(len(name))
        srcs = rng.integers(0, g.n, 64).astype(np.uint32)
        refs = [oracle.bfs_serial(g, int(s)) for s in srcs]
        for opts in [gb.BfsOptions()] + [gb.BfsOptions(force_strategy=s) for s in range(5)] + \
                    [gb.BfsOptions(alpha=2.0, beta=2.0), gb.BfsOptions(hub_min=32, block=256)]:
            d, tr = bfs.run_batch(srcs, opts=opts, trace=True)
            for i in range(len(srcs)):
                assert np.array_equal(d[i], refs[i]), (name, i, opts.force_strategy)


def test_batch_sizes_and_duplicates(gb, oracle):
    g = gb.gen.rmat(14, 16, False, 5)
    bfs = gb.GpuBfs(g)
    for srcs in ([3], [3, 3, 3], list(range(7)), [0] * 64, list(gb.pick_sources(g, 64, 2))):
        check_batch(gb, oracle, g, bfs, np.array(srcs, np.uint32), gb.BfsOptions())
    with pytest.raises(gb.GraphError):
        bfs.run_batch(np.arange(65, dtype=np.uint32))
    with pytest.raises(gb.GraphError):
        bfs.run_batch(np.array([g.n], np.uint32))


def test_batch_larger_graphs(gb, oracle):
    graphs = [gb.gen.road(200, 200, 0.04, 0.005, 1), gb.gen.chung_lu(100000, 2.2, 30.0, 2),
              gb.permute(gb.gen.rmat(17, 16, False, 3), gb.random_perm(1 << 17, 4))]
    for g in graphs:
        bfs = gb.GpuBfs(g)
        srcs = gb.pick_sources(g, 64, 9)
        for opts in (gb.BfsOptions(), gb.BfsOptions(force_strategy="bu"), gb.BfsOptions(force_strategy="td_ept2"),
                     gb.BfsOptions(hub_min=64)):
            check_batch(gb, oracle, g, bfs, srcs, opts)


def test_batch_small_heavy_queue_split_exact(gb, oracle):
    """Few edge-balanced tiles with many edges each (hub list off) are pushed
    in edge-range parts over the grid: every edge-balanced strategy, on the
    full grid and on small ones, must give the oracle's depths for every
    source of the batch."""
    g = gb.gen.rmat(16, 16, False, 1)
    bfs = gb.GpuBfs(g)
    for k, seed in ((64, 9), (5, 3)):
        srcs = gb.pick_sources(g, k, seed)
        for strat in ("td_ept1", "td_ept2", "td_ept4"):
            for grid in (0, 148, 16):
                opts = gb.BfsOptions(force_strategy=strat, hub_min=1 << 30, grid_blocks=grid)
                check_batch(gb, oracle, g, bfs, srcs, opts)


def test_batch_learned_selector_exact(gb, oracle):
    g = gb.gen.rmat(15, 16, False, 8)
    bfs = gb.GpuBfs(g)
    srcs = gb.pick_sources(g, 64, 3)
    rng = np.random.default_rng(5)
    for _ in range(3):
        bfs.set_selector(rng.normal(0, 1, gb.selector_param_count()).astype(np.float32), 1)
        check_batch(gb, oracle, g, bfs, srcs, gb.BfsOptions(selector="learned"))


def test_batch_bottom_up_long_lists_exact(gb, oracle):
    """Bottom-up levels hand what is left of a long list to the whole warp
    (64 or more entries left after the thread's own first 64) or to the whole
    block (256 or more).  Hubs of 100 to 6,000 neighbours in one component and
    half of the sources in another component keep every hub's missing sources
    missing, so its scan runs to the end of its list; lists that finish early
    and short rests finishing serially are in the same warps.  Every source's
    depths must equal the oracle's, forced bottom-up and under the rule, on
    both adjacency orders."""
    rng = np.random.default_rng(11)
    n1 = 20000
    eu, ev = [], []
    for hub, deg in ((0, 6000), (1, 3000), (2, 700), (3, 513), (4, 200), (5, 100), (6, 65)):
        nb = rng.choice(np.arange(7, n1), deg, replace=False)
        eu.append(np.full(deg, hub)); ev.append(nb)
    # a sparse random graph on the rest of component A, and a path joining the hubs
    eu.append(rng.integers(7, n1, 3 * n1)); ev.append(rng.integers(7, n1, 3 * n1))
    eu.append(np.arange(0, 6)); ev.append(np.arange(1, 7))
    # component B: a grid-like ladder, no edge to A
    b0 = n1
    nb2 = 5000
    eu.append(np.arange(b0, b0 + nb2 - 1)); ev.append(np.arange(b0 + 1, b0 + nb2))
    eu.append(np.arange(b0, b0 + nb2 - 50)); ev.append(np.arange(b0 + 50, b0 + nb2))
    u = np.concatenate(eu).astype(np.uint32)
    v = np.concatenate(ev).astype(np.uint32)
    keep = u != v
    g = gb.from_edges(n1 + nb2, u[keep], v[keep], False)
    srcs = np.concatenate([rng.integers(7, n1, 32), rng.integers(b0, b0 + nb2, 32)]).astype(np.uint32)
    refs = [oracle.bfs_serial(g, int(s)) for s in srcs]
    for hub_first in (False, True):
        bfs = gb.GpuBfs(g)
        if hub_first:
            bfs.hub_first()
        for opts in (gb.BfsOptions(force_strategy="bu"), gb.BfsOptions(), gb.BfsOptions(block=512),
                     gb.BfsOptions(force_strategy="bu", grid_blocks=8)):
            d = bfs.run_batch(srcs, opts=opts)
            for i in range(len(srcs)):
                assert np.array_equal(d[i], refs[i]), (hub_first, i, opts.force_strategy, opts.grid_blocks)
