""".bin loading into GPU memory: gb_csr_load_pinned returns what gb_csr_load
returns (graph::load, src/graph/csr.cpp:54-84), and a BFS handle streamed
from a file (gb_bfs_create_from_file) gives the same depths as one built from
host arrays, on a graph whose adjacency spans several staging slices.
Malformed graphs (an id >= n, a decreasing row_ptr) are rejected by the
device check before any traversal reads them.  Integer work: exact."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_load_pinned_matches_load(gb, tmp_path):
    for name, g in (("rmat16", gb.gen.rmat(16, 16, False, 3)), ("web", gb.gen.web(50000, 5.8, 2.1, 4)),
                    ("empty", gb.gen.empty(10))):
        path = str(tmp_path / f"{name}.bin")
        gb.save(g, path)
        a, b = gb.load(path), gb.load_pinned(path)
        assert a.equal(g) and b.equal(g)


def test_bfs_from_file_matches_host_handle(gb, oracle, tmp_path):
    g = gb.gen.rmat(21, 16, False, 8)  # ~64M entries: several 64 MiB staging slices
    path = str(tmp_path / "rmat21.bin")
    gb.save(g, path)
    f = gb.GpuBfs.from_file(path)
    assert (f.n, f.m) == (g.n, g.m)
    h = gb.GpuBfs(g)
    for s in gb.pick_sources(g, 4, 2):
        for variant in ("gpu_do_persistent", "gpu_do"):
            assert np.array_equal(f.run(variant, int(s)), h.run(variant, int(s)))
    small = gb.gen.grid2d(50, 50)
    p2 = str(tmp_path / "grid.bin")
    gb.save(small, p2)
    og = oracle.HostGraph(small.n, small.m, small.flags, small.row_ptr, small.col_idx)
    assert np.array_equal(gb.GpuBfs.from_file(p2).run("gpu_do_persistent", 7), oracle.bfs_serial(og, 7))


def test_bfs_from_file_rejects(gb, tmp_path):
    d = gb.gen.rmat(10, 8, True, 5)  # directed
    path = str(tmp_path / "dir.bin")
    gb.save(d, path)
    with pytest.raises(gb.GraphError) as e:
        gb.GpuBfs.from_file(path)
    assert e.value.status == 1
    with pytest.raises(gb.GraphError) as e:
        gb.GpuBfs.from_file(str(tmp_path / "absent.bin"))
    assert e.value.status == 6
    # an adjacency id >= n in the file: the device check refuses the handle
    g = gb.gen.grid2d(20, 20)
    bad = str(tmp_path / "bad.bin")
    gb.save(g, bad)
    raw = bytearray(open(bad, "rb").read())
    off = 32 + 4 * (g.n + 1) + 4 * 17
    raw[off:off + 4] = np.uint32(g.n + 5).tobytes()
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(gb.GraphError) as e:
        gb.GpuBfs.from_file(bad)
    assert e.value.status == 1
    # the same check guards handles built from host arrays
    ci = g.col_idx.copy()
    ci[17] = g.n + 5
    with pytest.raises(gb.GraphError):
        gb.GpuBfs(gb.Graph(g.n, g.m, g.flags, g.row_ptr, ci))
    rp = g.row_ptr.copy()
    rp[5], rp[6] = rp[6], rp[5]  # decreasing row_ptr
    with pytest.raises(gb.GraphError):
        gb.GpuBfs(gb.Graph(g.n, g.m, g.flags, rp, g.col_idx))


def test_bfs_graph_view(gb, tmp_path):
    """GpuBfs::graph() (src/metal/bfs_gpu.hpp:39; the reference's test checks
    graph::equal(bfs.graph(), g), tests/test_main.cpp:510): the handle's graph
    comes back equal to the one it was built from, in hub-first order after
    hub_first(), and with the file's flags for a file handle."""
    g = gb.gen.rmat(14, 16, False, 6)
    b = gb.GpuBfs(g)
    v = b.graph()
    assert (v.n, v.m) == (g.n, g.m)
    assert np.array_equal(v.row_ptr, g.row_ptr) and np.array_equal(v.col_idx, g.col_idx)
    b.hub_first()
    h = gb.hub_first_gpu(g)
    w = b.graph()
    assert np.array_equal(w.col_idx, h.col_idx) and not (w.flags & 2)
    path = str(tmp_path / "g.bin")
    gb.save(g, path)
    f = gb.GpuBfs.from_file(path).graph()
    assert f.equal(g)
