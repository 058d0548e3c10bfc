"""gb_bfs_run_many: the per-source loop of gbench (src/bench/main.cpp:324-364)
as one call.  For the persistent kernel the traversals run back to back on the
stream and each result is packed, copied and widened on the host while the
next traversals run; the packed width is predicted from the sources already
finished, and a source whose depths do not fit is copied whole.  Every depth
must equal the oracle's serial BFS (integer work: exact), in every width, in
the fallback, below the packing threshold, for the host-loop variants, and
with the result kept on the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rmat_plus_path(gb, path_len):
    """R-MAT 18 (few levels) with a separate path of path_len vertices (hundreds
    or thousands of levels from a source on it) and nothing else unreached."""
    a = gb.gen.rmat(18, 8, False, 21)
    n = a.n + path_len
    rows = np.repeat(np.arange(a.n, dtype=np.uint32), np.diff(a.row_ptr.astype(np.int64)))
    keep = rows < a.col_idx
    eu = np.concatenate([rows[keep], np.arange(a.n, n - 1, dtype=np.uint32)])
    ev = np.concatenate([a.col_idx[keep], np.arange(a.n + 1, n, dtype=np.uint32)])
    return gb.from_edges(n, eu, ev, False), a.n


def _og(oracle, g):
    return oracle.HostGraph(g.n, g.m, g.flags, g.row_ptr, g.col_idx)


def test_run_many_every_width_and_fallback(gb, oracle):
    g, first_path = _rmat_plus_path(gb, 3000)
    og = _og(oracle, g)
    power = gb.pick_sources(g, 5, 3)
    power = [int(s) for s in power if s < first_path]
    # two power-law sources and the path's middle queue before any result is
    # known (1 byte per depth: the path's 1,501 levels overflow it and its
    # buffer is copied whole), two power-law sources (4 bits, from the first
    # results), then the path's far end (2 bytes, from the path's count)
    srcs = np.array(power[:2] + [first_path + 1500] + power[2:4] + [g.n - 1], np.uint32)
    want = [oracle.bfs_serial(og, int(s)) for s in srcs]
    for hub_first in (False, True):
        bfs = gb.GpuBfs(g)
        if hub_first:
            bfs.hub_first()
        out, ms, lv = bfs.run_many("gpu_do_persistent", srcs)
        for i, s in enumerate(srcs):
            assert np.array_equal(out[i], want[i]), (hub_first, i, int(s))
            assert lv[i] == int(want[i][want[i] != 0xFFFFFFFF].max()) + 1
            assert ms[i] > 0
        assert lv[2] >= 255 and lv[0] < 15  # the path source and a power-law source
        assert bfs.lastLevels() == lv[-1]
        # a second call starts from the last call's level count (2 bytes here)
        out2, _, _ = bfs.run_many("gpu_do_persistent", srcs[::-1].copy())
        for i in range(len(srcs)):
            assert np.array_equal(out2[i], want[len(srcs) - 1 - i])


def test_run_many_stride_zero_device_and_selector(gb, oracle):
    g = gb.gen.chung_lu(300000, 2.8, 1.6, 24)  # 20-30 levels: one byte per depth
    og = _og(oracle, g)
    srcs = gb.pick_sources(g, 7, 5)
    want = [oracle.bfs_serial(og, int(s)) for s in srcs]
    bfs = gb.GpuBfs(g)
    one = np.empty(g.n, np.uint32)
    out, _, lv = bfs.run_many("gpu_do_persistent", srcs, out=one, stride=0)
    assert out is one and np.array_equal(one, want[-1])
    assert 15 <= lv.max() < 255
    # results kept on the device: the handle's depth buffer is the last source's
    _, ms, lv2 = bfs.run_many("gpu_do_persistent", srcs[:5], device=True)
    assert np.array_equal(lv2, lv[:5]) and (ms > 0).all()
    dev = _device_dist(gb, bfs, g.n)
    assert np.array_equal(dev, want[4])
    # a single run afterwards uses the moved buffer alike
    assert np.array_equal(bfs.run("gpu_do_persistent", int(srcs[6])), want[6])
    params = gb.default_selector_params("single")
    if params is not None:
        bfs.set_selector(params)
        o = gb.BfsOptions(selector="learned")
        out, _, _ = bfs.run_many("gpu_do_persistent", srcs, opts=o)
        for i in range(len(srcs)):
            assert np.array_equal(out[i], want[i])


def test_run_many_small_graph_and_host_loop_variants(gb, oracle):
    g = gb.gen.rmat(12, 16, False, 3)  # below the packing threshold: plain copies
    og = _og(oracle, g)
    srcs = gb.pick_sources(g, 9, 1)
    want = [oracle.bfs_serial(og, int(s)) for s in srcs]
    bfs = gb.GpuBfs(g)
    for variant in ("gpu_do_persistent", "gpu_do", "gpu_edge", "gpu_binned"):
        out, ms, lv = bfs.run_many(variant, srcs)
        for i in range(len(srcs)):
            assert np.array_equal(out[i], want[i]), (variant, i)
        assert (lv > 0).all()
    out, _, _ = bfs.run_many("gpu_do_persistent", np.zeros(0, np.uint32))
    assert out.shape == (0, g.n)


def test_run_many_rejects_bad_arguments(gb):
    g = gb.gen.rmat(12, 16, False, 3)
    bfs = gb.GpuBfs(g)
    with pytest.raises(gb.GraphError) as e:
        bfs.run_many("gpu_do_persistent", [0, g.n])
    assert e.value.status == 1 and "source out of range" in str(e.value)
    with pytest.raises(gb.GraphError) as e:
        bfs.run_many("gpu_do_persistent", [0, 1], out=np.empty(2 * g.n, np.uint32), stride=g.n - 1)
    assert e.value.status == 1 and "stride" in str(e.value)
    with pytest.raises(ValueError):
        bfs.run_many("gpu_do_persistent", [0, 1], out=np.empty(g.n, np.uint32), stride=g.n)
    with pytest.raises(gb.GraphError) as e:
        bfs.run_many(99, [0])
    assert e.value.status == 1


def _device_dist(gb, bfs, n):
    """Copies the handle's device depth array to the host (CUDA runtime)."""
    from cuda.bindings import runtime as rt
    ptr = gb.lib().gb_bfs_device_dist(bfs._h)
    host = np.empty(n, np.uint32)
    err, = rt.cudaMemcpy(host.ctypes.data, ptr, 4 * n, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    return host


@pytest.mark.parametrize("in_flight", [2, 3, 4, 8, 16])
def test_run_many_several_in_flight(gb, oracle, in_flight):
    """in_flight traversals at once, each on its own stream, state slot and
    share of the SMs: every source's depths, in every packed width and in the
    whole-buffer fallback, into separate rows, into one reused buffer (the last
    source's), and kept on the device -- equal to the oracle's serial BFS, with
    both selectors; more sources than depth buffers, so buffers are reused
    across streams."""
    g, first_path = _rmat_plus_path(gb, 2000)
    og = _og(oracle, g)
    power = [int(s) for s in gb.pick_sources(g, 14, 3) if s < first_path]
    srcs = np.array(power[:4] + [first_path + 1000] + power[4:9] + [g.n - 1] + power[9:12], np.uint32)
    want = [oracle.bfs_serial(og, int(s)) for s in srcs]
    bfs = gb.GpuBfs(g).hub_first()
    sels = [("rule", None)]
    params = gb.default_selector_params("single")
    if params is not None:
        bfs.set_selector(params)
        sels.append(("learned", params))
    for sel, _ in sels:
        o = gb.BfsOptions(selector=sel, in_flight=in_flight)
        out, ms, lv = bfs.run_many("gpu_do_persistent", srcs, opts=o)
        for i in range(len(srcs)):
            assert np.array_equal(out[i], want[i]), (sel, i)
            assert lv[i] == int(want[i][want[i] != 0xFFFFFFFF].max()) + 1
        assert (ms > 0).all()
        one = np.empty(g.n, np.uint32)
        bfs.run_many("gpu_do_persistent", srcs, out=one, stride=0, opts=o)
        assert np.array_equal(one, want[-1])
        _, _, lv2 = bfs.run_many("gpu_do_persistent", srcs, opts=o, device=True)
        assert np.array_equal(lv2, lv)
        assert np.array_equal(_device_dist(gb, bfs, g.n), want[-1])
        # a one-at-a-time call afterwards sees the same results
        assert np.array_equal(bfs.run("gpu_do_persistent", int(srcs[3]), opts=gb.BfsOptions(selector=sel)), want[3])


def test_run_many_in_flight_limits(gb):
    bfs = gb.GpuBfs(gb.gen.rmat(12, 16, False, 3))
    with pytest.raises(gb.GraphError) as e:
        bfs.run_many("gpu_do_persistent", [0], opts=gb.BfsOptions(in_flight=17))
    assert e.value.status == 1 and "in_flight" in str(e.value)


def test_run_many_batched_variant(gb, oracle):
    """gb_bfs_run_many with the batched kernel: 64 sources to a launch, then
    every row packed, copied and widened.  70 sources make two launches: the
    first of power-law sources only (4-bit rows), the second with sources on a
    300-vertex path (150+ levels: byte rows).  Every row equals the oracle's
    serial BFS, into separate rows, into one reused buffer (the last source's)
    and kept on the device."""
    g, first_path = _rmat_plus_path(gb, 300)
    og = _og(oracle, g)
    power = [int(s) for s in gb.pick_sources(g, 100, 3) if s < first_path][:64]
    assert len(power) == 64
    srcs = np.array(power + [first_path + 150, first_path, g.n - 1, power[0], power[1], first_path + 7], np.uint32)
    want = [oracle.bfs_serial(og, int(s)) for s in srcs]
    bfs = gb.GpuBfs(g).hub_first()
    for sel in ("rule", "learned"):
        params = gb.default_selector_params("batch")
        if sel == "learned":
            if params is None:
                continue
            bfs.set_selector(params, 1)
        o = gb.BfsOptions(selector=sel)
        out, ms, lv = bfs.run_many("batch", srcs, opts=o)
        for i in range(len(srcs)):
            assert np.array_equal(out[i], want[i]), (sel, i)
        assert (ms > 0).all()
        assert lv[0] == lv[63] and lv[64] == lv[69] and lv[64] > lv[0]
        assert lv[0] >= int(max(w[w != 0xFFFFFFFF].max() for w in want[:64])) + 1
        one = np.empty(g.n, np.uint32)
        bfs.run_many("batch", srcs, out=one, stride=0, opts=o)
        assert np.array_equal(one, want[-1])
        bfs.run_many("batch", srcs[:5], opts=o, device=True)
        assert np.array_equal(_device_dist(gb, bfs, g.n), want[4])
