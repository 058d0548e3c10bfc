"""gb_prim_scan_device_noalloc, the exclusive scan that allocates no device
memory, checked through the C ABI against numpy's 64-bit cumulative sum
(reduced mod 2^32, shifted to exclusive) and against gb_prim_scan (the
allocating entry point) on the same inputs.  Integer work, so the tolerance is
exact equality.  Several calls run back to back on one stream, so each must
clear the fixed scratch the previous one left behind.  The file is named to be
collected last; it also passes alone in a fresh process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 4096 * 2048  # the entry point's documented maximum n


def _scan_noalloc(gb, torch, x: np.ndarray, in_place: bool = False):
    d_in = torch.from_numpy(x.view(np.int32)).to("cuda")
    d_out = d_in if in_place else torch.full_like(d_in, -1)
    d_tot = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    d_flag = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    gb.prim_scan_device_noalloc(d_in.data_ptr(), x.size, d_out.data_ptr(), d_tot.data_ptr(), d_flag.data_ptr(),
                                stream.cuda_stream)
    stream.synchronize()
    out = d_out.cpu().numpy().view(np.uint32)
    return out, int(d_tot.cpu().numpy().view(np.uint32)[0]), int(d_flag.cpu()[0])


def _numpy_scan(x: np.ndarray):
    """Exclusive scan mod 2^32 and the total, independently of the library."""
    c = np.cumsum(x, dtype=np.uint64)
    want = np.empty(x.size, np.uint32)
    if x.size:
        want[0] = 0
        want[1:] = (c[:-1] & 0xFFFFFFFF).astype(np.uint32)
    return want, int(c[-1] & 0xFFFFFFFF) if x.size else 0


def test_noalloc_scan_matches_numpy_at_the_limit(gb):
    """n = 8,388,608 (4096 full tiles), full 32-bit values so the sums wrap,
    out of place and in place."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(77)
    x = rng.integers(0, 1 << 32, size=LIMIT, dtype=np.uint64).astype(np.uint32)
    want, want_total = _numpy_scan(x)
    for in_place in (False, True):
        got, total, flag = _scan_noalloc(gb, torch, x, in_place)
        assert flag == 0
        np.testing.assert_array_equal(got, want)
        assert total == want_total


def test_noalloc_scan_matches_allocating_scan(gb):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024)
    # full 32-bit values (wrap-around sums), a ragged tail, the exact limit,
    # then a smaller call after a larger one
    cases = [(LIMIT, False), (3_000_001, False), (2049, True), (1, False), (LIMIT - 5, True), (77, False)]
    for n, in_place in cases:
        x = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
        want, want_total = gb.prim_scan(x)
        got, total, flag = _scan_noalloc(gb, torch, x, in_place)
        assert flag == 0, n
        np.testing.assert_array_equal(got, want)
        assert total == want_total, n
        np_want, np_total = _numpy_scan(x)
        np.testing.assert_array_equal(got, np_want)
        assert total == np_total, n


def test_noalloc_scan_two_calls_in_a_row(gb):
    """Same input twice on one stream without a host wait between the two
    enqueues: both results equal the allocating scan."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    n = 5_000_000
    x = rng.integers(0, 1000, size=n, dtype=np.uint64).astype(np.uint32)
    want, want_total = gb.prim_scan(x)
    np_want, np_total = _numpy_scan(x)
    np.testing.assert_array_equal(want, np_want)
    assert want_total == np_total
    d_in = torch.from_numpy(x.view(np.int32)).to("cuda")
    outs = [torch.empty_like(d_in), torch.empty_like(d_in)]
    tots = torch.zeros(2, dtype=torch.int32, device="cuda")
    flags = torch.full((2,), 7, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    for i in range(2):
        gb.prim_scan_device_noalloc(d_in.data_ptr(), n, outs[i].data_ptr(), tots[i:].data_ptr(),
                                    flags[i:].data_ptr(), s.cuda_stream)
    s.synchronize()
    for i in range(2):
        np.testing.assert_array_equal(outs[i].cpu().numpy().view(np.uint32), want)
    assert tots.cpu().numpy().view(np.uint32).tolist() == [want_total, want_total]
    assert flags.cpu().tolist() == [0, 0]


def test_noalloc_scan_limits(gb):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    tot = torch.full((1,), 5, dtype=torch.int32, device="cuda")
    # over the limit: rejected before anything is enqueued (buf is never read)
    with pytest.raises(gb.GraphError) as e:
        gb.prim_scan_device_noalloc(buf.data_ptr(), LIMIT + 1, buf.data_ptr(), tot.data_ptr())
    assert e.value.status == 7  # GB_ERR_CAPACITY
    with pytest.raises(gb.GraphError):
        gb.prim_scan_device_noalloc(0, 10, buf.data_ptr())
    # n == 0 writes a zero total
    gb.prim_scan_device_noalloc(buf.data_ptr(), 0, buf.data_ptr(), tot.data_ptr())
    torch.cuda.synchronize()
    assert int(tot.cpu()[0]) == 0


def test_noalloc_scan_leaves_device_memory_unchanged(gb):
    """After a first call (which looks up the scratch address), many more
    calls leave the device's free memory exactly as it was: nothing is
    allocated and kept per call."""
    torch = pytest.importorskip("torch")
    n = 1_000_003
    d_in = torch.ones(n, dtype=torch.int32, device="cuda")
    d_out = torch.empty_like(d_in)
    d_tot = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    gb.prim_scan_device_noalloc(d_in.data_ptr(), n, d_out.data_ptr(), d_tot.data_ptr(), 0, s.cuda_stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        gb.prim_scan_device_noalloc(d_in.data_ptr(), n, d_out.data_ptr(), d_tot.data_ptr(), 0, s.cuda_stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert int(d_tot.cpu()[0]) == n
    assert int(d_out[-1].cpu()) == n - 1
