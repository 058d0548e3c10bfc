"""bench.py's multi-GPU path splits the headline's sources: with N ranks, 64*N sources
are picked and rank k runs sources [64k, 64k+64) in its own persistent launches; every
rank's per-source component edges and 128-bit depth digests are gathered to rank 0, which
checks all of them against the reference's cpu_do and reports the whole job's edges over
the slowest rank's device time.  The cross-rank pieces run here as two gloo ranks on
127.0.0.1 (no GPU; the oracle's serial BFS stands in for the GPU's depths): the split, the
gather, the reference check (including a planted mismatch on rank 1), the max-over-ranks
reduction every figure goes through, and the reference arm's rule that only rank 0 works
and prints."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    return dist


def _max_worker(rank, world, port, q):
    dist = _init(rank, world, port)
    try:
        import bench
        # rank r "took" 10 + r ms for the step and 5 - r ms end to end
        got = bench.max_over_ranks([10.0 + rank, 5.0 - rank], world)
        # whole-job value as the BFS workload computes it: all ranks' edges over the slowest time
        edges_per_rank = 1e9
        value = world * edges_per_rank / (got[0] * 1e-3) / 1e9
        q.put((rank, got, value))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _split_worker(rank, world, port, per_rank, plant, q):
    dist = _init(rank, world, port)
    try:
        import bench
        import oracle_py as O
        g = O.gen("rmat", 11, 8, 0, 7)
        srcs_all = O.pick_sources(g, per_rank * world, 1)
        srcs = bench.split_sources(srcs_all, world, rank, per_rank)
        depths = np.stack([O.bfs_serial(g, int(s)) for s in srcs])  # stands in for the GPU's output
        if plant and rank == 1:
            v = int(np.flatnonzero(depths[2] != O.UNREACHED)[-1])
            depths[2][v] += 1  # a wrong depth on the other rank: only its digest reaches rank 0
        deg = np.diff(g.row_ptr.astype(np.int64))
        rows = bench.gather_rows(bench.source_rows(depths, deg), world)
        res = None
        if rank == 0:
            own = {i: depths[i] for i in range(per_rank)}
            hashes = {r * per_rank + i: rows[r][i, 1:].tobytes() for r in range(world) for i in range(per_rank)}
            ok, bad, comp, cpu = bench.check_against_reference(g, srcs_all, own, hashes, timed=per_rank)
            gpu_comp = [int(x) for r in range(world) for x in rows[r][:, 0]]
            res = {"ok": ok, "bad": bad, "comp": comp, "gpu_comp": gpu_comp, "kind": cpu["kind"],
                   "srcs_all": [int(x) for x in srcs_all], "first": [int(x) for x in O.pick_sources(g, per_rank, 1)],
                   "ref_comp": [O.component_edges(g, O.bfs_serial(g, int(s))) for s in srcs_all]}
        q.put((rank, [int(x) for x in srcs], res))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _run(target, world, *args):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port) + args + (q,)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        item = q.get(timeout=180)
        out[item[0]] = item[1:]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def test_max_over_ranks_two_gloo_ranks():
    out = _run(_max_worker, 2)
    for rank in (0, 1):
        got, value = out[rank]
        assert got == [11.0, 5.0]                 # the slowest rank's times, on every rank
        assert value == pytest.approx(2 * 1e9 / 11e-3 / 1e9)


def test_source_split_gather_and_reference_check_two_gloo_ranks():
    per_rank = 6
    out = _run(_split_worker, 2, per_rank, False)
    s0, res = out[0]
    s1, _ = out[1]
    assert res["kind"] == "reference"
    # disjoint shares that cover the 2*64-style list; rank 0 keeps the 1-GPU sources
    assert s0 + s1 == res["srcs_all"] and not set(s0) & set(s1)
    assert s0 == res["first"]
    assert res["ok"] and res["bad"] is None
    # TEPS denominators from the reference's depths, equal to the GPU-side counts gathered
    assert res["comp"] == res["gpu_comp"] == res["ref_comp"]


def test_source_split_catches_a_wrong_depth_on_another_rank():
    out = _run(_split_worker, 2, 6, True)
    _, res = out[0]
    assert not res["ok"]
    assert res["bad"]["source_index"] == 6 + 2  # rank 1's third source


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3, 4.5], 1) == [3.0, 4.5]
    assert bench.gather_rows(np.ones((2, 3), np.int64), 1)[0].shape == (2, 3)


def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, ROOT)
    import bench
    bench.reference_arm(None, 2, 1)  # returns before touching args, a graph or a device
    assert capsys.readouterr().out == ""
