"""bench.py's multi-GPU path runs replicas: every rank runs the whole workload on its own
GPU, and the reported figures are the whole job's work over the slowest rank's device
time.  The cross-rank pieces run here as two gloo ranks on 127.0.0.1 (no GPU): the
max-over-ranks reduction every figure goes through, and the reference arm's rule that only
rank 0 works and prints."""
import datetime
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
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


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, got, value = q.get(timeout=120)
        out[rank] = (got, value)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        got, value = out[rank]
        assert got == [11.0, 5.0]                 # the slowest rank's times, on every rank
        assert value == pytest.approx(2 * 1e9 / 11e-3 / 1e9)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3, 4.5], 1) == [3.0, 4.5]


def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, ROOT)
    import bench
    bench.reference_arm(None, 2, 1)  # returns before touching args, a graph or a device
    assert capsys.readouterr().out == ""
