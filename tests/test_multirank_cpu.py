"""The multi-rank host logic of bench.py, as two gloo ranks on the CPU.

`bench.py --gpus N` runs one batched mix per rank with no collective in the
data path (independent systems shard; weak scaling).  What is shared is the
result: the timed region is the max over ranks, the instance-steps are
summed, and only rank 0 prints.  The reference arm runs on rank 0 alone.
"""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t, n = bench.combine_ranks(dist, 10.0 + rank, 100 * (rank + 1), "cpu")
        # the reference arm does its work on rank 0 only; rank 1 returns at once
        skipped = None
        if rank == 1:
            skipped = bench.run_reference(None) is None
        q.put((rank, t, n, skipped))
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, n, _ in res:
        assert t == 11.0  # max over ranks
        assert n == 300  # summed
    assert res[1][3] is True


def test_single_rank_combine_is_identity():
    sys.path.insert(0, REPO)
    import bench

    assert bench.combine_ranks(None, 12.5, 7, "cpu") == (12.5, 7)
