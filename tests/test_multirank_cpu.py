"""The multi-rank host logic, as two gloo ranks on the CPU.

`bench.py --gpus N` draws N x 256 jobs from one seeded stream and assigns
them to ranks by HBM footprint (1d-mctdhb_b200/partition.py), every rank
computing the same assignment with no collective in the data path
(independent systems shard; weak scaling).  What is shared is the result:
the timed region is the max over ranks, the instance-steps are summed, and
only rank 0 prints.  The reference arm runs on rank 0 alone.
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


def _partition_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "1d-mctdhb_b200"))
    import bench
    import partition

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sizes = bench.mix_sizes(bench.MIX_N * world)
        # footprint proxy without the library: coefficient and Krylov bytes
        fp = [(bench.LZ + 1) * 16 * bench.dim(N, M) + 16 * 7 * M * G for N, M, G in sizes]
        mine = partition.by_footprint(fp, world)[rank]
        # the assignment every rank computed alone, gathered only to check it
        allv = [None] * world
        dist.all_gather_object(allv, (mine, sum(fp[i] for i in mine)))
        q.put((rank, allv, fp))
    finally:
        dist.destroy_process_group()


def test_footprint_partition_over_two_gloo_ranks():
    """every job of the 2 x 256-job stream lands on exactly one rank, and
    each rank's footprint is within mean + largest job"""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
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
    (r0, allv, fp), (r1, allv1, _) = res
    assert allv == allv1  # both ranks saw the same assignment
    idx = sorted(i for share, _ in allv for i in share)
    assert idx == list(range(len(fp)))  # each job exactly once
    mean = sum(fp) / 2
    for _, load in allv:
        assert load <= mean + max(fp)
    assert max(load for _, load in allv) / mean < 1.05  # LPT on a 512-job stream


def test_partition_rules_on_the_cpu():
    sys.path.insert(0, os.path.join(REPO, "1d-mctdhb_b200"))
    import partition

    sizes = [5, 9, 1, 7, 3, 3, 8, 2]
    share = partition.by_footprint(sizes, 3)
    assert sorted(i for s in share for i in s) == list(range(len(sizes)))
    loads = partition.loads(sizes, share)
    assert max(loads) <= sum(sizes) / 3 + max(sizes)
    assert partition.by_footprint(sizes, 1) == [list(range(len(sizes)))]
    ranks = partition.stream_by_footprint(sizes, 2)
    assert ranks[:3] == [0, 1, 0]  # each to the rank with the least footprint so far
    with pytest.raises(ValueError):
        partition.by_footprint(sizes, 0)


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
