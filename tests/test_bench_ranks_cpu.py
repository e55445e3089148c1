"""Multi-rank bench logic on CPU: two gloo ranks run the same reduction the
bench runs over NCCL after its timed region (max of the per-rank times, sum of
the per-rank counts), and the reference arm does its work on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r reports time 1 + r and counts (10 r, 1); then a second reduction
        # with no counts, as the bench's e2e leg does
        times, counts = bench.reduce_over_ranks([1.0 + rank], [10.0 * rank, 1.0], world)
        t2, c2 = bench.reduce_over_ranks([0.5 * (world - rank)], [], world)
        out[rank] = (times, counts, t2, c2, bench.rank_seed(5, rank))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        times, counts, t2, c2, seed = out[r]
        assert times == [2.0]                  # max over ranks
        assert counts == [10.0, 2.0]           # sums: pair evaluations, instances
        assert t2 == [1.0] and c2 == []
    assert out[0][4] != out[1][4]              # each rank generates its own batch


def test_reduce_single_rank_is_identity():
    import bench
    assert bench.reduce_over_ranks([3.5], [7], 1) == ([3.5], [7.0])


def test_reference_arm_other_ranks_do_no_work(capsys):
    import bench

    class A:
        pass
    assert bench.reference_arm(A(), 2, 1) == 0
    assert capsys.readouterr().out == ""
