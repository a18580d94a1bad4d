"""The multi-rank plumbing of bench.py on CPU (gloo, two ranks): max-over-ranks timing, whole-job
throughput of independent replicas, and the reference arm running on rank 0 only."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        slowest = bench.max_over_ranks(1.5 + rank, dist)            # rank 1 is the slow one
        value = bench.replica_throughput(world, 2, bench.WINDOW_BED_S, slowest)
        ran_reference = (bench.reference_arm(None, rank) is not None) if rank != 0 else None
        out[rank] = (slowest, value, ran_reference)
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_is_the_slowest_and_throughput_counts_every_replica():
    import bench
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for rank in range(world):
        slowest, value, _ = out[rank]
        assert slowest == pytest.approx(2.5)
        assert value == pytest.approx(world * 2 * bench.WINDOW_BED_S / 2.5)
    assert out[1][2] is False                                    # rank 1 does no reference work


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.0) == 3.0
    assert bench.replica_throughput(1, 1, bench.CYCLE_BED_S, 10.0) == pytest.approx(bench.CYCLE_BED_S / 10.0)
