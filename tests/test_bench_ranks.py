"""The bench's multi-replica plumbing on CPU: two gloo ranks (no GPU).

bench.py --gpus N runs N independent replicas (one process per GPU, no
collective on the data path). What crosses ranks is the timing: a barrier
before and after the timed region and the maximum of the per-rank step times,
from which the whole-job throughput is formed. These tests run those helpers
in two gloo processes on 127.0.0.1.
"""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        bench.rank_barrier(world)
        # rank 0 is the slower replica in the first value, rank 1 in the second
        step_ms, e2e_ms = bench.max_over_ranks([2.0 if rank == 0 else 1.5, 3.0 + rank], world, "cpu")
        bench.rank_barrier(world)
        rate = bench.job_rate(262144, world, step_ms)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{step_ms} {e2e_ms} {rate}\n")
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    for row in rows:
        step_ms, e2e_ms, rate = map(float, row)
        assert step_ms == 2.0 and e2e_ms == 4.0  # the max over ranks, on every rank
        assert rate == pytest.approx(2 * 262144 / 2e-3)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([1.25, 2.5], 1, "cpu") == [1.25, 2.5]
    bench.rank_barrier(1)
    assert bench.job_rate(100, 1, 10.0) == pytest.approx(1e4)
