"""The multi-GPU form is replicas only: each rank runs its own workload and
the job's time is the slowest rank's.  The rank-combining logic of bench.py,
run as two gloo ranks on the CPU."""

import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.slowest_rank_ms(100.0 + 50.0 * rank, world, "cpu")
        value = bench.replica_throughput(1_000_000, 4, ms, world)
        dist.barrier()
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == pytest.approx(150.0)
        # two replicas of 4 x 1e6 voxels in 150 ms
        assert value == pytest.approx(2 * 4 * 1e6 / 0.150 / 1e6)


def test_single_rank_passes_through():
    sys.path.insert(0, str(REPO))
    import bench
    assert bench.slowest_rank_ms(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(10, 2, 1000.0, 1) == pytest.approx(2e-5)
