"""The multi-GPU form of the bench is replicas only: each rank applies H to
its own vector, with one collective, the max of the step times over ranks.
Checked here with two gloo ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, gbs = bench.replica_throughput(1.0 + rank, 1e9, world, dist, "cpu")
        q.put((rank, ms, gbs))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, gbs in res:
        assert ms == 2.0                        # slowest rank
        assert gbs == pytest.approx(world * 1e9 / 2e-3 / 1e9)


def test_single_rank_needs_no_collective():
    import bench
    ms, gbs = bench.replica_throughput(4.0, 2e9, 1)
    assert ms == 4.0 and gbs == pytest.approx(500.0)
