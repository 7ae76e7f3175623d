"""The multi-GPU form is replicas only: every rank commits its own data and the
bench reports the whole-job rate from the slowest rank.  These tests run that
plumbing (max-over-ranks timing, whole-job throughput) on world_size 2 with
the gloo backend on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's phases take r + 1, 10 - r and 3 ms
        got = bench.max_over_ranks([rank + 1.0, 10.0 - rank, 3.0], dist, "cpu")
        dist.barrier()
        out.put((rank, got, bench.replica_throughput(world, 135 << 18, 10, got[0] * 10)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_replica_throughput_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, tput in res:
        assert got == [2.0, 10.0, 3.0], (rank, got)
        # 2 replicas x 135 * 2^18 elements x 10 steps in 10 x 2 ms
        assert tput == pytest.approx(2 * (135 << 18) * 10 / 0.020)


def test_single_process_is_identity():
    import bench

    assert bench.max_over_ranks([1.5, 2.5], None, "cpu") == [1.5, 2.5]
    assert bench.replica_throughput(1, 100, 4, 2.0) == pytest.approx(200_000.0)
