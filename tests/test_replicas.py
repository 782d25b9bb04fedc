"""The multi-GPU form of the bench is replicas only: each rank solves its
own seeded replica, ranks meet only to take the max of their times, and the
reported throughput is all ranks' units over the slowest rank's time.  The
rank plumbing is exercised here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        import bench
        # each rank reports a different time; every rank sees the max
        ms = bench.max_over_ranks(100.0 + 25.0 * rank, ws)
        bench.barrier(ws)
        out[rank] = (ms, bench.replica_seed(rank),
                     bench.aggregate_rate(1000, ms, ws, steps=2))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time_and_aggregate():
    ws = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(ws, _free_port(), out), nprocs=ws, join=True)
    got = dict(out)
    assert set(got) == {0, 1}
    for r in (0, 1):
        ms, seed, rate = got[r]
        assert ms == pytest.approx(125.0)                # the slower rank
        assert rate == pytest.approx(2 * 1000 * 2 / 0.125)
    assert got[0][1] != got[1][1]                        # distinct replicas
