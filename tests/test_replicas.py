"""The multi-GPU path of bench.py is N independent replicas (the step does not
shard); its only collective is the max-over-ranks timing.  Covered here with
world_size 2 over gloo on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [10.0 + 5.0 * rank, 100.0 - rank]
    got = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (got, bench.aggregate_throughput(world, 1000, got[0]))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        got, thr = out[r]
        assert got == [15.0, 100.0]
        assert thr == pytest.approx(2 * 1000 / 0.015)


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]
    assert bench.aggregate_throughput(1, 500, 250.0) == pytest.approx(2000.0)
