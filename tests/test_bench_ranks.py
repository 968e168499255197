"""Multi-rank bookkeeping of bench.py with two gloo ranks on the CPU: each
rank runs its own tip, times are maxed and event counts summed over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank r reports a time of 1 + r seconds and 10 + r events
    mx, sm = bench.reduce_over_ranks(dist, [1.0 + rank, 5.0 - rank], [10 + rank], "cpu")
    out[rank] = (mx, sm, bench.tip_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_max_time_sum_events():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        mx, sm, seed = out[r]
        assert mx == [2.0, 5.0]          # max over ranks
        assert sm == [21.0]              # 10 + 11 events
    assert out[0][2] != out[1][2]        # each rank its own tip


def test_single_process_passes_through():
    import bench
    assert bench.reduce_over_ranks(None, [3.0], [7], "cpu") == ([3.0], [7.0])
