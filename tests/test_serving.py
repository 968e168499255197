"""Many-tip serving on the host: the seeded tip specs, the greedy
size-balanced partition of tips over GPUs, the latency percentiles, and the
whole-job bookkeeping with two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_tip_specs_are_seeded_and_in_range():
    from tapsim_modified_b200.serving import estimated_atoms, tip_specs
    a, b = tip_specs(64), tip_specs(64)
    assert a == b and len(a) == 64
    assert a != tip_specs(64, seed=7)
    r = np.array([s["cap_radius"] for s in a])
    L = np.array([s["shank_length"] for s in a])
    h = np.array([s["half_angle_deg"] for s in a])
    assert r.min() >= 4e-9 and r.max() <= 12e-9
    assert L.min() >= 10e-9 and L.max() <= 30e-9
    assert h.min() >= 0.0 and h.max() <= 15.0
    assert len({s["seed"] for s in a}) == 64
    atoms = np.array([estimated_atoms(s) for s in a])
    # the workload's span: tens of thousands to about a million atoms a tip
    assert atoms.min() > 2e4 and atoms.max() < 2e6


def test_estimated_atoms_of_the_5nm_tip():
    """A 5 nm cap on a 10 nm cylinder: the generator places 88,859 atoms."""
    from tapsim_modified_b200.serving import estimated_atoms
    est = estimated_atoms(dict(cap_radius=5e-9, shank_length=10e-9, half_angle_deg=0.0))
    assert abs(est - 88859) / 88859 < 0.05


def test_partition_is_greedy_balanced_and_complete():
    from tapsim_modified_b200.serving import partition_tips
    rng = np.random.default_rng(3)
    sizes = rng.uniform(5e4, 1e6, 64)
    for ranks in (1, 2, 3, 8):
        parts = partition_tips(sizes, ranks)
        assert len(parts) == ranks
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [sizes[p].sum() for p in parts]
        # longest-processing-time bound: max load <= mean + largest item
        assert max(loads) <= sizes.sum() / ranks + sizes.max()
        assert all(p == sorted(p) for p in parts)
    # ties go to the lowest rank; equal sizes spread round robin
    assert partition_tips([1.0] * 4, 2) == [[0, 2], [1, 3]]
    assert partition_tips([5.0, 1.0, 1.0, 1.0, 1.0, 1.0], 2) == [[0], [1, 2, 3, 4, 5]]
    with pytest.raises(ValueError):
        partition_tips([1.0], 0)


def test_latency_percentiles_nearest_rank():
    from tapsim_modified_b200.serving import latency_percentiles
    x = np.arange(1, 101, dtype=float)
    assert latency_percentiles(x) == {"p50": 50.0, "p99": 99.0}
    assert latency_percentiles([7.0]) == {"p50": 7.0, "p99": 7.0}
    assert latency_percentiles([]) == {"p50": None, "p99": None}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from tapsim_modified_b200.serving import estimated_atoms, partition_tips, tip_specs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    specs = tip_specs(64)
    mine = partition_tips([estimated_atoms(s) for s in specs], world)[rank]
    # rank r: its tips' events of 3 rounds, wall time 2 + r s, latencies
    # 10 * (r + 1) ms for each of them
    lat = [10.0 * (rank + 1)] * (3 * len(mine))
    stats = bench.merge_tip_stats(dist, 3 * len(mine), 2.0 + rank, lat)
    out[rank] = (mine, stats)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partition_and_merge():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (m0, s0), (m1, s1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(64)) and not set(m0) & set(m1)
    assert s0 == s1                                   # every rank holds the merged figures
    assert s0["events"] == 3 * 64
    assert s0["wall_s"] == 3.0                        # the slowest rank
    assert s0["events_per_s"] == 3 * 64 / 3.0
    assert s0["latencies"] == 3 * 64
    # latencies of both ranks merged: rank 0's 10 ms and rank 1's 20 ms
    n0 = 3 * len(m0)
    assert s0["p50"] == (10.0 if n0 >= 96 else 20.0)
    assert s0["p99"] == 20.0


def test_merge_without_process_group():
    import bench
    s = bench.merge_tip_stats(None, 10, 2.0, [1.0, 2.0, 3.0])
    assert s["events"] == 10 and s["events_per_s"] == 5.0 and s["p50"] == 2.0
