"""Many independent tips: one event of every tip per round (tg_run_tips), and
the assignment of tips to GPUs.

A tip is an independent unit: its relaxations, flights and removals never
read another tip's state, so tips shard across GPUs with no exchange on the
data path (one process per GPU, each with its share of the tips).  The
shares are balanced by a greedy longest-first assignment on the tips'
estimated sizes; only the per-event latencies and counts are gathered at
the end.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N

# bcc Fe: 2 atoms per cubic cell of a = 0.2866 nm
FE_ATOMS_PER_M3 = 2.0 / (0.2866e-9) ** 3


def tip_specs(count: int = 64, seed: int = 2024, fine_shell: float = 3e-9) -> list[dict]:
    """Seeded tips of the many-tip workload: hemispherical cap radius U(4, 12)
    nm on a shank of length U(10, 30) nm with half angle U(0, 15) degrees,
    each in a vacuum box graded out to a counter-electrode at 1 um; every
    tip gets its own generator seed."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        out.append(dict(cap_radius=float(rng.uniform(4e-9, 12e-9)), shank_length=float(rng.uniform(10e-9, 30e-9)),
                        half_angle_deg=float(rng.uniform(0.0, 15.0)), fine_shell=fine_shell,
                        box_half_width=0.5e-6, box_height=1.0e-6, seed=int(seed) * 1000 + k))
    return out


def estimated_atoms(spec: dict) -> float:
    """Atoms of a tip spec: a hemisphere of the cap radius on a conical
    frustum whose top radius is the cap radius and whose sides open
    downwards at the half angle, times the bcc Fe number density."""
    r, L = spec["cap_radius"], spec["shank_length"]
    a = math.radians(spec["half_angle_deg"])
    R = r + L * math.tan(a)
    cap = 2.0 / 3.0 * math.pi * r ** 3
    frustum = math.pi * L / 3.0 * (r * r + r * R + R * R)
    return (cap + frustum) * FE_ATOMS_PER_M3


def partition_tips(sizes, ranks: int) -> list[list[int]]:
    """Greedy size-balanced assignment (longest processing time first): the
    tips, largest first (ties by index), each go to the rank with the least
    total size so far (ties: the lowest rank).  Returns each rank's tip
    indices in ascending order."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-float(sizes[k]), k))
    load = [0.0] * ranks
    parts: list[list[int]] = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += float(sizes[k])
    return [sorted(p) for p in parts]


def latency_percentiles(latencies_ms, qs=(50, 99)) -> dict:
    """Percentiles (nearest rank) of per-event latencies in ms."""
    x = np.sort(np.asarray(latencies_ms, np.float64))
    if x.size == 0:
        return {f"p{q}": None for q in qs}
    return {f"p{q}": float(x[min(x.size - 1, max(0, int(math.ceil(q / 100.0 * x.size)) - 1))]) for q in qs}


def run_tips(grids: list, opts: list, event_index: int, threads: int = 0):
    """One event on every grid (Process::evaporation steps I-VI per tip), the
    grids driven concurrently from a pool of host threads (each grid by one
    thread; tg_run_tips).  Returns (records, latency_ms, status) per grid; a
    grid whose surface is empty reports TG_ERR_NO_SURFACE in its status."""
    n = len(grids)
    hs = (C.c_void_p * n)(*[g._h.value for g in grids])
    ops = (N.tg_event_opts * n)(*opts)
    recs = (N.tg_event_record * n)()
    lat = np.zeros(n, np.float32)
    st = np.zeros(n, np.int32)
    rc = N.lib().tg_run_tips(hs, n, ops, event_index, recs, N.ptr(lat), N.ptr(st), threads)
    if rc not in (N.TG_OK, N.TG_ERR_NO_SURFACE):
        bad = int(np.nonzero(st)[0][0]) if np.any(st) else 0
        N.check(rc, grids[bad]._h)
    return list(recs), lat, st
