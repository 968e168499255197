"""Evaporation-event throughput of the device hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--tip tip15|tip5]

A step is one evaporation event of the reference's loop (Process::evaporation
steps I-VI): field ratio + argmax over the surface, removal of the chosen
atom with its coupling update, relaxation to a relative residual <= 1e-8,
fields of the new surface, and the flight of the removed ion to the
detector.  Workload (default): bcc Fe [110] tip, 15 nm cap on a 40 nm shank
with a 10 degree half angle (4.06M atoms), in a vacuum box coarsened to a
counter-electrode at 1 um (7.3M cells).  Inputs are synthetic (seeded tip
generator); the mesh working set (about 2.5 GB of CSR) is far larger than L2.

Prints one JSON line (rank 0).  With --gpus N under torchrun, every rank runs
its own independent tip (different seed): weak scaling, no collective on the
data path; the reported throughput is the sum of events over the maximum
device time across ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "events/s at 3M-atom tip: learned warm-start vs plain relax, same GPU, resid<=1e-8"
TIPS = {
    # the timed tip: r=15 nm cap, 40 nm shank, 10 deg half angle, vacuum to
    # 1 um (4.06M atoms, 7.3M cells)
    "tip15": dict(cap_radius=15e-9, shank_length=40e-9, half_angle_deg=10.0, fine_shell=5e-9,
                    box_half_width=0.5e-6, box_height=1.0e-6),
    # r=5 nm cap on a 10 nm cylinder, the size the reference's CPU path
    # relaxes in minutes
    "tip5": dict(cap_radius=5e-9, shank_length=10e-9, half_angle_deg=0.0, fine_shell=3e-9,
                    box_half_width=0.5e-6, box_height=1.0e-6),
    # small tip (1.06M cells): SpMV stream about 75 MB, inside L2
    "mid": dict(cap_radius=8e-9, shank_length=20e-9, half_angle_deg=5.0, fine_shell=3e-9,
                box_half_width=0.5e-6, box_height=1.0e-6),
    # profiling case (3.4M cells): SpMV stream about 210 MB, above L2 (126 MB),
    # about 3 GB on the device
    "prof": dict(cap_radius=12e-9, shank_length=30e-9, half_angle_deg=8.0, fine_shell=4e-9,
                 box_half_width=0.5e-6, box_height=1.0e-6),
    # alloy tip with probe ions: bcc Fe-1.5 at.% Cu, r=10 nm cap on a 30 nm
    # cylinder (about 1M atoms), Cu in precipitates at 2e24 m^-3 (lognormal
    # radius clipped to 1-2 nm) and at random sites
    "alloy10": dict(cap_radius=10e-9, shank_length=30e-9, half_angle_deg=0.0, fine_shell=4e-9,
                    box_half_width=0.5e-6, box_height=1.0e-6, solute_fraction=0.015, precip_density=2e24,
                    precip_rmin=1e-9, precip_rmax=2e-9),
    # training tip of the learned warm start: another shape and seed than the
    # timed tip (the network sees only neighbourhoods of removed atoms)
    "train": dict(cap_radius=10e-9, shank_length=20e-9, half_angle_deg=8.0, fine_shell=4e-9,
                  box_half_width=0.5e-6, box_height=1.0e-6),
}
REL_TOL = 1e-8
# inner preconditioner of every solve: the multigrid V-cycle
PRECOND = 1


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = []
        for line in self.path.read_text().splitlines()[1:]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        mhz = [float(r[1].split()[0]) for r in rows if r[1].split()[0].replace(".", "").isdigit()]
        mx = [float(r[2].split()[0]) for r in rows if r[2].split()[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic_ratio(kernel: str):
    """DRAM traffic / algorithmic bytes of the named kernel from its committed
    ncu summary (captured on a smaller tip; scales with the rows processed)."""
    p = ROOT / "profiles" / f"{kernel}_prof_tip.md"
    if not p.exists():
        return None
    m = re.search(r"^(?:\w+_)?traffic_ratio:\s*([0-9.eE+-]+)", p.read_text(), re.M)
    return float(m.group(1)) if m else None


def reference_run(dump: Path, cfg: Path, n_events: int, threads: int, ini: dict | None = None,
                  label: str | None = None) -> tuple[list[float], str]:
    """The reference's own per-event path (oracle/_ref/ref_harness, built from
    the reference sources) on the same mesh, resumed from a TAPSIM dump;
    per-event wall times.  ini: the evaporation options (default: the
    reference's shipped defaults)."""
    harness = ROOT / "oracle" / "_ref" / "ref_harness"
    if not harness.exists():
        raise FileNotFoundError(harness)
    from tapsim_modified_b200.tapsim import INI_DEFAULTS
    ini_path = dump.with_suffix(".ini")
    # the reference's shipped defaults (tapsim.ini): local 3-hop relaxation
    # plus one global sweep per event, no refresh
    ini_path.write_text("".join(f"{k} = {v}\n" for k, v in (ini or INI_DEFAULTS).items()))
    out = dump.with_suffix(".events")
    cmd = [str(harness), "evap", str(cfg), "-", str(ini_path), str(n_events), str(out), "--dump", str(dump),
           "--no-sync", "--no-init-relax", "--threads", str(threads)]
    subprocess.run(cmd, check=True, capture_output=True)
    walls = []
    for line in out.read_text().splitlines():
        if line.startswith("#"):
            continue
        walls.append(float(line.split()[-1]))
    return walls, label or "reference TAPSim default ini: localRelax(shell 3) + 1 global sweep per event"


def reduce_over_ranks(dist, maxed: list, summed: list, device: str):
    """Max over ranks of the times, sum over ranks of the event counts (the
    whole-job throughput is the events of all ranks over the slowest rank's
    time).  Without a process group the values pass through."""
    if not dist:
        return [float(x) for x in maxed], [float(x) for x in summed]
    import torch
    t = torch.tensor([*maxed, *summed], dtype=torch.float64, device=device)
    mx = t[:len(maxed)].clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t[len(maxed):].clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return [float(x) for x in mx], [float(x) for x in sm]


def tip_seed(rank: int) -> int:
    """Each rank evaporates its own tip (independent units, weak scaling)."""
    return 1 + rank


def build_mesh(tip: str, seed: int):
    from tapsim_modified_b200.tapsim import Mesh
    t = time.time()
    m = Mesh.from_tip(seed=seed, **TIPS[tip])
    log(f"mesh {m.num_nodes} nodes, {m.nnz} couplings, built in {time.time() - t:.1f} s")
    return m


def train_learner(args, rank: int, opts):
    """Learned near field: samples from events on a training tip of another
    shape and seed (recycled start, one sample per event), trained on the
    device by the project's own forward and backward kernels; the last tenth
    of the samples is held out.  Returns the learner and a summary."""
    from tapsim_modified_b200.tapsim import Evaporation, Grid, Learner, Mesh, solve_opts
    t0 = time.perf_counter()
    tmesh = Mesh.from_tip(seed=101 + rank, **TIPS["train"])
    tgrid = Grid(tmesh)
    tgrid.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
    learner = Learner(hops=6, max_cells=1024, ell_width=64, seed=7 + rank)
    learner.set_refine(args.refine)
    learner.attach(tgrid, collect=True)
    # samples of the state the learned start sees: the recycled far field
    tev = Evaporation(tgrid, opts, relax_mode=1,
                      solve=solve_opts(rel_tol=REL_TOL, max_outer=50, max_inner=20000, warm_start=1,
                                       preconditioner=PRECOND))
    tev.run(args.train_events)
    learner.attach(tgrid)
    tgrid.close()
    n, cells = learner.samples()
    hold = max(1, n // 10)
    train_n = n - hold
    before = learner.gradients(train_n, hold)[0]
    last = learner.train(args.train_steps, batch=8, lr=1e-3, seed=rank, first=0, count=train_n)
    after = learner.gradients(train_n, hold)[0]
    return learner, {"train_tip": f"train: r={TIPS['train']['cap_radius'] * 1e9:g} nm cap, "
                                  f"{TIPS['train']['shank_length'] * 1e9:g} nm shank, seed {101 + rank}, "
                                  f"{tmesh.num_nodes} cells",
                     "samples": n, "cells_per_sample": cells / max(n, 1), "train_steps": args.train_steps,
                     "train_loss_last": last, "heldout_loss_untrained": before, "heldout_loss_trained": after,
                     "setup_s": time.perf_counter() - t0}


def run_ours(args, rank: int, world: int, dist):
    import ctypes as C

    import numpy as np
    import torch

    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Learner, Mesh, solve_opts

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    L = N.lib()
    # context and library warm-up on a small tip
    warm = Grid(Mesh.from_tip(cap_radius=1.5e-9, shank_length=2e-9, fine_shell=0.6e-9, box_half_width=10e-9,
                              box_height=40e-9))
    warm.solve()
    warm.close()

    mesh = build_mesh(args.tip, seed=tip_seed(rank))
    arrays = mesh.arrays()
    atoms = int((arrays["type"] == 4).sum())
    h2d_bytes = sum(v.nbytes for k, v in arrays.items() if isinstance(v, np.ndarray))
    opts = EvaporationOptions.from_ini(None)

    def run_arm(name: str, warm_start: int, learner=None, inner_precision: int = 0, long_run: int = 0):
        """Mesh upload, initial relaxation, W warm-up and K timed events with
        the given solve start (and long_run more events timed after them);
        returns the timings and the event records.  The grid stays open."""
        sopts = solve_opts(rel_tol=REL_TOL, max_outer=50, max_inner=20000, inner_rtol=args.inner_rtol,
                           warm_start=warm_start,
                           preconditioner=PRECOND, inner_precision=inner_precision)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        grid = Grid(mesh)                       # host -> device upload of the mesh
        grid.set_launch_mode(args.launch_mode)
        # initial relaxation; builds the multigrid hierarchy
        info0 = grid.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        if learner is not None:
            learner.attach(grid, predict=True)
        ev = Evaporation(grid, opts, relax_mode=1, solve=sopts)
        # the clock sampler runs from before the warm-up to the end of the
        # long run, so that its 200 ms samples cover the timed events
        with ClockSampler(local) as clocks:
            ev.run(args.warmup)
            # timed region: K events in one call of the public API (flights
            # overlap the next event's relaxation); device time with CUDA
            # events on the handle's stream, end-to-end time on the host clock
            # around the call, which takes each event's options from host
            # memory and returns its record to host memory
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            launches0 = L.tg_launch_count(grid._h)
            torch.cuda.nvtx.range_push(f"timed_{name}")
            t1 = time.perf_counter()
            N.check(L.tg_timer_start(grid._h), grid._h)
            ev.run(args.steps)
            ms = C.c_float()
            N.check(L.tg_timer_stop(grid._h, C.byref(ms)), grid._h)
            t_e2e = time.perf_counter() - t1
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
            launches = L.tg_launch_count(grid._h) - launches0
            long_ms = None
            if long_run:
                N.check(L.tg_timer_start(grid._h), grid._h)
                ev.run(long_run)
                lm = C.c_float()
                N.check(L.tg_timer_stop(grid._h, C.byref(lm)), grid._h)
                long_ms = lm.value
        phi = grid.potentials()                 # device -> host result
        return {"grid": grid, "info0": info0, "dev_s": ms.value / 1e3, "t_e2e": t_e2e, "launches": launches,
                "records": ev.records, "clocks": clocks, "phi": phi, "setup_s": setup_s, "long_ms": long_ms}

    def iters(arm, first=None, last=None):
        recs = arm["records"][args.warmup:][first:last]
        return [r["relax_iterations"] for r in recs]

    def seq_diff(a, b):
        return next((k for k, (x, y) in enumerate(zip([r["node"] for r in a["records"]],
                                                      [r["node"] for r in b["records"]])) if x != y), None)

    learner, learn_info = (None, None) if args.no_learned else train_learner(args, rank, opts)
    plain = run_arm("plain", 0)
    plain["grid"].close()
    recycled = run_arm("recycled", 1)
    recycled["grid"].close()
    fp64 = run_arm("fp64_inner", 0, inner_precision=1)
    fp64["grid"].close()
    # the headline arm: the learned warm start (warm_start 2), the metric's
    # subject; without a learner the plain start
    arm = run_arm("learned", 2, learner, long_run=args.long_events) if learner is not None \
        else run_arm("plain_value", 0, long_run=args.long_events)
    grid, info0, dev_s, t_e2e, phi, clocks = (arm[k] for k in ("grid", "info0", "dev_s", "t_e2e", "phi", "clocks"))
    launches = arm["launches"]
    # the autotuned schedule of the value arm's hierarchy: per level its rows,
    # lanes per CSR row (level 0: the smoothing pass's load depth, 1000+ for
    # the pipelined kernel) and the kept launches' times
    schedule = [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in lv.items()} for lv in grid.amg_schedule()] \
        if PRECOND == 1 else None
    recs = arm["records"][args.warmup:]
    resid = max(r["rel_residual"] for r in recs + plain["records"][args.warmup:])
    # roofline of the dominant kernel (the multigrid's level-0 smoothing
    # pass, the largest share of the event's device time) on this mesh, and
    # of the CG SpMV and the FP64 residual beside it
    avg = C.c_float()
    nbytes = C.c_double()
    N.check(L.tg_bench_kernel(grid._h, 2, 50, C.byref(avg), C.byref(nbytes)), grid._h)
    fine_gbs = nbytes.value / (avg.value / 1e3) / 1e9
    s_avg = C.c_float()
    s_bytes = C.c_double()
    N.check(L.tg_bench_kernel(grid._h, 0, 50, C.byref(s_avg), C.byref(s_bytes)), grid._h)
    spmv_gbs = s_bytes.value / (s_avg.value / 1e3) / 1e9
    r_avg = C.c_float()
    r_bytes = C.c_double()
    N.check(L.tg_bench_kernel(grid._h, 1, 20, C.byref(r_avg), C.byref(r_bytes)), grid._h)
    long_iters = [r["relax_iterations"] for r in arm["records"][args.warmup + args.steps:]]
    grid.close()
    if learner is not None:
        learner.close()
    precision = precision_errors(mesh, opts, args.precision_events) if args.precision_events > 0 else None

    (dev_max, e2e_max, plain_max, rec_max, f64_max), (ev_total, ev_e2e_total) = reduce_over_ranks(
        dist, [dev_s, t_e2e, plain["dev_s"], recycled["dev_s"], fp64["dev_s"]], [args.steps, args.steps], "cuda")
    if rank != 0:
        return None

    peak, peak_kind = measured_peak_hbm()
    traffic_ratio = ncu_traffic_ratio("k_amg_fine")
    value_arm = "learned" if learner is not None else "plain"
    windows = [long_iters[k:k + 50] for k in range(0, len(long_iters), 50)]
    out = {
        "metric": METRIC,
        "value": ev_total / dev_max,
        "unit": "events/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_max * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 residual/update + f32 inner CG, f64 flights",
        "data": "synthetic (seeded bcc Fe [110] tip generator; random-init free)",
        "config": {
            "workload": f"{args.tip}: bcc Fe [110] tip r={TIPS[args.tip]['cap_radius'] * 1e9:g} nm cap, "
                        f"{TIPS[args.tip]['shank_length'] * 1e9:g} nm shank, "
                        f"{TIPS[args.tip]['half_angle_deg']:g} deg, vacuum to 1 um; {atoms} atoms, "
                        f"{mesh.num_nodes} cells per GPU; relax to rel. residual <= {REL_TOL:g} every event; "
                        + ("solve started from the learned warm start (warm_start 2)" if learner is not None
                           else "plain start (no learner)"),
            "value_arm": f"{value_arm}; the plain start (warm_start 0) is config.plain, the recycled correction "
                         "(warm_start 1) config.recycled and the FP64 inner iterations config.fp64_inner, each "
                         "timed on the same tip",
            "learned_over_plain": (plain_max / dev_max) if learner is not None else None,
            "recycled_over_plain": plain_max / rec_max,
            "events_per_gpu": args.steps,
            "plain": {"value": ev_total / plain_max, "ms_per_step": plain_max * 1e3 / args.steps,
                      "solver_iterations_median": statistics.median(iters(plain)),
                      "start": "previous event's potentials (plain relaxation)"},
            "recycled": {"value": ev_total / rec_max, "ms_per_step": rec_max * 1e3 / args.steps,
                         "solver_iterations_median": statistics.median(iters(recycled)),
                         "sequence_first_difference": seq_diff(recycled, plain),
                         "start": "plus the previous event's correction (warm_start 1)"},
            "learned": None if learner is None else dict(learn_info, **{
                "value": ev_total / dev_max, "ms_per_step": dev_max * 1e3 / args.steps,
                "solver_iterations_median": statistics.median(iters(arm)),
                "sequence_first_difference": seq_diff(arm, plain),
                "start": "recycled far field plus the network's near-field prediction (warm_start 2); training on "
                         "the device outside the timed region"}),
            "fp64_inner": {"value": ev_total / f64_max, "ms_per_step": f64_max * 1e3 / args.steps,
                           "solver_iterations_median": statistics.median(iters(fp64)),
                           "sequence_first_difference": seq_diff(fp64, plain),
                           "note": "FP64 couplings, vectors and recurrences in the inner CG (tg_solve_opts."
                                   "inner_precision 1), FP32 V-cycle; same outer FP64 test"},
            "fp64_error": precision,
            "long_run": None if not args.long_events else {
                "events": args.long_events, "arm": value_arm,
                "value": args.long_events / (arm["long_ms"] / 1e3),
                "solver_iterations_median_per_50": [statistics.median(w) for w in windows if w],
                "note": "events after the K timed ones, in one call, device time with CUDA events; shows the "
                        "rows that removals append (smoothed only until the hierarchy is rebuilt at 2% growth)"},
            "l2": "inputs larger than L2 (CSR working set ~GB)",
            "parallelism": f"independent tips, one per GPU (x{world})",
            "solver_iterations_median": statistics.median(iters(arm)),
            "max_rel_residual": resid,
            "initial_solve": {"outer": info0.outer, "inner": info0.inner, "rel_residual": info0.rel_residual},
            "preconditioner": "smoothed-aggregation multigrid V(1,1)-cycle (tg_solve_opts.preconditioner 1)"
                              if PRECOND == 1 else "Jacobi",
            "multigrid_schedule": schedule,
            "inner_rtol": args.inner_rtol,
            "launch_mode": {0: "every kernel launched from the host",
                            1: "each multigrid CG iteration replayed from one captured CUDA graph",
                            2: "the replayed CG iteration inside a device-side loop, one launch per inner solve"}
                           [args.launch_mode],
            "setup": {"seconds": arm["setup_s"], "multigrid_hierarchy_s": info0.setup_seconds,
                      "mesh_h2d_bytes": h2d_bytes,
                      "note": "mesh upload (tg_create), multigrid hierarchy and initial relaxation, once per tip"},
        },
        "e2e": {"value": ev_e2e_total / e2e_max, "unit": "events/s",
                "h2d_bytes_per_step": C.sizeof(N.tg_event_opts), "d2h_bytes_per_step": C.sizeof(N.tg_event_record),
                "note": "host clock around Evaporation.run over the K timed events (tg_run_events): each event's "
                        "options from host memory, its record (fields, impact, residual) back to host memory, the "
                        "Python record processing included; the one-time setup is config.setup"},
        "gpu_launches": int(launches),
        "roofline": {
            "kernel": "k_amg_fine (multigrid level-0 smoothing pass t = b - A y, FP32 SELL-32, non-Neumann "
                      "free rows; the largest share of an event's device time)",
            "bound": "hbm",
            "achieved": fine_gbs,
            "peak": peak,
            "unit": "GB/s",
            "frac": fine_gbs / peak,
            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_launch": nbytes.value,
            "launch_ms": avg.value,
            "timing": "CUDA events around 50 back-to-back launches on the handle's stream, on this tip's V "
                      "system after the timed events",
            "traffic": None if traffic_ratio is None else traffic_ratio * nbytes.value,
            "traffic_source": "ncu dram__bytes_read+write per launch on the 3.4M-cell tip "
                              "(profiles/k_amg_fine_prof_tip.md), scaled by the algorithmic bytes of this launch",
            "cg_spmv_kernel_gbs": spmv_gbs,
            "residual_kernel_gbs": r_bytes.value / (r_avg.value / 1e3) / 1e9,
        },
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline and world == 1:
        try:
            # beside the repository: the dump of the timed tip is a few hundred MB
            with tempfile.TemporaryDirectory(prefix=".bench-", dir=str(ROOT)) as td:
                dump = Path(td) / "bench.dump"
                cfg = Path(td) / "bench.cfg"
                mesh.write_dump(str(dump), phi.astype(np.float32))
                mesh.write_config(str(cfg))
                threads = os.cpu_count() or 1
                walls, kind = reference_run(dump, cfg, args.cpu_events, threads)
            per = statistics.median(walls)
            out["cpu_baseline"] = {"value": 1.0 / per, "unit": "events/s", "cores": threads, "kind": "reference",
                                   "sample": f"{len(walls)} events of the same tip, {kind}; mesh and couplings "
                                             "resumed from a TAPSIM dump written by this library"}
        except Exception as e:  # the reference binary is built here; report why it could not run
            out["cpu_baseline"] = {"value": None, "unit": "events/s", "cores": os.cpu_count(), "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    return out


def precision_errors(mesh, opts, events: int) -> dict:
    """Per-event errors of the FP32-inner solve against FP64 solves of the
    same events (untimed).  Three grids of the tip run the same events in
    lockstep, each relaxed by the defect-correction solve with:

      fp32   FP32 inner iterations, rel. residual 1e-8 (the timed path)
      fp64   FP64 inner iterations, rel. residual 1e-8
      ref64  FP64 inner iterations, rel. residual 1e-12 (the FP64 reference)

    After every event: max |phi - phi_ref64| over all cells, max |E - E_ref64|
    of field_o1 over the surface cells (relative to the largest |E| there)
    and the distance of the detector impacts (relative to the reference
    impact's radius), for fp32 and fp64.  The comparison stops where a
    removal sequence differs from ref64's (a near-tie)."""
    import numpy as np

    from tapsim_modified_b200.tapsim import Evaporation, Grid, solve_opts
    setups = {"fp32": (REL_TOL, 0), "fp64": (REL_TOL, 1), "ref64": (1e-12, 1)}
    grids, evs = {}, {}
    for name, (tol, prec) in setups.items():
        g = Grid(mesh)
        g.solve(1e-12, 50, 50000, 1e-4, preconditioner=PRECOND, inner_precision=1)
        grids[name] = g
        evs[name] = Evaporation(g, opts, relax_mode=1,
                                solve=solve_opts(rel_tol=tol, max_outer=50, max_inner=20000, preconditioner=PRECOND,
                                                 inner_precision=prec))
    rows = {"fp32": [], "fp64": []}
    compared = 0
    for _ in range(events):
        rec = {k: evs[k].step() for k in setups}
        if len({rec[k]["node"] for k in setups}) != 1:
            break
        compared += 1
        phi = {k: grids[k].potentials() for k in setups}
        surf, _ = grids["ref64"].surface()
        field = {k: grids[k].field_o1(surf) for k in setups}
        emax = float(np.linalg.norm(field["ref64"], axis=1).max())
        ref_stop = np.array(rec["ref64"]["stop"])
        for k in ("fp32", "fp64"):
            rows[k].append((float(np.abs(phi[k] - phi["ref64"]).max()),
                            float(np.linalg.norm(field[k] - field["ref64"], axis=1).max()) / emax,
                            float(np.hypot(*(np.array(rec[k]["stop"])[:2] - ref_stop[:2])) / np.hypot(*ref_stop[:2]))))
    for g in grids.values():
        g.close()
    out = {"events_compared": compared, "events_asked": events,
           "reference": "FP64 inner iterations to rel. residual 1e-12, same events",
           "columns": "max over the compared events of: max |dphi| [V] over all cells; max |dE| over the surface "
                      "cells / max |E| there (field_o1); detector impact distance / impact radius"}
    for k, v in rows.items():
        if v:
            out[k] = {"max_abs_dphi_V": max(r[0] for r in v), "max_rel_dE_surface": max(r[1] for r in v),
                      "max_rel_dimpact": max(r[2] for r in v),
                      "median_abs_dphi_V": statistics.median(r[0] for r in v)}
    return out


def merge_tip_stats(dist, events: int, wall_s: float, latencies_ms) -> dict:
    """Whole-job figures of the many-tip run: events summed over ranks, the
    slowest rank's wall time, and the per-event latency percentiles over the
    events of every rank (gathered to every rank).  Without a process group
    the values pass through."""
    from tapsim_modified_b200.serving import latency_percentiles
    lat = [float(x) for x in latencies_ms]
    if dist:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (int(events), float(wall_s), lat))
    else:
        parts = [(int(events), float(wall_s), lat)]
    total = sum(p[0] for p in parts)
    wall = max(p[1] for p in parts)
    merged = [x for p in parts for x in p[2]]
    return {"events": total, "wall_s": wall, "events_per_s": total / wall if wall > 0 else None,
            **latency_percentiles(merged), "latencies": len(merged)}


def run_many_tips(args, rank: int, world: int, dist):
    """Many-tip serving: args.tips seeded tips (cap radius U(4,12) nm, shank
    U(10,30) nm, half angle U(0,15) deg), split over the ranks by the greedy
    size-balanced partition; each round runs one event of every tip of the
    rank (tg_run_tips: one host thread per tip's handle, the device work of
    all tips overlapping on their streams).  W warm-up rounds, K timed
    rounds; aggregate events/s and the p50/p99 per-event latency over all
    ranks."""
    import ctypes as C

    import torch

    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.serving import estimated_atoms, partition_tips, run_tips, tip_specs
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Learner, Mesh, solve_opts

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    specs = tip_specs(args.tips)
    sizes = [estimated_atoms(s) for s in specs]
    mine = partition_tips(sizes, world)[rank]
    t0 = time.perf_counter()
    # independent tips: built side by side, one host thread each (the
    # library call releases the interpreter lock)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(mine), os.cpu_count() or 1))) as pool:
        meshes = list(pool.map(lambda k: Mesh.from_tip(threads=1, **specs[k]), mine))
    t_mesh = time.perf_counter() - t0
    opts = EvaporationOptions.from_ini(None)
    # the learned warm start: one network trained once, a copy of it per tip
    # (a learner's graph buffers serve one handle at a time)
    trained, learn_info = (None, None) if args.no_learned else train_learner(args, rank, opts)
    sopts = solve_opts(rel_tol=REL_TOL, max_outer=50, max_inner=20000, inner_rtol=args.inner_rtol,
                       warm_start=0 if trained is None else 2, preconditioner=PRECOND)
    grids, evopts, learners = [], [], []
    t0 = time.perf_counter()
    for m in meshes:
        g = Grid(m)
        g.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
        if trained is not None:
            lr = Learner(hops=6, max_cells=1024, ell_width=64, seed=7)
            lr.set_params(trained.params())
            lr.set_refine(args.refine)
            lr.attach(g, predict=True)
            learners.append(lr)
        ev = Evaporation(g, opts, relax_mode=1, solve=sopts)   # surface set and first selection
        grids.append(g)
        evopts.append(ev.opts)
    t_setup = time.perf_counter() - t0
    for w in range(args.warmup):
        run_tips(grids, evopts, w + 1)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    lat = []
    with ClockSampler(local) as clocks:
        t1 = time.perf_counter()
        for k in range(args.steps):
            _, l, _ = run_tips(grids, evopts, args.warmup + k + 1)
            lat.extend(l.tolist())
        torch.cuda.synchronize()
        wall = time.perf_counter() - t1
    cells = sum(m.num_nodes for m in meshes)
    for g in grids:
        g.close()
    for lr in learners:
        lr.close()
    if trained is not None:
        trained.close()
    stats = merge_tip_stats(dist, args.steps * len(mine), wall, lat)
    if rank != 0:
        return None
    return {"metric": "many-tip serving: aggregate events/s and p50/p99 per-event latency, resid<=1e-8",
            "value": stats["events_per_s"], "unit": "events/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": stats["wall_s"] * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64 residual/update + f32 inner CG, f64 flights",
            "data": "synthetic (seeded bcc Fe [110] tips)",
            "config": {"workload": f"{args.tips} tips, cap radius U(4,12) nm, shank U(10,30) nm, half angle "
                                   "U(0,15) deg, vacuum to 1 um; a step is one event of every tip, each relaxed "
                                   f"to rel. residual <= {REL_TOL:g}",
                       "tips_rank0": len(mine), "cells_rank0": cells,
                       "partition": "greedy size-balanced (largest first) over the ranks, no data-path exchange",
                       "latency_ms": {"p50": stats["p50"], "p99": stats["p99"], "events": stats["latencies"]},
                       "start": "learned warm start (warm_start 2), one trained network copied to every tip"
                                if learn_info else "plain start",
                       "learner": learn_info,
                       "setup_s": {"meshes_rank0": t_mesh, "upload_and_initial_relaxation_rank0": t_setup},
                       "wall_clock": "host clock around the K rounds, synchronised; max over ranks"},
            "clocks": clocks.summary()}


def run_probe_ions(args):
    """Alloy tip with probe ions: bcc Fe-1.5 at.% Cu, r = 10 nm cap on a 30 nm
    shank (about 1M atoms), Cu in seeded spherical precipitates (lognormal
    radius clipped to 1-2 nm, 2e24 m^-3) and the rest at random sites;
    evaporation fields Fe 33 V/nm, Cu 30 V/nm.  Every event (relaxed to
    1e-8) is followed by args.probe_ions probe ions launched in one kernel
    from surface cells drawn uniformly (seeded per event) and traced to the
    detector three times: in FP64, in FP32 (the reference's arithmetic) and
    mixed (FP64 within 3 cap radii of the start, FP32 beyond).  Reports the
    probe launches' ions/s and accepted steps/s (CUDA events on the handle's
    stream), the integrator's trials per ion (accepted and rejected; a warp
    waits for its slowest ion), and the FP32 and mixed hit maps against the
    FP64 one."""
    import ctypes as C

    import numpy as np
    import torch

    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts

    torch.cuda.set_device(0)
    L = N.lib()
    mesh = build_mesh("alloy10", seed=tip_seed(0))
    a = mesh.arrays()
    cu = int((a["type"] == 5).sum())
    atoms = int((a["type"] == 4).sum()) + cu
    g = Grid(mesh)
    g.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
    opts = EvaporationOptions.from_ini(None)
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=REL_TOL, max_outer=50, max_inner=20000,
                                                            preconditioner=PRECOND))
    qm = {k: v[0] / v[1] for k, v in ev.charge_mass.items() if v[1] > 0.0}
    xyz, node_tet = a["xyz"], a["node_tet"]
    fp64_radius = 3.0 * TIPS["alloy10"]["cap_radius"]
    modes = {"fp64": dict(precision=0), "fp32": dict(precision=1), "mixed": dict(precision=2, fp64_radius=fp64_radius)}
    ms = {k: 0.0 for k in modes}
    steps = {k: 0 for k in modes}
    trials = {k: [] for k in modes}   # integrator trials (accepted and rejected) per ion
    dev = {k: [] for k in ("fp32", "mixed")}
    status_ok = {k: 0 for k in modes}
    ev_ms = 0.0
    ions = 0
    rng = np.random.default_rng(11)
    ev.run(args.warmup)
    for k in range(args.steps):
        t = C.c_float()
        N.check(L.tg_timer_start(g._h), g._h)
        ev.run(1)
        N.check(L.tg_timer_stop(g._h, C.byref(t)), g._h)
        ev_ms += t.value
        cells, _ = g.surface()
        pick = rng.choice(cells, size=args.probe_ions, replace=len(cells) < args.probe_ions)
        # ions from neighbouring sites follow neighbouring paths: ordered by
        # azimuth and height, a warp's ions walk and step alike
        order = np.lexsort((np.round(xyz[pick, 2] / 1e-9), np.arctan2(xyz[pick, 1], xyz[pick, 0])))
        pick = pick[order]
        q = np.array([qm[int(t_)] for t_ in a["type"][pick]], np.float32)
        imp = {}
        for name, kw in modes.items():
            t = C.c_float()
            N.check(L.tg_timer_start(g._h), g._h)
            imp[name] = g.trace(xyz[pick], q, node_tet[pick], **kw)
            N.check(L.tg_timer_stop(g._h, C.byref(t)), g._h)
            ms[name] += t.value
            steps[name] += sum(r.steps for r in imp[name])
            trials[name].extend(r.trials for r in imp[name])
            status_ok[name] += sum(r.status == 5 for r in imp[name])
        ions += len(pick)
        ref = np.array([[r.stop[0], r.stop[1]] for r in imp["fp64"]], np.float64)
        rad = np.hypot(ref[:, 0], ref[:, 1])
        for name in dev:
            got = np.array([[r.stop[0], r.stop[1]] for r in imp[name]], np.float64)
            dev[name].extend((np.hypot(*(got - ref).T) / np.maximum(rad, 1e-30)).tolist())
    g.close()
    out = {"metric": "probe ions per event: ions/s of one launch of the event's probe ions (mixed: FP64 within "
                     "3 cap radii of the start, FP32 beyond), hit maps FP32 and mixed vs FP64",
           "value": ions / (ms["mixed"] / 1e3), "unit": "ions/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": (ev_ms + ms["mixed"]) / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 flights within 3 cap radii of the start, f32 beyond (f64 point location)",
           "data": "synthetic (seeded bcc Fe-1.5 at.% Cu tip)",
           "config": {"workload": f"alloy10: bcc Fe-1.5 at.% Cu, r=10 nm cap, 30 nm shank, {atoms} atoms ({cu} Cu), "
                                  f"{mesh.num_nodes} cells; per event: the event (rel. residual 1e-8) and "
                                  f"{args.probe_ions} probe ions from uniformly drawn surface cells in one launch",
                      "event_ms": ev_ms / args.steps,
                      "probe": {name: {"ms_per_launch": ms[name] / args.steps, "ions_per_s": ions / (ms[name] / 1e3),
                                       "steps_per_s": steps[name] / (ms[name] / 1e3),
                                       "steps_per_ion": steps[name] / ions,
                                       "trials_per_ion": {"mean": float(np.mean(trials[name])),
                                                          "p99": float(np.percentile(trials[name], 99)),
                                                          "max": int(np.max(trials[name]))},
                                       "reached_detector": status_ok[name] / ions} for name in modes},
                      "hit_map_vs_fp64": {name: {"median_rel_impact_diff": float(np.median(v)),
                                                 "p99_rel_impact_diff": float(np.percentile(v, 99)),
                                                 "max_rel_impact_diff": float(np.max(v))} for name, v in dev.items()},
                      "mixed_fp64_radius_m": fp64_radius,
                      "value_arm": "mixed, FP64 where the field is steep near the start and FP32 beyond: the all-FP32 "
                                   "launch lasts as long as its "
                                   "slowest ion, whose float step control near the tip takes several times the "
                                   "trials of any FP64 one (probe.fp32.trials_per_ion.max)",
                      "note": "impact differences relative to the FP64 impact's radius on the detector plane"}}
    return out


def hop_ball(row_ptr, col, site: int, hops: int):
    """Cells within `hops` steps of `site` in the cell graph (site included)."""
    import numpy as np
    seen = np.zeros(len(row_ptr) - 1, bool)
    seen[site] = True
    front = np.array([site], np.int64)
    for _ in range(hops):
        nb = np.concatenate([col[row_ptr[i]:row_ptr[i + 1]] for i in front]) if len(front) else front
        nb = np.unique(nb)
        nb = nb[~seen[nb]]
        seen[nb] = True
        front = nb
    return seen


def run_warm_bounds(args):
    """Upper bounds of warm starts under the solver the events use (multigrid
    PCG to a relative residual of 1e-8).  Two grids of the same tip run the
    same events in lockstep: grid A takes the plain path, which gives each
    event's exact correction d_k = phi_post - phi_pre; grid B, after the same
    removal, is set to a constructed start and re-solved, once per start:

      plain          phi_pre
      recycled       phi_pre + d_{k-1}            (previous event's correction)
      exact_ball6    phi_pre + d_k on the 6-hop ball of the removed atom
      exact_ball12   phi_pre + d_k on the 12-hop ball
      ball6+recycled phi_pre + d_k on the 6-hop ball, d_{k-1} elsewhere
      exact          phi_pre + d_k everywhere      (ceiling of any warm start)

    Every start's solve takes the full FP64 first residual (the potentials
    were written), so the starts differ only in where they begin.  Prints one
    JSON line: per start, the median inner iterations and the median solve
    time on the host clock (the call synchronises)."""
    import numpy as np
    import torch

    from tapsim_modified_b200.tapsim import Grid

    torch.cuda.set_device(0)
    mesh = build_mesh(args.tip, seed=tip_seed(0))
    arr = mesh.arrays()
    row_ptr, col = arr["row_ptr"], arr["col"]
    A, B = Grid(mesh), Grid(mesh)
    for g in (A, B):
        g.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
        g.surface_init(0)
    starts = ["plain", "recycled", "exact_ball6", "exact_ball12", "ball6+recycled", "exact"]
    rows = {s: [] for s in starts}
    plain_path = []
    d_prev = None
    for k in range(args.warmup + args.steps):
        phi_pre = A.potentials()
        sa, sb = A.select(), B.select()
        if sa.candidate != sb.candidate:
            raise RuntimeError(f"grids diverged at event {k}: {sa.candidate} vs {sb.candidate}")
        c = sa.candidate
        A.take_away(c)
        B.take_away(c)
        t0 = time.perf_counter()
        info = A.solve(REL_TOL, 50, 20000, 1e-4, warm_start=0, preconditioner=PRECOND)
        t_plain = time.perf_counter() - t0
        phi_post = A.potentials()
        d = phi_post - phi_pre
        if k >= args.warmup and d_prev is not None:
            plain_path.append((info.inner, t_plain))
            b6 = hop_ball(row_ptr, col, c, 6)
            b12 = hop_ball(row_ptr, col, c, 12)
            cand = {"plain": phi_pre, "recycled": phi_pre + d_prev, "exact_ball6": phi_pre + np.where(b6, d, 0.0),
                    "exact_ball12": phi_pre + np.where(b12, d, 0.0),
                    "ball6+recycled": phi_pre + np.where(b6, d, d_prev), "exact": phi_post}
            for s in starts:
                B.set_potentials(cand[s])
                t0 = time.perf_counter()
                bi = B.solve(REL_TOL, 50, 20000, 1e-4, warm_start=0, preconditioner=PRECOND)
                rows[s].append((bi.inner, time.perf_counter() - t0, bi.initial_rel_residual, int(b6.sum()),
                                int(b12.sum()), bi.inner - bi.inner_neumann))
        B.set_potentials(phi_post)
        d_prev = d
    out = {"impl": "warm_bounds", "workload": args.tip, "cells": mesh.num_nodes, "events": len(plain_path),
           "rel_tol": REL_TOL, "preconditioner": "multigrid V(1,1)" if PRECOND == 1 else "Jacobi",
           "plain_event_path": {"inner_median": statistics.median(x[0] for x in plain_path),
                                "solve_ms_median": 1e3 * statistics.median(x[1] for x in plain_path)},
           "starts": {s: {"inner_median": statistics.median(r[0] for r in v),
                          "inner_mean": statistics.mean(r[0] for r in v),
                          "v_system_iterations_mean": statistics.mean(r[5] for r in v),
                          "solve_ms_median": 1e3 * statistics.median(r[1] for r in v),
                          "initial_rel_residual_median": statistics.median(r[2] for r in v)}
                      for s, v in rows.items()},
           "ball_cells_median": {"6": statistics.median(r[3] for r in rows["plain"]),
                                 "12": statistics.median(r[4] for r in rows["plain"])},
           "note": "each start's solve includes a full FP64 residual pass (the potentials were written)"}
    A.close()
    B.close()
    return out


def prepare_tip(args):
    """Child-process step of the reference arm: builds the timed tip (seed
    of rank 0), relaxes it on the device to rel. residual 1e-8 and writes
    what the reference resumes from into args.prepare_tip: the configuration
    (ref.cfg), a TAPSIM dump with the relaxed potentials (ref.dump), and
    pairs.json, a seeded sample of neighbour pairs with this library's
    couplings for the reference to check.  The reference arm's own process
    never loads this library."""
    import numpy as np

    from tapsim_modified_b200.tapsim import Grid
    out = Path(args.prepare_tip)
    mesh = build_mesh(args.tip, seed=tip_seed(0))
    g = Grid(mesh)
    g.solve(REL_TOL, 50, 50000, 1e-4, preconditioner=PRECOND)
    phi = g.potentials()
    g.close()
    mesh.write_config(str(out / "ref.cfg"))
    mesh.write_dump(str(out / "ref.dump"), phi.astype(np.float32))
    a = mesh.arrays()
    rp, col, cpl, typ = a["row_ptr"], a["col"], a["coupling"], a["type"]
    types = a["types"]
    rng = np.random.default_rng(5)
    # pairs around the surface (an atom and a vacuum neighbour) and deeper
    # in the vacuum, where the faces are large
    atoms = np.nonzero(typ == 4)[0]
    vac = np.nonzero(typ != 4)[0]
    pairs = []
    for surface, pool in ((True, atoms), (False, vac)):
        taken = 0
        for i in rng.choice(pool, size=min(len(pool), 4000), replace=False):
            # an atom with a vacuum neighbour, or any vacuum cell's neighbour
            cand = [q for q in range(rp[i], rp[i + 1]) if not surface or typ[col[q]] != typ[i]]
            if not cand:
                continue
            q = int(rng.choice(cand))
            j = int(col[q])
            ti, tj = types[int(typ[i])], types[int(typ[j])]
            if ti["neumann"] or tj["neumann"]:
                continue
            ei, ej = float(ti["epsilon"]), float(tj["epsilon"])
            pairs.append({"i": int(i), "j": j, "coupling": float(cpl[q]), "eps_factor": 2 * ei * ej / (ei + ej)})
            taken += 1
            if taken == 100:
                break
    (out / "pairs.json").write_text(json.dumps({"cells": mesh.num_nodes, "atoms": int(len(atoms)), "pairs": pairs}))
    return {"prepared": str(out), "cells": mesh.num_nodes}


def reference_faces(dump: Path, pairs: list) -> dict:
    """The reference's own coupling (computeCoupling, grid_3d.cpp:1392-1409:
    eps factor * area(0.5 d) / d from get_voronoiFace + finiteArea) of each
    sampled pair, against the coupling this library computed for the dump;
    relative differences binned by face area (the reference forms lengths in
    float, so atomic-scale faces carry float noise)."""
    harness = ROOT / "oracle" / "_ref" / "ref_harness"
    argv = [str(harness), "face", str(dump)]
    for p in pairs:
        argv += [str(p["i"]), str(p["j"])]
    r = subprocess.run(argv, check=True, capture_output=True, text=True)
    got = {}
    for line in r.stdout.splitlines():
        if line.startswith("pair"):
            f = line.split()
            got[(int(f[1]), int(f[2]))] = (float(f[8]), float(f[12]))  # areaHalf, d
    bins = {"area >= 1e-18 m^2": [], "1e-19 <= area < 1e-18": [], "area < 1e-19": []}
    for p in pairs:
        area, d = got[(p["i"], p["j"])]
        ref = p["eps_factor"] * area / d
        rel = abs(p["coupling"] - ref) / max(abs(ref), 1e-300) if ref != 0.0 or p["coupling"] != 0.0 else 0.0
        key = "area >= 1e-18 m^2" if area >= 1e-18 else ("1e-19 <= area < 1e-18" if area >= 1e-19 else "area < 1e-19")
        bins[key].append(rel)
    return {k: {"pairs": len(v), "max_rel_diff": max(v) if v else None,
                "median_rel_diff": statistics.median(v) if v else None} for k, v in bins.items()}


def run_reference(args, rank: int, world: int):
    """The reference TAPSim (oracle/_ref/ref_harness, built from the
    reference's own sources) on the timed tip, on the host cores.  A child
    process prepares the tip with this library (mesh, relaxation to 1e-8 on
    the device, TAPSIM dump); this process runs only the reference:

      value          the reference's shipped default ini: localRelax (shell 3)
                     plus one global sweep per event, no residual guarantee
      converged_ini  REFRESH_RELAXATION_INTERVAL = 1, threshold 0: relaxation
                     to the float fixed point after every event, the
                     reference's nearest analogue of a residual target
      couplings      the reference's own computeCoupling of sampled pairs
                     against the couplings in the dump it resumes from"""
    if rank != 0:
        return None
    from tapsim_modified_b200.tapsim import INI_DEFAULTS  # the ini keys only; no library load
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory(prefix=".bench-", dir=str(ROOT)) as td:
        env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
        subprocess.run([sys.executable, str(ROOT / "bench.py"), "--prepare-tip", td, "--tip", args.tip], check=True,
                       env=env)
        dump, cfg = Path(td) / "ref.dump", Path(td) / "ref.cfg"
        prep = json.loads((Path(td) / "pairs.json").read_text())
        walls, kind = reference_run(dump, cfg, args.warmup + args.steps, threads)
        conv_ini = dict(INI_DEFAULTS)
        conv_ini.update({"REFRESH_RELAXATION_INTERVAL": "1", "REFRESH_RELAXATION_ERROR_THRESHOLD": "0.0"})
        conv_walls, conv_kind = reference_run(dump, cfg, args.converged_events, threads, ini=conv_ini,
                                              label="reference TAPSim converged ini: relaxation to the float fixed "
                                                    "point after every event (REFRESH_RELAXATION_INTERVAL 1, "
                                                    "threshold 0)")
        faces = reference_faces(dump, prep["pairs"])
    timed = walls[args.warmup:]
    per = sum(timed) / len(timed)
    conv_per = statistics.median(conv_walls)
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": 1.0 / per,
        "unit": "events/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 storage, f64 accumulation (reference)",
        "data": "synthetic (same seeded tip as our arm)",
        "config": {"workload": f"{args.tip}: {prep['atoms']} atoms, {prep['cells']} cells; value: {kind} (no "
                               f"residual guarantee); config.converged_ini: {conv_kind}",
                   "converged_ini": {"value": 1.0 / conv_per, "events": len(conv_walls),
                                     "ms_per_event_median": conv_per * 1e3},
                   "couplings": faces,
                   "resumed_from": "TAPSIM dump of the tip written by a child process with this library (mesh, "
                                   "couplings, potentials relaxed to rel. residual 1e-8 on the device); resumed "
                                   "with --no-sync, its couplings checked against the reference's computeCoupling "
                                   "on sampled pairs (config.couplings)"},
        "cpu_baseline": {"value": 1.0 / per, "unit": "events/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(timed)} events after {args.warmup} warm-up, {kind}"},
        "e2e": {"value": 1.0 / per, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tip", default="tip15", choices=sorted(TIPS))
    # about 10 s of the reference's per-event work on the 16 host cores (the
    # median event time of the sample gives the rate)
    ap.add_argument("--cpu-events", type=int, default=60)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--train-events", type=int, default=300, help="events collected for the learned warm start")
    ap.add_argument("--train-steps", type=int, default=600, help="Adam steps of the learned warm start")
    ap.add_argument("--no-learned", action="store_true", help="skip training and timing the learned arm")
    ap.add_argument("--inner-rtol", type=float, default=1e-4,
                    help="the inner solves' least relative reduction per FP64 defect-correction step")
    ap.add_argument("--launch-mode", type=int, default=2, choices=(0, 1, 2),
                    help="1: the multigrid CG iterations replay a captured CUDA graph; 0: kernel by kernel; "
                         "2: the replayed iteration inside a device-side loop")
    ap.add_argument("--refine", type=int, default=8,
                    help="damped Jacobi sweeps over the learned start's cells after its prediction")
    ap.add_argument("--long-events", type=int, default=200,
                    help="events run and timed after the K timed ones on the headline arm")
    ap.add_argument("--precision-events", type=int, default=20,
                    help="events of the FP32-inner vs FP64 per-event error comparison (0: skip)")
    ap.add_argument("--converged-events", type=int, default=3,
                    help="events of the reference's converged ini timed beside its default ini (reference arm)")
    ap.add_argument("--prepare-tip", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--probe-ions", type=int, default=0,
                    help="alloy tip: this many probe ions per event in one launch, FP32 / mixed / FP64 (0: off)")
    ap.add_argument("--tips", type=int, default=0,
                    help="many-tip serving: this many seeded tips, one event of each per step (0: off)")
    ap.add_argument("--warm-bounds", action="store_true",
                    help="measure the iterations of exact and recycled starts instead of the events/s line")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.prepare_tip:
        log(json.dumps(prepare_tip(args)))
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(minutes=20))
    if args.warm_bounds:
        out = run_warm_bounds(args) if rank == 0 else None
    elif args.tips > 0:
        out = run_many_tips(args, rank, world, dist)
    elif args.probe_ions > 0:
        out = run_probe_ions(args) if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, rank, world)
    else:
        out = run_ours(args, rank, world, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
