"""Generates the golden fixtures of the test suite by running the reference
TAPSim built from its own sources (oracle/_ref, `make -C oracle ref`).

    python tests/golden/make_golden.py

Inputs are produced by this project's tip generator (a small bcc Fe [110]
tip in a coarsened vacuum box) and written in the reference's formats.  The
reference then meshes them with TetGen, relaxes, and evaporates with the
"oracle" ini (global relaxation to the float fixed point after every event,
maximum-probability choice).  Outputs:

    tip.nodes        node file (BINARY, meshgen layout)
    tip.cfg          configuration (ASCII)
    oracle.ini       evaporation options
    ref_mesh.dump.gz the reference's TAPSIM dump right after fastSync
                     (its TetGen tetrahedra and float couplings)
    ref_phi0.bin     float32 potential() of all nodes after the initial
                     relaxation
    ref_events.txt   one line per event (ref_harness evap columns)
    ref_phi_events.bin.gz  float32 potentials after each event

With `--modes` it adds, from the same dump, 15 events of each other
probability / choice mode of the reference (surface_3d.cpp:220-449):

    tip_t300.cfg                       tip.cfg with TEMPERATURE = 300 (Boltzmann; at
                                       1 V the field ratios are ~3e-3, and below ~70 K
                                       the reference's float exponentials underflow)
    ref_events_prob{P}_choice{C}.txt   ref_harness evap lines, P in 1..3 with
                                       choice 0, and P = 0 with choice 1
                                       (Monte-Carlo, rand() seeded 99)
    ref_events_int{I}_step{S}.txt      8 events with TRAJECTORY_INTEGRATOR_TYPE I and
                                       TRAJECTORY_STEPPER_TYPE S: (1, 2), (1, 3), (0, 1)

With `--results` it runs the reference's own `tapsim resumption` on the
dump for 6 events and keeps the results files its LogResults writes
(logResults.cpp:135-381): ref_results_ascii.txt (one file) and
ref_results_bin.00000001 / .00000004 (binary, chunk size 4).

With `--trajectories` it repeats the first 3 events of ref_events.txt and
keeps the trajectory files that the reference's own LogTrajectory writes
for them (logTrajectory.cpp:137-300, pushed as process.cpp:1048-1049 does):
ref_traj_ascii.txt (one file) and ref_traj_bin.00000001 / .00000002
(binary, chunk size 2).

With `--default-ini` it runs 40 events with the reference's shipped default
ini instead (localRelax of the 3-hop shell to 1e-2 V plus one global sweep
per event, no refresh; process.cpp:851-893) after the same initial
relaxation: ref_events_default.txt.

With `--commands` it runs two more of the reference's own `tapsim` modes
(tapsim.cpp:66-148): `make-ini` (the default initialization file,
ref_tapsim.ini) and `relaxation tip.cfg tip.nodes` with its defaults
(threshold 0, cycles of 100, a queue of 25), keeping the relaxed node file
it writes (ASCII, numbers and potentials; file_io.cpp:765-820), gzipped:
ref_relaxed_nodes.txt.gz.

With `--snapshots` it repeats the first event with Fe's DIELECTRICITY set
to 5 (tip_eps5.cfg; --no-sync keeps the dump's couplings, so only the
dielectric force changes) and keeps the snapshots that the reference's own
LogGrid and LogSurface write after it (logGrid.cpp:119-245,
logSurface.cpp:130-293), gzipped: ref_grid_ascii.00000001.gz,
ref_grid_bin.00000001.gz, ref_surf_ascii.00000001.gz (no neighbour lists)
and ref_surf_bin.00000001.gz (with neighbour lists).
"""
from __future__ import annotations

import gzip
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from tapsim_modified_b200.tapsim import INI_DEFAULTS, Mesh  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"

# small tip: R = 1.5 nm cap on a 2 nm shank, 0.6 nm lattice-vacuum shell,
# vacuum box 20 nm wide and 40 nm high
TIP = dict(cap_radius=1.5e-9, shank_length=2.0e-9, half_angle_deg=0.0, fine_shell=0.6e-9,
           box_half_width=10e-9, box_height=40e-9, seed=7)
N_EVENTS = 40
MODE_EVENTS = 15
MODES = [(1, 0), (2, 0), (3, 0), (0, 1)]
TRAJECTORY_MODES = [(1, 2), (1, 3), (0, 1)]
TRAJECTORY_EVENTS = 8


def main():
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    mesh = Mesh.from_tip(**TIP)
    mesh.write_node_file(str(HERE / "tip.nodes"), binary=True)
    mesh.write_config(str(HERE / "tip.cfg"))
    ini = dict(INI_DEFAULTS)
    ini.update({"REFRESH_RELAXATION_INTERVAL": "1", "REFRESH_RELAXATION_ERROR_THRESHOLD": "0.0",
                "RESULTS_FILENAME": "", "TRAJECTORY_FILENAME": "", "GRID_FILENAME": "", "SURFACE_FILENAME": "",
                "GEOMETRY_FILENAME": "", "DUMP_FILENAME": ""})
    (HERE / "oracle.ini").write_text("".join(f"{k} = {v}\n" for k, v in ini.items()))
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    subprocess.run([str(HARNESS), "mesh", str(HERE / "tip.cfg"), str(HERE / "tip.nodes"), str(tmp / "ref.dump")],
                   check=True, capture_output=True)
    with open(tmp / "ref.dump", "rb") as f, gzip.open(HERE / "ref_mesh.dump.gz", "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    subprocess.run([str(HARNESS), "evap", str(HERE / "tip.cfg"), "-", str(HERE / "oracle.ini"), str(N_EVENTS),
                    str(HERE / "ref_events.txt"), "--dump", str(tmp / "ref.dump"), "--threads", "1",
                    "--phi", str(HERE / "ref_phi0.bin"), "--phi-events", str(tmp / "phi_events.bin")],
                   check=True, capture_output=True)
    with open(tmp / "phi_events.bin", "rb") as f, gzip.open(HERE / "ref_phi_events.bin.gz", "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    shutil.rmtree(tmp)
    print("nodes", mesh.num_nodes, "written to", HERE)


def modes():
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    cfg = (HERE / "tip.cfg").read_text().replace("TEMPERATURE = 0\n", "TEMPERATURE = 300\n", 1)
    assert "TEMPERATURE = 300" in cfg
    (HERE / "tip_t300.cfg").write_text(cfg)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    with gzip.open(HERE / "ref_mesh.dump.gz", "rb") as f, open(tmp / "ref.dump", "wb") as g:
        shutil.copyfileobj(f, g)
    base = (HERE / "oracle.ini").read_text()
    for prob, choice in MODES:
        ini = base.replace("METHOD_EVAPORATION_PROBABILITY = 0", f"METHOD_EVAPORATION_PROBABILITY = {prob}")
        ini = ini.replace("METHOD_EVAPORATION_CHOICE = 0", f"METHOD_EVAPORATION_CHOICE = {choice}")
        (tmp / "mode.ini").write_text(ini)
        out = HERE / f"ref_events_prob{prob}_choice{choice}.txt"
        subprocess.run([str(HARNESS), "evap", str(HERE / "tip_t300.cfg"), "-", str(tmp / "mode.ini"),
                        str(MODE_EVENTS), str(out), "--dump", str(tmp / "ref.dump"), "--threads", "1"],
                       check=True, capture_output=True)
        print("mode", prob, choice, "->", out.name)
    for integ, step in TRAJECTORY_MODES:
        ini = base.replace("TRAJECTORY_INTEGRATOR_TYPE = 1", f"TRAJECTORY_INTEGRATOR_TYPE = {integ}")
        ini = ini.replace("TRAJECTORY_STEPPER_TYPE = 1", f"TRAJECTORY_STEPPER_TYPE = {step}")
        (tmp / "traj.ini").write_text(ini)
        out = HERE / f"ref_events_int{integ}_step{step}.txt"
        subprocess.run([str(HARNESS), "evap", str(HERE / "tip.cfg"), "-", str(tmp / "traj.ini"),
                        str(TRAJECTORY_EVENTS), str(out), "--dump", str(tmp / "ref.dump"), "--threads", "1"],
                       check=True, capture_output=True)
        print("trajectory", integ, step, "->", out.name)
    shutil.rmtree(tmp)


def results():
    tapsim = ROOT / "oracle" / "_ref" / "tapsim"
    if not tapsim.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    with gzip.open(HERE / "ref_mesh.dump.gz", "rb") as f, open(tmp / "ref.dump", "wb") as g:
        shutil.copyfileobj(f, g)
    shutil.copy(HERE / "oracle.ini", tmp / "oracle.ini")
    common = ["resumption", "ref.dump", "--ini-file=oracle.ini", "--event-limit=6", "--no-trajectories",
              "--no-grids", "--no-surfaces", "--no-dump", "--threads=1"]
    subprocess.run([str(tapsim), *common, "--write-ascii", "--no-chunks", "ref_results_ascii.txt"], cwd=tmp,
                   check=True, capture_output=True)
    subprocess.run([str(tapsim), *common, "--write-binary", "--chunk-size=4", "ref_results_bin"], cwd=tmp,
                   check=True, capture_output=True)
    for name in ("ref_results_ascii.txt", "ref_results_bin.00000001", "ref_results_bin.00000004"):
        shutil.copy(tmp / name, HERE / name)
        print("results ->", name)
    shutil.rmtree(tmp)


def trajectories():
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    with gzip.open(HERE / "ref_mesh.dump.gz", "rb") as f, open(tmp / "ref.dump", "wb") as g:
        shutil.copyfileobj(f, g)
    for mode, name, chunk in (("ascii", "ref_traj_ascii.txt", "0"), ("binary", "ref_traj_bin", "2")):
        subprocess.run([str(HARNESS), "evap", str(HERE / "tip.cfg"), "-", str(HERE / "oracle.ini"), "3",
                        str(tmp / "events.txt"), "--dump", str(tmp / "ref.dump"), "--threads", "1",
                        "--trajectories", str(tmp / name), mode, chunk], check=True, capture_output=True)
    for name in ("ref_traj_ascii.txt", "ref_traj_bin.00000001", "ref_traj_bin.00000002"):
        shutil.copy(tmp / name, HERE / name)
        print("trajectories ->", name)
    shutil.rmtree(tmp)


def snapshots():
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    cfg = (HERE / "tip.cfg").read_text()
    head, fe = cfg.split("NAME = Fe\n", 1)
    assert fe.startswith("CHARGE_DENSITY = 0\nDIELECTRICITY = 1\n")
    fe = fe.replace("DIELECTRICITY = 1\n", "DIELECTRICITY = 5\n", 1)
    (HERE / "tip_eps5.cfg").write_text(head + "NAME = Fe\n" + fe)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    with gzip.open(HERE / "ref_mesh.dump.gz", "rb") as f, open(tmp / "ref.dump", "wb") as g:
        shutil.copyfileobj(f, g)
    for mode, grid, surf, nb in (("ascii", "ref_grid_ascii", "ref_surf_ascii", "0"),
                                 ("binary", "ref_grid_bin", "ref_surf_bin", "1")):
        subprocess.run([str(HARNESS), "evap", str(HERE / "tip_eps5.cfg"), "-", str(HERE / "oracle.ini"), "1",
                        str(tmp / "events.txt"), "--dump", str(tmp / "ref.dump"), "--threads", "1", "--no-sync",
                        "--grids", str(tmp / grid), mode, "--surfaces", str(tmp / surf), mode, nb],
                       check=True, capture_output=True)
        for name in (grid, surf):
            with open(tmp / f"{name}.00000001", "rb") as f, \
                    gzip.open(HERE / f"{name}.00000001.gz", "wb", compresslevel=9) as g:
                shutil.copyfileobj(f, g)
            print("snapshot ->", f"{name}.00000001.gz")
    shutil.rmtree(tmp)


def default_ini():
    """40 events of the golden tip with the reference's shipped default ini
    (local relaxation of the 3-hop shell to 1e-2 V plus one global sweep per
    event, no refresh), one thread, after the initial relaxation to the float
    fixed point: ref_events_default.txt."""
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    with gzip.open(HERE / "ref_mesh.dump.gz", "rb") as f, open(tmp / "ref.dump", "wb") as g:
        shutil.copyfileobj(f, g)
    ini = dict(INI_DEFAULTS)
    ini.update({"RESULTS_FILENAME": "", "TRAJECTORY_FILENAME": "", "GRID_FILENAME": "", "SURFACE_FILENAME": "",
                "GEOMETRY_FILENAME": "", "DUMP_FILENAME": ""})
    (tmp / "default.ini").write_text("".join(f"{k} = {v}\n" for k, v in ini.items()))
    subprocess.run([str(HARNESS), "evap", str(HERE / "tip.cfg"), "-", str(tmp / "default.ini"), str(N_EVENTS),
                    str(HERE / "ref_events_default.txt"), "--dump", str(tmp / "ref.dump"), "--threads", "1",
                    "--init-relax", "0", "100", "25"], check=True, capture_output=True)
    print("default ini ->", "ref_events_default.txt")
    shutil.rmtree(tmp)


def commands():
    """The reference's make-ini and relaxation modes (see the docstring)."""
    tapsim = ROOT / "oracle" / "_ref" / "tapsim"
    if not tapsim.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    tmp = HERE / "_tmp"
    tmp.mkdir(exist_ok=True)
    subprocess.run([str(tapsim), "make-ini", str(HERE / "ref_tapsim.ini")], check=True, capture_output=True, cwd=tmp)
    subprocess.run([str(tapsim), "relaxation", str(HERE / "tip.cfg"), str(HERE / "tip.nodes"), str(tmp / "relaxed.nodes")],
                   check=True, capture_output=True, cwd=tmp)
    with open(tmp / "relaxed.nodes", "rb") as f, gzip.open(HERE / "ref_relaxed_nodes.txt.gz", "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    print("commands ->", "ref_tapsim.ini", "ref_relaxed_nodes.txt.gz")
    shutil.rmtree(tmp)


if __name__ == "__main__":
    if "--commands" in sys.argv:
        commands()
    elif "--default-ini" in sys.argv:
        default_ini()
    elif "--modes" in sys.argv:
        modes()
    elif "--results" in sys.argv:
        results()
    elif "--trajectories" in sys.argv:
        trajectories()
    elif "--snapshots" in sys.argv:
        snapshots()
    else:
        main()
