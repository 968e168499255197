"""Generates the parity fixture of the r = 5 nm tip by running the reference
TAPSim built from its own sources (oracle/_ref, `make -C oracle ref`) on it.

    python tests/golden/make_tip5.py [--events 200]

Tip: bcc Fe [110], hemispherical cap r = 5 nm on a 10 nm
cylindrical shank, in a vacuum box coarsened out to a counter-electrode at
1 um: 88,859 atoms, 306,982 cells.  This project's seeded generator writes
the node file; the reference then meshes it with its own TetGen, computes its
own couplings (fastSync), relaxes to its float fixed point and evaporates 200
events with the converged ("oracle") ini: global relaxation to the float
fixed point after every event (REFRESH_RELAXATION_INTERVAL = 1, threshold
0), maximum-probability choice, one thread (process.cpp:680-1109).

Outputs (committed):
    tip5_events.txt.gz   ref_harness evap lines, one per event (removed
                            node, near-tie margin, fields, impact, ...)
    tip5_phi0.bin.gz     float32 potentials after the initial relaxation
    tip5_nodes.sha256    sha256 of the generated node file, so a test can
                            check that the generator still writes these nodes

The node file itself is not committed: tests regenerate the tip with
TIP5 (bit-identical for any thread count) and compare the hash.
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import shutil
import subprocess
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from tapsim_modified_b200.tapsim import Mesh  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"

# r = 5 nm cap on a 10 nm cylinder (half angle 0), vacuum to 1 um
TIP5 = dict(cap_radius=5e-9, shank_length=10e-9, half_angle_deg=0.0, fine_shell=3e-9,
                   box_half_width=0.5e-6, box_height=1.0e-6, seed=11)


def node_file_hash(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--events", type=int, default=200)
    args = ap.parse_args()
    if not HARNESS.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    tmp = HERE / "_tmp_tip5"   # a directory of its own: make_golden.py clears _tmp
    tmp.mkdir(exist_ok=True)
    mesh = Mesh.from_tip(**TIP5)
    nodes, cfg = tmp / "tip5.nodes", tmp / "tip5.cfg"
    mesh.write_node_file(str(nodes), binary=True)
    mesh.write_config(str(cfg))
    (HERE / "tip5_nodes.sha256").write_text(node_file_hash(nodes) + "\n")
    print("cells", mesh.num_nodes, flush=True)
    t = time.time()
    subprocess.run([str(HARNESS), "mesh", str(cfg), str(nodes), str(tmp / "tip5.dump")], check=True,
                   capture_output=True)
    print(f"reference mesh + fastSync {time.time() - t:.0f} s", flush=True)
    t = time.time()
    subprocess.run([str(HARNESS), "evap", str(cfg), "-", str(HERE / "oracle.ini"), str(args.events),
                    str(tmp / "events.txt"), "--dump", str(tmp / "tip5.dump"), "--threads", "1",
                    "--phi", str(tmp / "phi0.bin")], check=True, capture_output=True)
    print(f"reference relaxation + {args.events} events {time.time() - t:.0f} s", flush=True)
    for src, dst in ((tmp / "events.txt", HERE / "tip5_events.txt.gz"), (tmp / "phi0.bin", HERE / "tip5_phi0.bin.gz")):
        with open(src, "rb") as f, gzip.open(dst, "wb", compresslevel=9) as g:
            shutil.copyfileobj(f, g)
    shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
