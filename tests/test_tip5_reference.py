"""The r = 5 nm, 307k-cell tip against the reference TAPSim built from source.

Tip: bcc Fe [110], r = 5 nm hemispherical cap on a 10 nm cylindrical shank,
vacuum coarsened out to a counter-electrode at 1 um: 88,859 atoms, 306,982
cells.  tests/golden/make_tip5.py ran the reference on this tip's node
file: its own TetGen mesh and fastSync couplings, relaxation to its float
fixed point, then 200 events with the converged ini (REFRESH_RELAXATION_
INTERVAL = 1, threshold 0, one thread; process.cpp:680-1109, 876-894).  The
device run here starts from the same node file through this project's own
mesh builder and relaxes every event to a relative residual of 1e-10.

The device run follows the reference's removals (tg_event_opts.force_nodes),
so that a near-tie where the two choices differ does not end the comparison:
at every event the reference's choice must be this run's choice too, unless
the two are within NEAR_TIE of each other in this run's probabilities.
"""
import gzip
import hashlib
import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, str(GOLDEN))
from make_tip5 import TIP5  # noqa: E402

NEAR_TIE = 1e-3   # relative probability gap below which two choices may differ
# Detector impacts, as a fraction of the hit map's radius (the largest
# impact radius of the 200 reference events): every event within
# IMPACT_MAX, their median within IMPACT_MEDIAN.  The reference holds the
# potentials at their float fixed point, and the fields before removal agree
# to 1e-4; the flight magnifies the launch region's field differences onto
# the detector, measured here at up to 1.2e-3 of the radius (median 1.5e-4),
# while this run's own FP32 and FP64 flights agree to 1.3e-4 of the impact
# radius, so the integration precision is not what moves them.
IMPACT_MAX = 2e-3
IMPACT_MEDIAN = 5e-4


def _events():
    with gzip.open(GOLDEN / "tip5_events.txt.gz", "rt") as f:
        return np.loadtxt(f)


@pytest.fixture(scope="module")
def tip5_mesh():
    from tapsim_modified_b200.tapsim import Mesh
    return Mesh.from_tip(**TIP5)


def test_generator_writes_the_fixture_nodes(tip5_mesh, tmp_path):
    """The seeded generator still writes the node file the reference ran on
    (bit for bit), so the committed reference events describe this tip."""
    p = tmp_path / "tip5.nodes"
    tip5_mesh.write_node_file(str(p), binary=True)
    want = (GOLDEN / "tip5_nodes.sha256").read_text().split()[0]
    assert hashlib.sha256(p.read_bytes()).hexdigest() == want
    a = tip5_mesh.arrays()
    assert tip5_mesh.num_nodes == 306982 and int((a["type"] == 4).sum()) == 88859


def test_reference_log_is_whole():
    ev = _events()
    assert ev.shape == (200, 34)
    assert len(set(ev[:, 1].astype(int))) == 200          # 200 distinct removals
    assert np.all(ev[:, 24] == 5)                          # every ion reached the detector plane


@pytest.mark.gpu
def test_tip5_sequence_fields_impacts(tip5_mesh):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    ev_ref = _events()
    with gzip.open(GOLDEN / "tip5_phi0.bin.gz") as f:
        phi0 = np.frombuffer(f.read(), np.float32).astype(np.float64)
    a = tip5_mesh.arrays()
    free = np.array([not a["types"][int(t)]["dirichlet"] for t in a["type"]])
    g = Grid(tip5_mesh)
    g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
    dphi0 = float(np.abs(g.potentials() - phi0)[free].max())
    print("initial relaxation: max |phi - phi_ref| over free cells", dphi0, "V")
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    sopts = solve_opts(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
    ev = Evaporation(g, opts, relax_mode=1, solve=sopts)
    recs = ev.run(len(ev_ref), force=ev_ref[:, 1].astype(np.int32))
    g.close()
    ties, worst_f, imp = [], 0.0, []
    r_map = float(np.hypot(ev_ref[:, 18], ev_ref[:, 19]).max())
    for k, (r, row) in enumerate(zip(recs, ev_ref)):
        assert r["node"] == int(row[1])
        assert r["rel_residual"] <= 1e-10
        # the reference's choice is this run's choice, or within a near-tie
        gap = (r["best_probability"] - r["probability"]) / r["best_probability"]
        assert gap < NEAR_TIE, f"event {k + 1}: reference removed {int(row[1])}, relative gap {gap:.3g}"
        if gap > 1e-6:
            ties.append((k + 1, int(row[1]), gap, float(row[6])))
        # field_o1 of the removed cell before its removal
        fb = np.array(r["fieldBefore"], np.float64)
        ef = np.linalg.norm(fb - row[8:11]) / np.linalg.norm(row[8:11])
        worst_f = max(worst_f, ef)
        assert ef <= 1e-4, f"event {k + 1}: field {fb} vs {row[8:11]}"
        # detector impact (the reference integrates in float)
        assert r["status"] == int(row[24]) == 5
        stop = np.array(r["stop"], np.float64)
        ei = np.hypot(*(stop[:2] - row[18:20])) / r_map
        imp.append(ei)
        assert ei <= IMPACT_MAX, f"event {k + 1}: impact {stop[:2]} vs {row[18:20]}"
    print("events", len(recs), "near-ties where the choices differ (event, node, gap, reference margin):", ties)
    print("largest relative field difference", worst_f, "; impact differences / hit-map radius", r_map,
          ": median", np.median(imp), "max", max(imp))
    assert np.median(imp) <= IMPACT_MEDIAN
