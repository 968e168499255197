"""The C++ host program (tapsim_b200, csrc/host/tapsim_b200.cpp) on the golden
tip: it runs the events through the C ABI, removes the reference's cells,
and its results file holds, field by field, what the Python host makes of the
same device records (the voltage queue and time scale of process.cpp:985-1036
in float in both)."""
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

PROGRAM = ROOT / "tapsim_modified_b200" / "tapsim_b200"
EVENTS = 12


def test_host_program_matches_python_host(golden_dump, ref_mesh, ref_events, tmp_path):
    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, read_results
    assert PROGRAM.exists(), "build the package first (python -m tapsim_modified_b200.build)"
    ini = tmp_path / "oracle.ini"
    ini.write_text((GOLDEN / "oracle.ini").read_text())
    out, raw = tmp_path / "results_cpp.txt", tmp_path / "records.bin"
    r = subprocess.run([str(PROGRAM), f"--ini-file={ini}", f"--event-limit={EVENTS}", "--write-ascii", "--no-chunks",
                        f"--records={raw}", "evaporation", f"--input-dump={golden_dump}", str(GOLDEN / "tip.cfg"),
                        str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert f"events {EVENTS}" in r.stdout
    _, rows = read_results(str(out))
    blob = raw.read_bytes()
    assert len(rows) == EVENTS and len(blob) == EVENTS * N.C.sizeof(N.tg_event_record)
    recs = (N.tg_event_record * EVENTS).from_buffer_copy(blob)
    # the program's removals are the reference's (converged ini, golden tip)
    assert [rec.node for rec in recs] == [int(x) for x in ref_events[:EVENTS, 1]]
    # the Python host's record processing of the same device records
    g = Grid(ref_mesh)
    ev = Evaporation(g, EvaporationOptions.from_ini(str(ini)), relax_mode=1)
    xyz = ref_mesh.arrays()["xyz"]
    for k, (row, rec) in enumerate(zip(rows, recs)):
        ev.event = k + 1
        d = ev._record(rec)
        row = np.asarray(row, np.float64)
        assert int(row[0]) == d["index"] == k + 1
        assert int(row[1]) == d["id"] and int(row[2]) == d["number"]
        py = np.array([d["voltage"], *xyz[d["node"]], *d["stop"], d["tof"], d["probability"], d["potentialBefore"],
                       *d["fieldBefore"], d["potentialAfter"], *d["fieldAfter"], *d["normal"], *d["apex"]],
                      np.float64)
        # the ASCII results file holds about seven significant digits
        assert np.allclose(row[3:26], py, rtol=2e-6, atol=1e-30), (k, row[3:26] - py)
    g.close()
