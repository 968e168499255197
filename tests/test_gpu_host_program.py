"""The C++ host program (tapsim_b200, csrc/host/tapsim_b200.cpp) against the
Python host on the golden tip: the same events through the same C ABI, the
results file written by the program against the Python records, field by
field, and the removal sequence against the reference's."""
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

PROGRAM = ROOT / "tapsim_modified_b200" / "tapsim_b200"
EVENTS = 12


def test_host_program_matches_python_host(golden_dump, ref_mesh, ref_events, tmp_path):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, read_results, solve_opts
    assert PROGRAM.exists(), "build the package first (python -m tapsim_modified_b200.build)"
    ini = tmp_path / "oracle.ini"
    ini.write_text((GOLDEN / "oracle.ini").read_text())
    out = tmp_path / "results_cpp.txt"
    r = subprocess.run([str(PROGRAM), f"--ini-file={ini}", f"--event-limit={EVENTS}", "--write-ascii", "--no-chunks",
                        "evaporation", f"--input-dump={golden_dump}", str(GOLDEN / "tip.cfg"), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert f"events {EVENTS}" in r.stdout
    _, rows_cpp = read_results(str(out))
    assert len(rows_cpp) == EVENTS

    g = Grid(ref_mesh)
    g.solve(rel_tol=1e-8, max_outer=50, max_inner=20000, inner_rtol=1e-4, preconditioner=1)
    opts = EvaporationOptions.from_ini(str(ini))
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-8, max_outer=50, max_inner=20000,
                                                               inner_rtol=1e-4, preconditioner=1))
    recs = ev.run(EVENTS)
    g.close()
    xyz = ref_mesh.arrays()["xyz"]
    numbers = ref_mesh.numbers()
    for k, (row, rec) in enumerate(zip(rows_cpp, recs)):
        row = np.asarray(row, np.float64)
        assert int(row[0]) == rec["index"] == k + 1
        assert int(row[1]) == rec["id"]
        assert int(row[2]) == rec["number"] == int(numbers[int(ref_events[k, 1])])
        # the ASCII results file holds about seven significant digits
        assert np.allclose(row[4:7], xyz[rec["node"]], rtol=1e-6, atol=1e-20)
        # the two hosts run separate solves to 1e-8 on the same device: the
        # float record fields agree to the solve's accuracy
        py = np.array([rec["voltage"], *rec["stop"], rec["tof"], rec["probability"], rec["potentialBefore"],
                       *rec["fieldBefore"], rec["potentialAfter"], *rec["fieldAfter"], *rec["normal"],
                       *rec["apex"]], np.float64)
        cpp = np.concatenate([[row[3]], row[7:26]])
        assert np.allclose(cpp, py, rtol=1e-5, atol=1e-12), (k, cpp - py)
