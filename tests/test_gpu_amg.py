"""The multigrid preconditioner of the inner solve (tg_solve_opts
.preconditioner = 1) against the Jacobi one: the same potentials at the same
tolerance, in fewer iterations, and the reference's event sequence."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_multigrid_solve_matches_jacobi(small_mesh):
    from tapsim_modified_b200.tapsim import Grid
    out = {}
    for pre in (0, 1):
        g = Grid(small_mesh)
        info = g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=pre)
        assert info.rel_residual <= 1e-10
        out[pre] = (g.potentials(), info.inner, info.setup_seconds)
        g.close()
    phi0, it0, _ = out[0]
    phi1, it1, setup = out[1]
    print("inner iterations: Jacobi", it0, "multigrid", it1, "setup", setup)
    assert setup > 0.0
    scale = np.abs(phi0).max()
    assert np.abs(phi1 - phi0).max() <= 1e-8 * scale
    assert it1 <= 0.5 * it0


def test_multigrid_events_follow_reference(ref_mesh, ref_events):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    g = Grid(ref_mesh)
    g.solve(rel_tol=1e-10, preconditioner=1)
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=1, preconditioner=1))
    recs = ev.run(20)
    for r, row in zip(recs, ref_events):
        assert r["node"] == int(row[1])
        assert r["rel_residual"] <= 1e-10
        fb = np.array(r["fieldBefore"])
        assert np.linalg.norm(fb - row[8:11]) <= 1e-4 * np.linalg.norm(row[8:11])
    g.close()
