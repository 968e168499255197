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


def test_tuned_schedules_of_the_hierarchy():
    """The hierarchy build chooses the lane-group size of each coarse
    operator and restriction, and the load depth of the level-0 pass, by
    timing whole V-cycles on the device (amg_tune_lanes): every level but the
    coarsest reports a restriction
    schedule, every level smoothed with CSR rows an operator schedule, each a
    power of two in 2..32 with a positive launch time; the solve converges
    with them.  On the r = 5 nm tip (307k cells) the hierarchy has at least
    three levels."""
    import sys
    from conftest import GOLDEN as G
    sys.path.insert(0, str(G))
    from make_tip5 import TIP5
    from tapsim_modified_b200.tapsim import Grid, Mesh
    g = Grid(Mesh.from_tip(**TIP5))
    info = g.solve(rel_tol=1e-8, max_outer=50, max_inner=20000, preconditioner=1)
    assert info.rel_residual <= 1e-8 and info.setup_seconds > 0
    sched = g.amg_schedule()
    print(sched)
    assert len(sched) >= 3
    assert sched[0]["rows"] > sched[1]["rows"] > sched[-1]["rows"]
    for k, lv in enumerate(sched):
        last = k == len(sched) - 1
        assert (lv["r_lanes"] in (2, 4, 8, 16, 32) and lv["r_ms"] > 0) if not last else lv["r_lanes"] == 0
        if k == 0:
            assert lv["a_lanes"] in (4, 8, 16, 1004, 1008) and lv["a_ms"] > 0   # the level-0 pass (1000+: pipelined)
        elif k < len(sched) - 1:
            assert lv["a_lanes"] in (2, 4, 8, 16, 32) and lv["a_ms"] > 0
        else:
            assert lv["a_lanes"] == 0
    g.close()


def test_replayed_iterations_match_launched_ones(ref_mesh, ref_events):
    """The multigrid solve's CG iterations replayed from a captured CUDA graph
    (the default), launched kernel by kernel, and replayed inside a
    device-side loop (one launch per inner solve) give the same events: the
    same removals, residuals at the tolerance and potentials equal to the
    solves' own accuracy; the graph's kernels count once per replay."""
    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    out = {}
    for mode in (0, 1, 2):
        g = Grid(ref_mesh)
        g.set_launch_mode(mode)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
        ev = Evaporation(g, EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini")), relax_mode=1,
                         solve=solve_opts(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1,
                                          warm_start=1))
        n0 = N.lib().tg_launch_count(g._h)
        recs = ev.run(12)
        launches = N.lib().tg_launch_count(g._h) - n0
        out[mode] = ([r["node"] for r in recs], [r["rel_residual"] for r in recs], g.potentials(), launches)
        g.close()
    (n0_, r0, phi0, l0), (n1, r1, phi1, l1), (n2, r2, phi2, l2) = out[0], out[1], out[2]
    print("launches over 12 events: kernel by kernel", l0, "replayed", l1, "in a device-side loop", l2)
    assert n0_ == n1 == n2 == [int(x) for x in ref_events[:12, 1]]
    assert max(r0 + r1 + r2) <= 1e-10
    assert np.abs(phi1 - phi0).max() <= 1e-8 * np.abs(phi0).max()
    assert np.abs(phi2 - phi0).max() <= 1e-8 * np.abs(phi0).max()
    # the same kernels run either way (the replay adds one counter step per
    # iteration and a start per solve, the loop a condition kernel; the
    # host-driven modes also count the early-exiting kernels of a batch)
    assert 0.6 * l0 <= l1 <= 1.3 * l0 and 0.6 * l0 <= l2 <= 1.3 * l0

