"""Many tips through tg_run_tips (one event of every tip per call, the
handles driven from a pool of host threads) against the same tips run one by
one through tg_run_events: the same removals, residuals and impacts."""
import numpy as np
import pytest

from conftest import SMALL_TIP

pytestmark = pytest.mark.gpu

EVENTS = 6


def _tips():
    return [dict(SMALL_TIP, seed=s, cap_radius=r) for s, r in ((31, 1.5e-9), (32, 1.8e-9), (33, 1.3e-9))]


def test_run_tips_matches_tips_run_alone():
    from tapsim_modified_b200.serving import run_tips
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Mesh, solve_opts
    opts = EvaporationOptions.from_ini(None)
    so = solve_opts(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
    meshes = [Mesh.from_tip(**t) for t in _tips()]
    alone = []
    for m in meshes:
        g = Grid(m)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
        alone.append(Evaporation(g, opts, relax_mode=1, solve=so).run(EVENTS))
        g.close()
    grids, ops = [], []
    for m in meshes:
        g = Grid(m)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
        ops.append(Evaporation(g, opts, relax_mode=1, solve=so).opts)
        grids.append(g)
    together = [[] for _ in meshes]
    for k in range(EVENTS):
        recs, lat, st = run_tips(grids, ops, k + 1, threads=3)
        assert np.all(st == 0) and np.all(lat > 0)
        for t, r in enumerate(recs):
            together[t].append(r)
    for g in grids:
        g.close()
    for a_tip, b_tip in zip(alone, together):
        for a, b in zip(a_tip, b_tip):
            assert a["node"] == b.node
            assert b.rel_residual <= 1e-10 and b.impact.status == 5
            sa, sb = np.array(a["stop"]), np.array(b.impact.stop)
            # separate solves to 1e-10 of the same tip: impacts within 1e-4
            assert np.linalg.norm(sa - sb) <= 1e-4 * np.linalg.norm(sa)


def test_run_tips_rejects_a_handle_listed_twice():
    import ctypes as C
    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Mesh
    g = Grid(Mesh.from_tip(**_tips()[0]))
    g.solve(rel_tol=1e-8, preconditioner=1)
    o = Evaporation(g, EvaporationOptions.from_ini(None), relax_mode=1).opts
    hs = (C.c_void_p * 2)(g._h.value, g._h.value)
    ops = (N.tg_event_opts * 2)(o, o)
    recs = (N.tg_event_record * 2)()
    lat = np.zeros(2, np.float32)
    st = np.zeros(2, np.int32)
    assert N.lib().tg_run_tips(hs, 2, ops, 1, recs, N.ptr(lat), N.ptr(st), 2) == N.TG_ERR_ARGUMENT
    g.close()
