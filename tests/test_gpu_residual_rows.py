"""The first residual of a solve that follows removals from a converged state
is recomputed only on the rows the removals touched: the flipped cells
(removed and detached) and their neighbours, from the residuals the last
full pass kept.  A second grid drops its kept residuals before every solve
(by writing its own potentials back), so it takes the pass over every row.
Both must start from the same residual and end with the same
potentials, on the plain Fe tip and on one whose Cu solute is a
free dielectric species, with both preconditioners."""
import numpy as np
import pytest

from conftest import SMALL_TIP

pytestmark = pytest.mark.gpu

EVENTS = 10


def _mesh(kind, tmp_path):
    from tapsim_modified_b200.tapsim import Mesh
    if kind == "fe":
        return Mesh.from_tip(**SMALL_TIP)
    m = Mesh.from_tip(**dict(SMALL_TIP, solute_fraction=0.3))
    m.write_node_file(str(tmp_path / "t.nodes"))
    m.write_config(str(tmp_path / "t.cfg"))
    head, cu = (tmp_path / "t.cfg").read_text().split("NAME = Cu\n", 1)
    cu = cu.replace("DIELECTRICITY = 1\n", "DIELECTRICITY = 5\n", 1)
    cu = cu.replace("DIRICHLET_BOUNDARY = 1\n", "DIRICHLET_BOUNDARY = 0\n", 1)
    (tmp_path / "d.cfg").write_text(head + "NAME = Cu\n" + cu)
    return Mesh.from_files(str(tmp_path / "t.nodes"), str(tmp_path / "d.cfg"))


@pytest.mark.parametrize("kind", ["fe", "dielectric"])
@pytest.mark.parametrize("preconditioner", [0, 1])
def test_kept_residuals_match_full_pass(kind, preconditioner, tmp_path):
    from tapsim_modified_b200.tapsim import Grid
    mesh = _mesh(kind, tmp_path)
    kept, full = Grid(mesh), Grid(mesh)
    opts = dict(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=preconditioner)
    for g in (kept, full):
        g.solve(**opts)
        g.surface_init(0)
    for k in range(EVENTS):
        node = kept.select().candidate
        assert full.select().candidate == node, k
        d = kept.take_away(node)
        assert full.take_away(node) == d
        full.set_potentials(full.potentials())
        a = kept.solve(**opts)
        b = full.solve(**opts)
        assert a.residual_cells == 1 + len(d), (k, a.residual_cells, d)
        assert b.residual_cells == 0
        # a row left out, or a stale kept value, would change the sum by
        # the removal's own share of it
        assert a.initial_rel_residual == pytest.approx(b.initial_rel_residual, rel=1e-9, abs=0.0), k
        assert a.rel_residual <= 1e-10 and b.rel_residual <= 1e-10, k
        # the device sums are atomic, so the steps may differ by rounding
        assert abs(a.outer - b.outer) <= 1, (k, a.outer, b.outer)
        assert np.abs(kept.potentials() - full.potentials()).max() <= 1e-8, k
    kept.close()
    full.close()


def test_other_changes_drop_kept_residuals():
    """Writes of the potentials, relaxation sweeps and local relaxation
    between solves make the next solve take the full pass."""
    from tapsim_modified_b200.tapsim import Grid, Mesh
    g = Grid(Mesh.from_tip(**SMALL_TIP))
    opts = dict(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
    g.solve(**opts)
    g.surface_init(0)
    for change in ("none", "set", "relax", "local"):
        node = g.select().candidate
        g.take_away(node)
        if change == "set":
            g.set_potentials(g.potentials())
        elif change == "relax":
            g.relax(1)
        elif change == "local":
            g.local_relax(node, 3, 1.0, 1, 10)
        info = g.solve(**opts)
        assert (info.residual_cells > 0) == (change == "none"), change
        assert info.rel_residual <= 1e-10
    g.close()


@pytest.mark.parametrize("kind", ["fe", "dielectric"])
@pytest.mark.parametrize("warm_start", [0, 1])
def test_first_residual_matches_fp64(kind, warm_start, tmp_path):
    """A solve stopped after its first residual (max_outer 0) reports the
    relative residual of the potentials it would start from: the kept
    residuals updated on the touched rows, and with warm_start 1 the
    recycled correction already added (A hist taken off in FP32).  The
    FP64 residual of those potentials, computed afresh, must agree."""
    import ctypes as C

    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import Grid, solve_opts
    g = Grid(_mesh(kind, tmp_path))
    opts = dict(rel_tol=1e-10, max_outer=50, max_inner=20000, warm_start=warm_start, preconditioner=1)
    g.solve(**opts)
    g.surface_init(0)
    probes = 0
    for k in range(8):
        g.take_away(g.select().candidate)
        if k % 2 == 1:
            # the previous solve followed a removal, so it left a start to recycle
            info = N.tg_solve_info()
            o = solve_opts(1e-10, 0, 20000, 1e-4, warm_start, 1)
            rc = N.lib().tg_solve(g._h, C.byref(o), C.byref(info))
            assert rc == N.TG_ERR_ITERATION_CAP
            assert info.residual_cells >= 1
            tol = 1e-9 if warm_start == 0 else 1e-4
            assert info.initial_rel_residual == pytest.approx(g.residual(), rel=tol, abs=0.0), k
            probes += 1
        info = g.solve(**opts)
        assert info.rel_residual <= 1e-10
    assert probes == 4
    g.close()
