"""Grid and surface snapshots from the device (tg_log_grid, tg_log_surface)
against the reference's own LogGrid / LogSurface files after the first
golden event with Fe's permittivity 5, and the snapshot schedule of the
event loop."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def after_event(ref_mesh_eps5):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    g = Grid(ref_mesh_eps5)
    g.solve(rel_tol=1e-10)
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10))
    r = ev.step()
    return g, ev, r


@pytest.mark.parametrize("binary", [False, True])
def test_grid_log_matches_reference(after_event, snapshot_files, tmp_path, binary):
    from tapsim_modified_b200.tapsim import read_grid_log
    g, ev, r = after_event
    name = g.log_grid(str(tmp_path / "grid"), 1, binary, ev.numbers)
    assert name.endswith(".00000001")
    ref_name = snapshot_files["ref_grid_bin" if binary else "ref_grid_ascii"]
    head = open(ref_name, "rb").read().split(b"\n", 3)[:3]
    assert open(name, "rb").read().split(b"\n", 3)[:3] == head
    _, mine = read_grid_log(name)
    _, ref = read_grid_log(ref_name)
    np.testing.assert_array_equal(mine["id"], ref["id"])
    np.testing.assert_array_equal(mine["number"], ref["number"])
    assert np.abs(mine["phi"] - ref["phi"]).max() < 2e-5
    assert np.abs(mine["field"] - ref["field"]).max() <= 1e-4 * np.abs(ref["field"]).max()
    scale = np.abs(ref["force"]).max()
    assert scale > 0
    assert np.abs(mine["force"] - ref["force"]).max() <= 1e-3 * scale
    np.testing.assert_array_equal(mine["force"] == 0.0, ref["force"] == 0.0)


@pytest.mark.parametrize("binary", [False, True])
def test_surface_log_matches_reference(after_event, snapshot_files, tmp_path, binary):
    """ASCII without and binary with neighbour lists, as the fixtures were
    written."""
    from tapsim_modified_b200.tapsim import read_surface_log
    g, ev, r = after_event
    name = g.log_surface(str(tmp_path / "surf"), 1, binary, with_neighbours=binary, numbers=ev.numbers)
    _, cells, nodes = read_surface_log(name)
    _, rc, rn = read_surface_log(snapshot_files["ref_surf_bin" if binary else "ref_surf_ascii"])
    for k in ("index", "type", "number"):
        np.testing.assert_array_equal(cells[k], rc[k])
    np.testing.assert_allclose(cells["probability"], rc["probability"], rtol=2e-4)
    if binary:
        for a, b in zip(cells["neighbours"], rc["neighbours"]):
            np.testing.assert_array_equal(a, b)
    else:
        assert cells["neighbours"] is None and rc["neighbours"] is None
    np.testing.assert_array_equal(nodes["index"], rn["index"])
    assert np.abs(nodes["phi"] - rn["phi"]).max() < 2e-5
    assert np.abs(nodes["field"] - rn["field"]).max() <= 1e-4 * np.abs(rn["field"]).max()
    on_surface = np.isin(nodes["index"], cells["index"])
    assert np.all(nodes["normal"][~on_surface] == 0.0)
    # normals: unit plane-fit normals, the reference's in float
    cosang = np.sum(nodes["normal"][on_surface] * rn["normal"][on_surface], axis=1)
    assert cosang.min() > 1 - 1e-4


def test_cell_values_match_oracle(after_event):
    """tg_cell_values on every cell and on a list, against the oracle's
    field_o1 and force on the device's own potentials."""
    from oracle import Oracle
    g, ev, r = after_event
    a = g.mesh.arrays()
    o = Oracle(a)
    o.phi[:] = g.potentials()
    o.type[:] = g.types()
    o.c[:] = g.couplings()
    phi, field, force = g.cell_values()
    np.testing.assert_array_equal(phi, o.phi.astype(np.float32))
    idx = np.arange(0, g.n, 7)
    E = np.array([o.field_o1(i) for i in idx])
    F = np.array([o.force(i) for i in idx])
    assert np.abs(field[idx] - E).max() <= 1e-6 * np.abs(E).max()  # float outputs
    assert np.abs(force[idx] - F).max() <= 1e-6 * np.abs(F).max()
    p2, f2, _ = g.cell_values(idx, force=False)
    np.testing.assert_array_equal(p2, phi[idx])
    np.testing.assert_array_equal(f2, field[idx])


def test_event_loop_snapshot_schedule(ref_mesh, tmp_path):
    """GRID_INTERVAL 2, SURFACE_INTERVAL 3: snapshots before the first event
    and after events 2, 3, 4, 6; batches split there, and single steps and
    batches write the same files."""
    import os
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, read_grid_log, solve_opts
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    contents = {}
    for batched in (False, True):
        d = tmp_path / ("batched" if batched else "single")
        d.mkdir()
        opts.values.update({"GRID_FILENAME": str(d / "grid"), "GRID_INTERVAL": "2", "GRID_BINARY_OUTPUT": "1",
                            "SURFACE_FILENAME": str(d / "surf"), "SURFACE_INTERVAL": "3",
                            "SURFACE_BINARY_OUTPUT": "0"})
        g = Grid(ref_mesh)
        g.solve(rel_tol=1e-10)
        ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=1), snapshots=True)
        if batched:
            recs = ev.run(6)
        else:
            recs = [ev.step() for _ in range(6)]
        assert [r["index"] for r in recs] == [1, 2, 3, 4, 5, 6]
        files = sorted(os.listdir(d))
        assert files == ["grid.00000000", "grid.00000002", "grid.00000004", "grid.00000006",
                         "surf.00000000", "surf.00000003", "surf.00000006"]
        contents[batched] = {f: read_grid_log(str(d / f))[1] for f in files if f.startswith("grid")}
        g.close()
    for f, rec in contents[False].items():
        other = contents[True][f]
        np.testing.assert_array_equal(rec["id"], other["id"])
        assert np.abs(rec["phi"] - other["phi"]).max() < 1e-6
