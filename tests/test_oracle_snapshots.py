"""The FP64 oracle against the reference's grid and surface snapshots
(LogGrid / LogSurface output after the first golden event with Fe's
permittivity 5, so that the dielectric force Grid_3d::Table::force is not
zero).  The reference's potentials sit at its float fixed point, a few 1e-6 V
from the exact solution."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def oracle_after_event(ref_mesh_eps5):
    from oracle import Oracle
    a = ref_mesh_eps5.arrays()
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    o.surface_init(0)
    info, _ = o.select()
    o.take_away(info.candidate, 0)
    o.solve(1e-11, 2_000_000, 1.9)
    return a, o, info.candidate


def test_grid_snapshot_matches_reference(oracle_after_event, snapshot_files):
    from tapsim_modified_b200.tapsim import read_grid_log
    a, o, node = oracle_after_event
    _, g = read_grid_log(snapshot_files["ref_grid_bin"])
    assert g["id"][node] == 0  # the removed atom is vacuum now
    assert np.abs(o.phi - g["phi"]).max() < 1e-5
    E = np.array([o.field_o1(i) for i in range(len(g))])
    assert np.abs(E - g["field"]).max() <= 1e-4 * np.abs(g["field"]).max()
    F = np.array([o.force(i) for i in range(len(g))])
    scale = np.abs(g["force"]).max()
    assert scale > 0 and (np.abs(g["force"]).max(axis=1) > 0).sum() > 1000
    assert np.abs(F - g["force"]).max() <= 1e-3 * scale
    # zero exactly where the permittivities of a cell and all its neighbours agree
    np.testing.assert_array_equal(F == 0.0, g["force"] == 0.0)


def test_surface_snapshot_matches_reference(oracle_after_event, snapshot_files):
    from tapsim_modified_b200.tapsim import read_surface_log
    a, o, node = oracle_after_event
    _, cells, nodes = read_surface_log(snapshot_files["ref_surf_bin"])
    info, ratio = o.select()
    np.testing.assert_array_equal(np.flatnonzero(o.surface), cells["index"])
    prob = ratio[cells["index"]] / ratio[cells["index"]].sum()
    np.testing.assert_allclose(prob, cells["probability"], rtol=2e-4)
    # neighbour lists are the cells' Delaunay rows
    rp, col = a["row_ptr"], a["col"]
    for c, nb in zip(cells["index"], cells["neighbours"]):
        np.testing.assert_array_equal(nb, col[rp[c]:rp[c + 1]])
    want = np.unique(np.concatenate([cells["index"]] + list(cells["neighbours"])))
    np.testing.assert_array_equal(nodes["index"], want)
    assert np.abs(o.phi[nodes["index"]] - nodes["phi"]).max() < 1e-5
    on_surface = np.isin(nodes["index"], cells["index"])
    assert np.all(nodes["normal"][~on_surface] == 0.0)
    assert np.allclose(np.linalg.norm(nodes["normal"][on_surface], axis=1), 1.0, atol=1e-5)
