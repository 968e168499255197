"""The sample mesher (tg_mesh_from_sample), MeshGen's role for an arbitrary
sample (meshgen/meshgen.cpp:2506-3986): the specimen atoms of a generated
tip, written out as a sample node file (meshgen's readSample input,
:197-360), are meshed again with their own vacuum cascade.  CPU tests check
the node layout against meshgen's (boundary markers :3855-3892, the sample
appended last :3908, numbering as readGeomGrid gives it), determinism across
thread counts, the exclusion distance, and that the specimen's surface (its
atoms with a vacuum neighbour) is the tip mesh's; the GPU test compares the
relaxed fields at the apex with the tip mesh's."""
import numpy as np
import pytest

from conftest import SMALL_TIP

ATOM_IDS = (4, 5)
BOX = dict(box_half_width=SMALL_TIP["box_half_width"], box_height=SMALL_TIP["box_height"])


def write_sample(path, xyz, ids, numbers=None):
    """An ASCII node file (the layout meshgen reads): tab-separated x y z id
    [number] per line."""
    with open(path, "w") as f:
        f.write(f"ASCII {len(ids)} {0 if numbers is None else 1} 0\n")
        for k in range(len(ids)):
            row = [repr(float(np.float32(c))) for c in xyz[k]] + [str(int(ids[k]))]
            if numbers is not None:
                row.append(str(int(numbers[k])))
            f.write("\t".join(row) + "\n")


@pytest.fixture(scope="module")
def tip_and_sample(tmp_path_factory):
    from tapsim_modified_b200.tapsim import Mesh
    tip = Mesh.from_tip(**SMALL_TIP)
    a = tip.arrays()
    atoms = np.isin(a["type"], ATOM_IDS)
    d = tmp_path_factory.mktemp("sample")
    path = d / "sample.txt"
    numbers = 1000 + 3 * np.arange(int(atoms.sum()))
    write_sample(path, a["xyz"][atoms], a["type"][atoms], numbers)
    cfg = d / "tip.cfg"
    tip.write_config(str(cfg))
    return tip, a, atoms, path, numbers, cfg


def sample_mesh(path, cfg=None, threads=0):
    from tapsim_modified_b200.tapsim import Mesh
    return Mesh.from_sample(str(path), str(cfg) if cfg else None, threads=threads,
                            fine_shell=SMALL_TIP["fine_shell"], seed=3, **BOX)


def test_layout_markers_and_numbers(tip_and_sample):
    tip, a, atoms, path, numbers, _ = tip_and_sample
    m = sample_mesh(path)
    b = m.arrays()
    n_s = int(atoms.sum())
    # the sample last, unchanged
    assert np.array_equal(b["xyz"][-n_s:], a["xyz"][atoms])
    assert np.array_equal(b["type"][-n_s:], a["type"][atoms])
    gen = b["type"][:-n_s]
    assert set(np.unique(gen).tolist()) == {0, 1, 2, 3}
    xyz = b["xyz"][:-n_s].astype(np.float64)
    W, H = BOX["box_half_width"], BOX["box_height"]
    tol = 1e-6 * H
    top, bottom, sides = gen == 1, gen == 2, gen == 3
    assert np.all(np.abs(xyz[top, 2] - H) < tol)
    assert np.all(np.abs(xyz[bottom, 2]) < tol)
    on_side = (np.abs(np.abs(xyz[:, 0]) - W) < tol) | (np.abs(np.abs(xyz[:, 1]) - W) < tol)
    assert np.all(on_side[sides])
    # bottom and top nodes keep off the side faces (edges and corners are sides)
    assert not np.any(on_side[top | bottom])
    # vacuum inside the box
    vac = xyz[gen == 0]
    assert np.all(np.abs(vac[:, :2]) < W) and np.all((vac[:, 2] > 0) & (vac[:, 2] < H))
    # numbers: the sample keeps its own, the generated nodes count on from the largest
    num = m.numbers()
    assert np.array_equal(num[-n_s:], numbers)
    assert np.array_equal(num[:-n_s], numbers.max() + 1 + np.arange(len(gen)))
    # meshgen's configuration template when no configuration is given
    t = b["types"]
    assert t[1]["dirichlet"] and t[3]["dirichlet"] and t[2]["neumann"] and not t[0]["dirichlet"]
    ids = np.unique(a["type"][atoms]).tolist()
    assert set(t) == {0, 1, 2, 3, *ids}
    assert all(t[i]["removable"] and t[i]["dirichlet"] and t[i]["phi"] == 1000.0 for i in ids)


def test_exclusion_and_spacing(tip_and_sample):
    from scipy.spatial import cKDTree
    _, a, atoms, path, _, _ = tip_and_sample
    b = sample_mesh(path).arrays()
    n_s = int(atoms.sum())
    sample = b["xyz"][-n_s:].astype(np.float64)
    vac = b["xyz"][:-n_s][b["type"][:-n_s] == 0].astype(np.float64)
    tree = cKDTree(sample)
    h0 = np.median(tree.query(sample, k=2)[0][:, 1])
    dv = tree.query(vac)[0]
    assert dv.min() >= 0.8 * h0 * (1 - 1e-6)
    # the fine shell holds the lattice's own vacuum sites, a nearest-neighbour
    # distance off the surface atoms (within their 1% jitter)
    near = dv[dv <= SMALL_TIP["fine_shell"]]
    assert len(near) > 200
    assert np.sum(np.abs(dv - h0) < 0.02 * h0) > 100


def test_deterministic_across_threads(tip_and_sample):
    _, _, _, path, _, _ = tip_and_sample
    m1, m4 = sample_mesh(path, threads=1), sample_mesh(path, threads=4)
    a1, a4 = m1.arrays(), m4.arrays()
    for k in ("xyz", "type", "row_ptr", "col", "coupling"):
        assert np.array_equal(a1[k], a4[k]), k


def test_surface_atoms_match_the_tip_mesh(tip_and_sample):
    """The specimen's surface (atoms with a vacuum neighbour in the mesh) is
    the same set in the tip mesh and in the sample's own vacuum cascade: both
    continue the bcc lattice into the vacuum around it."""
    _, a, atoms, path, _, cfg = tip_and_sample
    b = sample_mesh(path, cfg).arrays()

    def surface(arr):
        t = arr["type"]
        rows = np.repeat(np.arange(len(t)), np.diff(arr["row_ptr"]))
        hit = np.isin(t[rows], ATOM_IDS) & (t[arr["col"]] == 0)
        return np.unique(rows[hit])

    n_s = int(atoms.sum())
    s_tip = np.flatnonzero(atoms)
    tip_surf = np.searchsorted(s_tip, surface(a))
    smp_surf = surface(b) - (len(b["type"]) - n_s)
    assert len(tip_surf) > 100
    assert np.array_equal(tip_surf, smp_surf)


def test_errors(tmp_path):
    from tapsim_modified_b200.tapsim import Mesh
    below = tmp_path / "below.txt"
    write_sample(below, np.array([[0.0, 0.0, -1e-10], [2.5e-10, 0.0, 1e-10]]), np.array([4, 4]))
    with pytest.raises(Exception, match="above the bottom plane"):
        Mesh.from_sample(str(below), **BOX)
    wide = tmp_path / "wide.txt"
    write_sample(wide, np.array([[0.0, 0.0, 1e-9], [9.9e-9, 0.0, 1e-9]]), np.array([4, 4]))
    with pytest.raises(Exception, match="do not fit"):
        Mesh.from_sample(str(wide), **BOX)
    marker = tmp_path / "marker.txt"
    write_sample(marker, np.array([[0.0, 0.0, 1e-9], [2.5e-10, 0.0, 1e-9]]), np.array([4, 1]))
    with pytest.raises(Exception, match="marker"):
        Mesh.from_sample(str(marker), **BOX)


@pytest.mark.gpu
def test_apex_fields_match_the_tip_mesh(tip_and_sample):
    """Relaxed to 1e-10, the fields of the apex atoms on the sample's own
    vacuum mesh agree with the tip mesh's: both discretise the same
    specimen, so they differ only by their vacuum points."""
    from tapsim_modified_b200.tapsim import Grid
    tip, a, atoms, path, _, cfg = tip_and_sample
    m = sample_mesh(path, cfg)
    b = m.arrays()
    n_s = int(atoms.sum())
    s_tip = np.flatnonzero(atoms)
    z = a["xyz"][s_tip, 2]
    apex = np.argsort(-z)[:20]                       # the 20 highest atoms, by sample index
    fields = []
    for mesh, idx in ((tip, s_tip[apex]), (m, len(b["type"]) - n_s + apex)):
        g = Grid(mesh)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
        fields.append(np.linalg.norm(g.field_o1(idx.astype(np.int32)), axis=1))
        g.close()
    rel = np.abs(fields[1] - fields[0]) / fields[0]
    print("apex field magnitudes (tip mesh)", fields[0][:5], "relative differences: median", np.median(rel),
          "max", rel.max())
    assert np.median(rel) <= 0.05 and rel.max() <= 0.15


def test_host_program_meshgen(tip_and_sample, tmp_path):
    """`tapsim_b200 meshgen isample onodes` (meshgen's command line) writes the
    node file and the configuration template of the same mesh that
    tg_mesh_from_sample builds, and the evaporation path reads them back
    (tg_mesh_from_files) to the same nodes."""
    import subprocess

    from conftest import ROOT
    from tapsim_modified_b200.tapsim import Mesh
    program = ROOT / "tapsim_modified_b200" / "tapsim_b200"
    if not program.exists():
        pytest.skip("the host program is built by __graft_entry__.build()")
    _, _, _, path, _, _ = tip_and_sample
    nodes, cfg = tmp_path / "mesh.nodes", tmp_path / "mesh.cfg"
    r = subprocess.run([str(program), f"--box-half-width={BOX['box_half_width']}", f"--box-height={BOX['box_height']}",
                        f"--fine-shell={SMALL_TIP['fine_shell']}", f"--create-config-template={cfg}", "meshgen",
                        str(path), str(nodes)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "meshgen:" in r.stdout
    direct = Mesh.from_sample(str(path), fine_shell=SMALL_TIP["fine_shell"], **BOX).arrays()
    back = Mesh.from_files(str(nodes), str(cfg)).arrays()
    for k in ("xyz", "type", "row_ptr", "col"):
        assert np.array_equal(direct[k], back[k]), k
    assert back["types"].keys() == direct["types"].keys()


@pytest.mark.gpu
def test_events_run_on_the_sample_mesh(tip_and_sample):
    """The event loop on the sample's own vacuum mesh: every event removes a
    surface atom of the specimen, relaxes to the tolerance and sends its ion
    to the detector, and its first removals are the tip mesh's first ones
    (the same specimen, the same surface; measured: the same eight atoms,
    one of them taken earlier)."""
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    from conftest import GOLDEN
    tip, a, atoms, path, _, cfg = tip_and_sample
    m = sample_mesh(path, cfg)
    b = m.arrays()
    n_s = int(atoms.sum())
    first = len(b["type"]) - n_s
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    sopts = solve_opts(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
    removed = {}
    for name, mesh, offset in (("tip", tip, None), ("sample", m, first)):
        g = Grid(mesh)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1)
        recs = Evaporation(g, opts, relax_mode=1, solve=sopts).run(8)
        g.close()
        assert all(r["status"] == 5 and r["rel_residual"] <= 1e-10 for r in recs), name
        if offset is None:
            s_tip = np.flatnonzero(atoms)
            removed[name] = [int(np.searchsorted(s_tip, r["node"])) for r in recs]
        else:
            assert all(r["node"] >= offset for r in recs)       # a specimen atom
            removed[name] = [r["node"] - offset for r in recs]
    print("first removals (sample index): tip mesh", removed["tip"], "sample mesh", removed["sample"])
    assert len(set(removed["tip"]) & set(removed["sample"])) >= 6
