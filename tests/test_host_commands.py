"""The host program's command line (tapsim_b200, csrc/host/tapsim_b200.cpp):
its make-ini and relaxation modes against the reference's own `tapsim
make-ini` and `tapsim relaxation` outputs (tests/golden/make_golden.py
--commands; tapsim.cpp:66-148, commands.cpp:55-277), the reference's
evaporation and resumption options (commands.cpp:280-841), and the dump's
event index a resumption counts on from."""
import gzip
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

PROGRAM = ROOT / "tapsim_modified_b200" / "tapsim_b200"


def run(args, cwd, timeout=600):
    if not PROGRAM.exists():
        pytest.skip("the host program is built by __graft_entry__.build()")
    return subprocess.run([str(PROGRAM), *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=timeout)


def test_make_ini_writes_the_reference_defaults(tmp_path):
    """make-ini without a name writes tapsim.ini in the working directory,
    with one the named file; both byte for byte the reference's."""
    ref = (GOLDEN / "ref_tapsim.ini").read_bytes()
    r = run(["make-ini"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "tapsim.ini").read_bytes() == ref
    r = run(["make-ini", tmp_path / "other.ini"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "other.ini").read_bytes() == ref


def test_reference_defaults_are_the_python_hosts():
    """The Python host's defaults are the reference's make-ini values."""
    from tapsim_modified_b200.tapsim import INI_DEFAULTS, read_ini
    assert read_ini(str(GOLDEN / "ref_tapsim.ini")) == INI_DEFAULTS


@pytest.mark.parametrize("args", [["relaxation"], ["relaxation", "a.cfg"], ["relaxation", "--read-dump=x", "a.cfg"],
                                  ["relaxation", "a.cfg", "b", "c", "d"], ["make-ini", "a.ini", "b.ini"],
                                  ["relax"], ["make-ini", "--bogus"]])
def test_command_line_errors(args, tmp_path):
    r = run(args, tmp_path)
    assert r.returncode == 1
    assert r.stderr.startswith("tapsim_b200: ")


def test_relaxation_reads_files_before_the_device(tmp_path):
    """A missing input fails while the mesh is read, before any device call."""
    r = run(["relaxation", tmp_path / "none.cfg", tmp_path / "none.nodes"], tmp_path)
    assert r.returncode == 1
    assert "reading the mesh" in r.stderr


def read_node_lines(text):
    lines = text.splitlines()
    return lines[0], [ln.split("\t") for ln in lines[1:]]


def test_grid_node_writer_matches_the_reference(golden_dump, tmp_path):
    """tg_mesh_write_grid_nodes (File_Io::writeGeomGrid with numbers and
    potentials) writes the reference's relaxed node file byte for byte when
    given the reference's potentials on the reference's own mesh."""
    from tapsim_modified_b200.tapsim import Mesh
    text = gzip.open(GOLDEN / "ref_relaxed_nodes.txt.gz").read().decode()
    _, rows = read_node_lines(text)
    phi = np.array([float(x[5]) for x in rows], np.float32)
    Mesh.from_dump(str(golden_dump), None).write_grid_nodes(str(tmp_path / "nodes.txt"), phi)
    assert (tmp_path / "nodes.txt").read_text() == text


@pytest.mark.gpu
def test_relaxation_matches_the_reference(golden_dump, ref_mesh, ref_phi0, tmp_path):
    """relaxation --read-dump=? oconfig onode --write-dump=?: the node file has
    the reference's layout (header, coordinates, ids and numbers, text for
    text) and its potentials are the reference's float fixed point within
    2e-5 V; the configuration and the dump written beside it read back to
    the same potentials.  --relax-mode=reference (Grid_3d::Table::relax with
    the given threshold) ends within 1e-4 V of it."""
    from tapsim_modified_b200.tapsim import Mesh
    head_ref, rows_ref = read_node_lines(gzip.open(GOLDEN / "ref_relaxed_nodes.txt.gz").read().decode())
    a = ref_mesh.arrays()
    free = np.array([not a["types"][int(t)]["dirichlet"] for t in a["type"]])
    cfg, nodes, dump = tmp_path / "out.cfg", tmp_path / "out.nodes", tmp_path / "out.dump"
    r = run(["--rel-tol=1e-10", f"--write-dump={dump}", "relaxation", f"--read-dump={golden_dump}", cfg, nodes], tmp_path)
    assert r.returncode == 0, r.stderr
    head, rows = read_node_lines(nodes.read_text())
    assert head == head_ref == f"ASCII {len(rows_ref)} 1 1"
    assert len(rows) == len(rows_ref)
    assert all(x[:5] == y[:5] for x, y in zip(rows, rows_ref))
    phi = np.array([float(x[5]) for x in rows])
    phi_ref = np.array([float(x[5]) for x in rows_ref])
    assert np.abs(phi_ref - ref_phi0).max() < 1e-6  # the fixture is the reference's initial relaxation
    assert np.abs(phi - phi_ref)[free].max() < 2e-5
    assert np.array_equal(phi[~free], phi_ref[~free])
    back = Mesh.from_dump(str(dump), str(cfg)).arrays()
    assert np.allclose(back["phi"], phi, rtol=1e-7, atol=1e-12)
    # the reference's own rule, stopped at a deviation of 1e-8 V per sweep
    nodes2 = tmp_path / "ref_mode.nodes"
    r = run(["--relax-mode=reference", "--threshold=1e-8", "--cycle-size=100", "--queue-size=25", "relaxation",
             f"--read-dump={golden_dump}", tmp_path / "out2.cfg", nodes2], tmp_path)
    assert r.returncode == 0, r.stderr
    _, rows2 = read_node_lines(nodes2.read_text())
    phi2 = np.array([float(x[5]) for x in rows2])
    assert np.abs(phi2 - phi_ref)[free].max() < 1e-4


@pytest.mark.parametrize("opt", ["--write-trajectories=t", "--write-grids=g", "--write-surfaces=s",
                                 "--snapshot-interval=5", "--dump-interval=5"])
def test_evaporation_refuses_outputs_it_does_not_write(opt, tmp_path):
    r = run([opt, "evaporation", tmp_path / "a.cfg", tmp_path / "a.nodes"], tmp_path)
    assert r.returncode == 1
    assert "results file only" in r.stderr


def test_evaporation_takes_the_reference_options(tmp_path):
    """Every evaporation/resumption option of the reference parses; the run
    then fails where the mesh is read (before any device call)."""
    opts = ["--skip-relaxation", "--init-potentials", "--reset-potentials", "--threshold=0", "--cycle-size=100",
            "--queue-size=25", "--no-trajectories", "--no-grids", "--no-surfaces", "--no-dump", "--no-chunks",
            "--chunk-size=10", "--vacuum-identifier=Vacuum", "--trajectory-error-threshold=1e-6",
            "--shrink-limit=1e-9", "--event-limit=5", "--voltage-queue-limit=250", "--voltage-queue-size=250",
            "--evap-threshold=1e-2", "--evap-shell-size=3", "--evap-cycle-size=5", "--evap-queue-size=5",
            "--evap-global-cycles=1", "--refresh-interval=0", "--refresh-threshold=0", "--refresh-cycle-size=100",
            "--refresh-queue-size=25", "--last-event=3", "--write-ascii", "--write-binary", "--no-file-output",
            "--threads=2"]
    r = run([*opts, "evaporation", tmp_path / "none.cfg", tmp_path / "none.nodes"], tmp_path)
    assert r.returncode == 1
    assert "reading the mesh" in r.stderr, r.stderr
    r = run(["--write-dump=d", "evaporation", tmp_path / "none.cfg", tmp_path / "none.nodes"], tmp_path)
    assert r.returncode == 1 and "--write-dump" in r.stderr


def test_dump_index_is_kept(golden_dump, tmp_path):
    """A dump's LAST_INDEX reads into the mesh (a resumption numbers its
    events on from it) and is written back with the dump."""
    from tapsim_modified_b200.tapsim import Mesh
    data = golden_dump.read_bytes()
    assert data.startswith(b"TAPSIM DUMP INFORMATION\nLAST_INDEX 0\n")
    src = tmp_path / "indexed.dump"
    src.write_bytes(data.replace(b"LAST_INDEX 0\n", b"LAST_INDEX 37\n", 1))
    assert Mesh.from_dump(str(golden_dump), None).dump_index == 0
    m = Mesh.from_dump(str(src), None)
    assert m.dump_index == 37
    m.write_dump(str(tmp_path / "back.dump"))
    assert Mesh.from_dump(str(tmp_path / "back.dump"), None).dump_index == 37
