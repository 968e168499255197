"""Byte-compatible file formats: node file, configuration, ini, dump, results."""
import struct

import numpy as np
import pytest

from conftest import GOLDEN


def test_node_file_roundtrip(tmp_path, small_mesh):
    from tapsim_modified_b200.tapsim import Mesh
    a = small_mesh.arrays()
    for binary in (True, False):
        p = tmp_path / f"n{int(binary)}.nodes"
        small_mesh.write_node_file(str(p), binary=binary)
        small_mesh.write_config(str(tmp_path / "c.cfg"))
        m2 = Mesh.from_files(str(p), str(tmp_path / "c.cfg"))
        b = m2.arrays()
        assert np.array_equal(a["type"], b["type"])
        if binary:
            assert np.array_equal(a["xyz"], b["xyz"])
        else:
            assert np.allclose(a["xyz"], b["xyz"], rtol=1e-8, atol=0)


def test_binary_node_file_layout(tmp_path, small_mesh):
    p = tmp_path / "x.nodes"
    small_mesh.write_node_file(str(p), binary=True)
    raw = p.read_bytes()
    header, body = raw.split(b"\n", 1)
    assert header == f"BINARY {small_mesh.num_nodes} 0 0".encode()
    rec = np.frombuffer(body, dtype=[("xyz", "<f4", 3), ("id", "<i2")])
    assert len(rec) == small_mesh.num_nodes


def test_config_written_by_reference_layout_reads_back(tmp_path):
    from tapsim_modified_b200.tapsim import Mesh
    m = Mesh.from_files(str(GOLDEN / "tip.nodes"), str(GOLDEN / "tip.cfg"))
    types = m.arrays()["types"]
    assert types[4]["evap_field"] == pytest.approx(33e9)
    assert types[4]["dirichlet"] == 1 and types[2]["neumann"] == 1 and types[3]["neumann"] == 1
    assert types[1]["dirichlet"] == 1 and types[1]["phi"] == 0.0


def test_dump_roundtrip(tmp_path, small_mesh):
    from tapsim_modified_b200.tapsim import Mesh
    a = small_mesh.arrays()
    p = tmp_path / "d.dump"
    small_mesh.write_dump(str(p))
    b = Mesh.from_dump(str(p)).arrays()
    assert np.array_equal(a["xyz"], b["xyz"])
    assert np.array_equal(a["type"], b["type"])
    assert np.array_equal(a["tet_v"], b["tet_v"])
    assert np.array_equal(a["tet_n"], b["tet_n"])
    assert np.array_equal(a["col"], b["col"])
    assert np.array_equal(a["coupling"].astype(np.float32), b["coupling"].astype(np.float32))
    assert np.array_equal(a["phi"], b["phi"])


def test_reference_dump_reads(ref_mesh):
    a = ref_mesh.arrays()
    assert len(a["type"]) == 9110
    assert (a["type"] == 4).sum() > 1000
    # ascending neighbour lists as std::set leaves them
    rp, col = a["row_ptr"], a["col"]
    assert all(np.all(np.diff(col[rp[i]:rp[i + 1]]) > 0) for i in range(0, len(rp) - 1, 37))


def test_ini_strict_keys(tmp_path):
    from tapsim_modified_b200.tapsim import INI_DEFAULTS, EvaporationOptions
    o = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    assert o.i("REFRESH_RELAXATION_INTERVAL") == 1
    assert o.i("GEOMETRY_CONTENTS") == 0xFF
    bad = tmp_path / "bad.ini"
    bad.write_text("".join(f"{k} = {v}\n" for k, v in INI_DEFAULTS.items() if k != "VOLTAGE_QUEUE_SIZE"))
    with pytest.raises(ValueError, match="VOLTAGE_QUEUE_SIZE"):
        EvaporationOptions.from_ini(str(bad))
    dup = tmp_path / "dup.ini"
    dup.write_text("A = 1\nA = 2\n")
    with pytest.raises(ValueError):
        EvaporationOptions.from_ini(str(dup))


def test_results_writer_layout(tmp_path):
    from tapsim_modified_b200.tapsim import write_results
    xyz = np.array([[1e-9, 2e-9, 3e-9]], np.float32)
    rec = {"index": 1, "node": 0, "id": 4, "number": 1, "voltage": 1.5, "stop": (1.0, 2.0, 3.0), "tof": 1e-9,
           "probability": 0.25, "potentialBefore": 1.0, "fieldBefore": (1.0, 2.0, 3.0), "potentialAfter": 0.9,
           "fieldAfter": (4.0, 5.0, 6.0), "normal": (0.0, 0.0, 1.0), "apex": (0.0, 0.0, 5e-9)}
    p = tmp_path / "r.bin"
    write_results(str(p), [rec], xyz, binary=True)
    raw = p.read_bytes()
    assert raw.startswith(b"TAPSIM RESULTS DATA\nVERSION 1.0\n")
    body = raw.split(b"BINARY\n", 1)[1]
    # 3 integers (4+2+4 bytes) and 23 floats per event (logResults.cpp:305-329)
    assert len(body) == 10 + 23 * 4
    idx, tid, num = struct.unpack_from("<IhI", body)
    assert (idx, tid, num) == (1, 4, 1)
    vals = struct.unpack_from("<23f", body, 10)
    assert vals[0] == 1.5 and vals[1] == pytest.approx(1e-9)
    p2 = tmp_path / "r.txt"
    write_results(str(p2), [rec], xyz, binary=False)
    line = p2.read_text().splitlines()[-1].split("\t")
    assert len(line) == 26 and line[0] == "1" and line[1] == "4"


def test_results_files_round_trip_the_reference_bytes():
    """Results written by the reference's own LogResults (tapsim resumption,
    ASCII in one file and binary in chunks of 4 events) are read and written
    back byte for byte, chunk file names included."""
    import os
    import tempfile
    from tapsim_modified_b200.tapsim import read_results, write_results_rows
    from conftest import GOLDEN
    header, rows = read_results(str(GOLDEN / "ref_results_ascii.txt"))
    assert len(rows) == 6 and rows[0][0] == 1 and header.startswith("# Generated by TAPSim")
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "r.txt")
        names = write_results_rows(out, rows, binary=False, header=header)
        assert open(names[0], "rb").read() == (GOLDEN / "ref_results_ascii.txt").read_bytes()
        h1, rows1 = read_results(str(GOLDEN / "ref_results_bin.00000001"))
        h2, rows2 = read_results(str(GOLDEN / "ref_results_bin.00000004"))
        assert [r[0] for r in rows1 + rows2] == [1, 2, 3, 4, 5, 6] and h2 == ""
        names = write_results_rows(os.path.join(td, "b"), rows1 + rows2, binary=True, header=h1, chunk_size=4)
        assert [os.path.basename(n) for n in names] == ["b.00000001", "b.00000004"]
        assert open(names[0], "rb").read() == (GOLDEN / "ref_results_bin.00000001").read_bytes()
        assert open(names[1], "rb").read() == (GOLDEN / "ref_results_bin.00000004").read_bytes()
    # the ASCII and binary runs are the same events
    assert [r[2] for r in rows] == [r[2] for r in rows1 + rows2]


def test_trajectory_files_round_trip_the_reference_bytes(tmp_path):
    """The reference's own LogTrajectory output (logTrajectory.cpp:137-300),
    ASCII in one file and binary in chunks of 2, read and written back byte
    for byte."""
    from tapsim_modified_b200.tapsim import read_trajectories, write_trajectory_items
    binary, items = read_trajectories(str(GOLDEN / "ref_traj_ascii.txt"))
    assert not binary and [it["index"] for it in items] == [1, 2, 3]
    assert [len(it["points"]) for it in items] == [273, 115, 120]
    names = write_trajectory_items(str(tmp_path / "a.txt"), items)
    assert open(names[0], "rb").read() == (GOLDEN / "ref_traj_ascii.txt").read_bytes()
    b1, items1 = read_trajectories(str(GOLDEN / "ref_traj_bin.00000001"))
    b2, items2 = read_trajectories(str(GOLDEN / "ref_traj_bin.00000002"))
    assert b1 and b2 and [it["index"] for it in items1 + items2] == [1, 2, 3]
    names = write_trajectory_items(str(tmp_path / "b"), items1 + items2, binary=True, chunk_size=2)
    assert [n.rsplit(".", 1)[1] for n in names] == ["00000001", "00000002"]
    assert open(names[0], "rb").read() == (GOLDEN / "ref_traj_bin.00000001").read_bytes()
    assert open(names[1], "rb").read() == (GOLDEN / "ref_traj_bin.00000002").read_bytes()
    # the binary points are the ASCII ones at full float precision
    for a, b in zip(items, items1 + items2):
        assert a["status"] == b["status"] and a["number"] == b["number"]
        np.testing.assert_array_equal(a["points"]["tet"], b["points"]["tet"])
        np.testing.assert_allclose(a["points"]["position"], b["points"]["position"], rtol=1e-6)


def test_reference_trajectory_structure():
    """Trajectory_3d's data in the reference's files: the start point at
    time 0 and rest, steps inside the mesh, the step that leaves it with
    tetrahedron -1, then the point extrapolated to the top of the box."""
    from tapsim_modified_b200.tapsim import read_trajectories
    _, items = read_trajectories(str(GOLDEN / "ref_traj_ascii.txt"))
    for it in items:
        p = it["points"]
        assert it["status"] == 5
        assert p["time"][0] == 0.0 and np.all(p["velocity"][0] == 0.0)
        assert np.all(p["tet"][1:-2] >= 0) and p["tet"][-2] == -1 and p["tet"][-1] == -1
        assert np.all(np.diff(p["time"]) > 0)
        # the extrapolated point keeps the last velocity and reaches the top
        np.testing.assert_array_equal(p["velocity"][-1], p["velocity"][-2])
        assert abs(p["position"][-1][2] - 4.0e-8) <= 1e-14


def test_snapshot_files_round_trip_the_reference_bytes(tmp_path, snapshot_files):
    """The reference's LogGrid and LogSurface output (ASCII, binary, with and
    without neighbour lists) read and written back by the library's native
    writers byte for byte."""
    from tapsim_modified_b200.tapsim import read_grid_log, read_surface_log, write_grid_log, write_surface_log
    for name in ("ref_grid_ascii", "ref_grid_bin"):
        binary, g = read_grid_log(snapshot_files[name])
        assert binary == name.endswith("bin") and len(g) == 9110
        write_grid_log(str(tmp_path / name), g["id"], g["number"], g["phi"], g["field"], g["force"], binary)
        assert (tmp_path / name).read_bytes() == open(snapshot_files[name], "rb").read()
    for name in ("ref_surf_ascii", "ref_surf_bin"):
        binary, cells, nodes = read_surface_log(snapshot_files[name])
        assert binary == name.endswith("bin") and len(cells["index"]) == 617 and len(nodes["index"]) == 1960
        assert (cells["neighbours"] is None) == (not binary)
        write_surface_log(str(tmp_path / name), cells, nodes, binary)
        assert (tmp_path / name).read_bytes() == open(snapshot_files[name], "rb").read()
    # the ASCII files carry the binary ones' values at 7 digits
    _, ga = read_grid_log(snapshot_files["ref_grid_ascii"])
    _, gb = read_grid_log(snapshot_files["ref_grid_bin"])
    np.testing.assert_array_equal(ga["number"], gb["number"])
    np.testing.assert_allclose(ga["force"], gb["force"], rtol=1e-6, atol=0)
