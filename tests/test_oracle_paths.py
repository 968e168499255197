"""Recorded flight paths of the FP64 oracle against the reference's own
trajectory files (LogTrajectory output of the first 3 events of the golden
evaporation, tests/golden/ref_traj_bin.*).  The reference integrates in
float, the oracle in FP64, so their step sequences differ; the paths are
compared as curves, the error estimates by order of magnitude."""
import numpy as np
import pytest

from conftest import GOLDEN, QM_FE, path_deviation


@pytest.fixture(scope="module")
def oracle_paths(ref_mesh):
    from oracle import Oracle
    from tapsim_modified_b200.tapsim import read_trajectories
    # the binary files hold the same points at full float precision
    items = read_trajectories(str(GOLDEN / "ref_traj_bin.00000001"))[1] + \
        read_trajectories(str(GOLDEN / "ref_traj_bin.00000002"))[1]
    a = ref_mesh.arrays()
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    o.surface_init(0)
    out = []
    for it in items:
        info, _ = o.select()
        node = info.candidate
        o.take_away(node, 0)
        o.solve(1e-11, 2_000_000, 1.9)
        imp, path, err = o.trace_path(a["xyz"][node], np.zeros(3), QM_FE, a["node_tet"][node])
        out.append((node, imp, path, err, it))
    return a, out


def test_paths_follow_the_reference(oracle_paths):
    a, out = oracle_paths
    for node, imp, path, err, it in out:
        ref = it["points"]
        assert node + 1 == it["number"]
        assert imp.status == it["status"] == 5
        assert len(path) == imp.steps + 2
        # the start: the node, at rest, in its associated tetrahedron
        np.testing.assert_array_equal(path[0, 1:4].astype(np.float32), ref["position"][0])
        assert path[0, 7] == ref["tet"][0] and path[0, 0] == 0.0
        # the step that leaves the mesh and the extrapolated point are outside
        assert path[-1, 7] == path[-2, 7] == -1 and ref["tet"][-1] == ref["tet"][-2] == -1
        assert np.all(path[1:-2, 7] >= 0)
        assert abs(len(path) - len(ref)) <= 0.15 * len(ref)
        dev, disp = path_deviation(path[:, 0], path[:, 1:4], ref, it["time_scale"])
        assert dev <= 1e-3 * disp
        # the extrapolated impact
        np.testing.assert_allclose(path[-1, 1:3], ref["position"][-1][:2], rtol=1e-3, atol=1e-12)
        # cumulative error estimates: same order of magnitude
        ratio = err / it["error"].astype(np.float64)
        assert np.all((ratio > 0.1) & (ratio < 10.0)), ratio


def test_path_error_estimate_is_the_root_sum_of_squares(oracle_paths):
    """cumulative_error (trajectory_3d.cpp:683-700) in the oracle: the
    estimate grows monotonically with the path, so a truncated run's
    estimate (fewer steps) is not above the full one's."""
    from oracle import Oracle
    a, out = oracle_paths
    node, imp, path, err, it = out[0]
    o = Oracle(a)  # a fresh oracle: only the relation between the two runs matters
    o.solve(1e-12, 2_000_000, 1.9)
    full, p_full, e_full = o.trace_path(a["xyz"][node], np.zeros(3), QM_FE, a["node_tet"][node])
    part, p_part, e_part = o.trace_path(a["xyz"][node], np.zeros(3), QM_FE, a["node_tet"][node], max_steps=20)
    assert part.status == 3 and part.steps == 20 and len(p_part) == 22
    np.testing.assert_array_equal(p_part[:21], p_full[:21])
    assert np.all(e_part[3:] <= e_full[3:])
