"""The FP64 oracle against the reference TAPSim built from its own sources.

Golden data (tests/golden, made by make_golden.py) come from the reference:
its TetGen mesh and float couplings (dump), its potentials relaxed to the
float fixed point, and a 40-event evaporation with the "oracle" ini.  The
oracle runs on the reference's own mesh and couplings, relaxes to a relative
residual of 1e-12, and follows the reference's removal sequence.
"""
import numpy as np
import pytest

from conftest import QM_FE, free_mask


@pytest.fixture(scope="module")
def oracle_on_ref(ref_mesh):
    from oracle import Oracle
    a = ref_mesh.arrays()
    o = Oracle(a)
    sweeps, rel = o.solve(1e-12, 2_000_000, 1.9)
    assert sweeps > 0 and rel <= 1e-12
    return a, o


def test_initial_potentials_match_reference(oracle_on_ref, ref_phi0):
    a, o = oracle_on_ref
    free = free_mask(a)
    # the reference stops at its float fixed point: a few 1e-6 V from the
    # exact solution of the same linear system
    assert np.abs(o.phi - ref_phi0)[free].max() < 1e-5
    assert np.array_equal(o.phi[~free].astype(np.float32), ref_phi0[~free])


def test_reference_float_fixed_point_cannot_reach_1e8(oracle_on_ref, ref_phi0):
    """Why the device path defines its own criterion: the reference's float
    potentials have a relative residual far above 1e-8."""
    from oracle import Oracle
    a, _ = oracle_on_ref
    chk = Oracle(a)
    chk.phi[:] = ref_phi0
    assert chk.residual() > 1e-8


def test_event_sequence_fields_and_impacts_match_reference(ref_mesh, ref_events):
    from oracle import Oracle
    a = ref_mesh.arrays()
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    o.surface_init(0)
    for k, row in enumerate(ref_events):
        info, ratio = o.select()
        node = int(row[1])
        assert info.candidate == node, f"event {k + 1}: oracle {info.candidate}, reference {node}"
        # near-tie margin computed the same way (the reference's fields carry
        # ~2e-5 relative error from its float fixed point)
        assert abs((info.best - info.second) / info.best - row[6]) <= 1e-4
        E = o.field_o1(node)
        assert np.linalg.norm(E - row[8:11]) <= 1e-4 * np.linalg.norm(row[8:11])
        o.take_away(node, 0)
        o.solve(1e-11, 2_000_000, 1.9)
        if k < 10:
            imp = o.trace(a["xyz"][node], QM_FE, a["node_tet"][node])
            assert imp.status == int(row[24])
            d = np.hypot(imp.stop[0] - row[18], imp.stop[1] - row[19])
            assert d <= 1e-3 * np.hypot(row[18], row[19]) + 1e-11
            assert abs(imp.stop[2] - row[20]) <= 1e-6 * row[20]
            # potential after removal
            assert abs(o.phi[node] - row[11]) < 2e-5


def test_local_set_is_find_local_nodes_minus_dirichlet(ref_mesh):
    """orc_local_set follows find_localNodes (grid_3d.cpp:1284-1315): the
    shell-1 set holds the neighbours only, the start joins from shell 2 on,
    Dirichlet cells are dropped, and each shell contains the smaller one."""
    from oracle import Oracle
    a = ref_mesh.arrays()
    o = Oracle(a)
    types = a["types"]
    dirichlet = np.array([bool(types[int(t)]["dirichlet"]) for t in a["type"]])
    rp, col = a["row_ptr"], a["col"]
    node = int(np.nonzero(~dirichlet)[0][len(np.nonzero(~dirichlet)[0]) // 2])
    s1 = o.local_set(node, 1)
    nb = set(col[rp[node]:rp[node + 1]].tolist())
    assert set(s1.tolist()) == {j for j in nb if not dirichlet[j]}
    s2, s3 = o.local_set(node, 2), o.local_set(node, 3)
    assert node in set(s2.tolist()) and set(s1) <= set(s2) <= set(s3)
    assert not dirichlet[s3].any() and np.all(np.diff(s3) > 0)


def test_stagnation_rule_matches_the_reference_formula():
    """The slope test of relax(thr, cycle, queue): a flat history is a
    fault, a decreasing one is not, a short queue never is, and a queue of
    one never is either (its slope is 0 / 0, which is not equal to 0)."""
    from oracle import stagnated
    assert stagnated([1e-3, 1e-3, 1e-3], 3, 5)
    assert stagnated([0.0, 0.0, 0.0], 3, 2)
    assert not stagnated([3e-3, 2e-3, 1e-3], 3, 5)
    assert not stagnated([1e-3, 1e-3], 3, 5)
    assert not stagnated([0.5], 1, 5)
    # symmetric values around the mean cancel exactly
    assert stagnated([1.0, 2.0, 1.0], 3, 1)
