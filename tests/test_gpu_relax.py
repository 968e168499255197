"""Device relaxation vs the FP64 oracle (same mesh, same couplings)."""
import numpy as np
import pytest

from conftest import free_mask

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solved(small_mesh):
    from oracle import Oracle
    from tapsim_modified_b200.tapsim import Grid
    a = small_mesh.arrays()
    g = Grid(small_mesh)
    info = g.solve(rel_tol=1e-8)
    o = Oracle(a)
    sweeps, rel = o.solve(1e-12, 2_000_000, 1.9)
    assert sweeps >= 0
    return a, g, info, o


def test_solve_reaches_tolerance(solved):
    a, g, info, o = solved
    assert info.rel_residual <= 1e-8
    assert info.initial_rel_residual > 1e-3
    # the oracle's own residual evaluation of the device potentials
    from oracle import Oracle
    chk = Oracle(a)
    chk.phi[:] = g.potentials()
    assert chk.residual() <= 1.05e-8


def test_solve_matches_oracle_potentials(solved):
    a, g, info, o = solved
    phi = g.potentials()
    free = free_mask(a)
    # both solutions have a relative residual <= 1e-8; the potentials (0..1 V)
    # then agree to a few 1e-7 V on this mesh
    assert np.abs(phi - o.phi)[free].max() < 2e-6
    # Dirichlet cells are untouched
    assert np.array_equal(phi[~free], o.phi[~free])


def test_device_residual_matches_oracle(solved):
    a, g, info, o = solved
    from oracle import Oracle
    chk = Oracle(a)
    chk.phi[:] = g.potentials()
    assert abs(g.residual() - chk.residual()) <= 1e-3 * chk.residual() + 1e-15


def test_relax_threshold_converges_to_solution(small_mesh):
    from tapsim_modified_b200.tapsim import Grid
    from oracle import Oracle
    a = small_mesh.arrays()
    g = Grid(small_mesh)
    rc, it, dev = g.relax_threshold(1e-11, 100, 25, max_sweeps=200_000)
    assert rc == 0 and dev <= 1e-11
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    free = free_mask(a)
    assert np.abs(g.potentials() - o.phi)[free].max() < 1e-6


def test_relax_cycles_deviation_decreases(small_mesh):
    from tapsim_modified_b200.tapsim import Grid
    g = Grid(small_mesh)
    d1 = g.relax(5)
    d2 = g.relax(50)
    assert d2 < d1


def test_local_relax_keeps_dirichlet_and_converges(small_mesh):
    from tapsim_modified_b200.tapsim import Grid
    a = small_mesh.arrays()
    g = Grid(small_mesh)
    g.solve(rel_tol=1e-8)
    g.surface_init(0)
    s = g.select()
    g.take_away(s.candidate)
    before = g.potentials()
    rc, it, dev = g.local_relax(s.candidate, 3, 1e-6, 5, 5)
    after = g.potentials()
    assert rc in (0, 6) and it >= 5
    free = free_mask(a)
    free[s.candidate] = True
    changed = np.nonzero(after != before)[0]
    assert len(changed) > 0
    assert free[changed].all()
    # only cells within three hops of the removed atom move
    rp, col = a["row_ptr"], a["col"]
    ring = {s.candidate}
    frontier = {s.candidate}
    for _ in range(3):
        nxt = set()
        for u in frontier:
            nxt.update(col[rp[u]:rp[u + 1]].tolist())
        frontier = nxt - ring
        ring |= nxt
    assert set(changed.tolist()) <= ring


def test_fp64_inner_iterations_match_oracle_and_fp32(small_mesh, ref_mesh, ref_events):
    """inner_precision 1 (FP64 couplings, vectors and recurrences in the
    inner CG, FP32 V-cycle): the initial solve and six events solved to
    1e-10 agree with the oracle's potentials and with the FP32 inner solve,
    and remove the same cells as the reference.  Options it does not take
    are refused."""
    from oracle import Oracle
    from tapsim_modified_b200 import _native as N
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    a = small_mesh.arrays()
    g = Grid(small_mesh)
    info = g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1, inner_precision=1)
    assert info.rel_residual <= 1e-10
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    free = free_mask(a)
    assert np.abs(g.potentials() - o.phi)[free].max() < 1e-7
    with pytest.raises(N.TapsimError):
        g.solve(rel_tol=1e-8, preconditioner=0, inner_precision=1)
    with pytest.raises(N.TapsimError):
        g.solve(rel_tol=1e-8, preconditioner=1, warm_start=1, inner_precision=1)
    g.close()
    from conftest import GOLDEN
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    runs = {}
    for prec in (0, 1):
        g = Grid(ref_mesh)
        g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, preconditioner=1, inner_precision=prec)
        ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, max_outer=50, max_inner=20000,
                                                                   preconditioner=1, inner_precision=prec))
        runs[prec] = (ev.run(6), g.potentials())
        g.close()
    (r32, phi32), (r64, phi64) = runs[0], runs[1]
    assert [r["node"] for r in r32] == [r["node"] for r in r64] == [int(x) for x in ref_events[:6, 1]]
    assert all(r["rel_residual"] <= 1e-10 for r in r32 + r64)
    assert np.abs(phi32 - phi64).max() < 1e-8
    # detector impacts of the two solves' potentials (1e-10 apart in the
    # residual): the adaptive stepper's accept/reject decisions are
    # discontinuous in the field, so potentials 1e-8 V apart can take a
    # different step sequence, whose impact then differs at the stepper's
    # error tolerance (measured 1.6e-6 to 2e-3 of the impact radius)
    for x, y in zip(r32, r64):
        d = np.hypot(x["stop"][0] - y["stop"][0], x["stop"][1] - y["stop"][1])
        assert d <= 1e-2 * np.hypot(y["stop"][0], y["stop"][1])


def _five_cell_handle():
    """A hand-built system: one free cell coupled to four Dirichlet cells
    (two at 1 V, two at 0 V) and nothing else, so that one sweep puts it at
    its exact value (0.5 V) and every later sweep moves nothing."""
    import ctypes as C
    from tapsim_modified_b200 import _native as N
    xyz = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0]], np.float32) * 1e-9
    type_id = np.array([0, 1, 1, 2, 2], np.int8)
    hull = np.zeros(5, np.uint8)
    phi = np.array([0.0, 1.0, 1.0, 0.0, 0.0], np.float32)
    row_ptr = np.array([0, 4, 5, 6, 7, 8], np.int32)
    col = np.array([1, 2, 3, 4, 0, 0, 0, 0], np.int32)
    cpl = np.ones(8, np.float64)
    types = (N.tg_type * 3)()
    for k, (dirichlet, p) in enumerate(((0, 0.0), (1, 1.0), (1, 0.0))):
        types[k].id, types[k].epsilon, types[k].dirichlet, types[k].phi = k, 1.0, dirichlet, p
        types[k].removable = 0
    keep = (xyz, type_id, hull, phi, row_ptr, col, cpl, types)
    d = N.tg_mesh_desc(num_nodes=5, xyz=xyz.ctypes.data, type_id=type_id.ctypes.data, hull=hull.ctypes.data,
                       phi=phi.ctypes.data, row_ptr=row_ptr.ctypes.data, col=col.ctypes.data,
                       coupling=cpl.ctypes.data, num_tets=0, num_types=3, types=types)
    h = C.c_void_p()
    N.check(N.lib().tg_create(C.byref(d), C.byref(h)))
    return h, keep


def test_stagnation_fault_on_a_built_case():
    """The stagnation rule (grid_3d.cpp:625-654, RelaxationFault) fires, as
    TG_ERR_RELAX_FAULT, once a full queue of deviations is flat: with the
    threshold below any deviation the relaxation only ends that way.  The
    free cell is exact after the first sweep (couplings of 1, so 0.5 V is
    exact in FP64), so each cycle's deviation (its last sweep's largest
    change) is 0: the queue of 3 is flat at the third cycle, where the rule
    fires with two cycles of two sweeps counted (the count grows after the
    test, as in the reference).  The same for localRelax on the cell's
    shell-2 set."""
    import ctypes as C
    from oracle import stagnated
    from tapsim_modified_b200 import _native as N
    h, keep = _five_cell_handle()
    L = N.lib()
    it, dev = C.c_int64(), C.c_double()
    rc = L.tg_relax_threshold(h, -1.0, 2, 3, 1000, C.byref(it), C.byref(dev))
    assert rc == N.TG_ERR_RELAX_FAULT, rc
    assert it.value == 4 and dev.value == 0.0
    assert stagnated([0.0, 0.0, 0.0], 3, 2) and not stagnated([0.0, 0.0], 3, 2)
    phi = np.empty(5, np.float64)
    N.check(L.tg_get_phi(h, N.ptr(phi)), h)
    assert phi[0] == 0.5
    # localRelax from the free cell: its shell-2 set is the cell itself
    N.check(L.tg_set_phi(h, N.ptr(np.array([0.25, 1.0, 1.0, 0.0, 0.0]))), h)
    rc = L.tg_local_relax(h, 0, 2, -1.0, 2, 3, C.byref(it), C.byref(dev))
    assert rc == N.TG_ERR_RELAX_FAULT, rc
    assert it.value == 4 and dev.value == 0.0
    N.check(L.tg_get_phi(h, N.ptr(phi)), h)
    assert phi[0] == 0.5
    L.tg_destroy(h)


def test_local_relax_reaches_the_oracle_fixed_point(ref_mesh):
    """tg_local_relax after a removal, to a deviation of 1e-13 V, against the
    oracle's fixed point of localRelax on find_localNodes' set minus the
    Dirichlet cells (grid_3d.cpp:707-795, 1284-1315): the same potentials on
    the set, and no cell outside it moves.  The device sweeps in colour
    order and the reference in index order, but both converge to this one
    fixed point (the local Dirichlet problem)."""
    from oracle import Oracle
    from tapsim_modified_b200.tapsim import Grid
    a = ref_mesh.arrays()
    g = Grid(ref_mesh)
    g.solve(rel_tol=1e-10)
    g.surface_init(0)
    s = g.select()
    o = Oracle(a)
    o.phi[:] = g.potentials()
    o.surface_init(0)
    g.take_away(s.candidate)
    o.take_away(s.candidate, 0)
    before = g.potentials()
    for shell in (3, 5):
        g.set_potentials(before)
        o.phi[:] = before
        rc, it, dev = g.local_relax(s.candidate, shell, 1e-13, 5, 5)
        assert rc == 0 and dev <= 1e-13
        cells = o.local_set(s.candidate, shell)
        assert o.local_solve(cells, 1e-14, 200_000) > 0
        after = g.potentials()
        inside = np.zeros(len(after), bool)
        inside[cells] = True
        assert np.array_equal(after[~inside], before[~inside])
        assert np.abs(after[inside] - o.phi[inside]).max() < 1e-11
        print("shell", shell, "cells", len(cells), "sweeps", it,
              "max |dphi| vs oracle", np.abs(after[inside] - o.phi[inside]).max())
