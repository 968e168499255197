"""Removals of a dielectric species: Cu solute atoms with permittivity 5 that
are free cells (not Dirichlet) inside the Fe tip.  Their rows stay in the
inner system when they are removed, so the device must re-copy the couplings
the flip changed (k_vsys_refresh); the removal sequence, the potentials and
the solver's convergence are checked against the FP64 oracle, with both
preconditioners."""
import numpy as np
import pytest

from conftest import SMALL_TIP

pytestmark = pytest.mark.gpu

EVENTS = 12
NEAR_TIE = 1e-4


@pytest.fixture(scope="module")
def dielectric_mesh(tmp_path_factory):
    from tapsim_modified_b200.tapsim import Mesh
    d = tmp_path_factory.mktemp("dielectric")
    m = Mesh.from_tip(**dict(SMALL_TIP, solute_fraction=0.3))
    m.write_node_file(str(d / "t.nodes"))
    m.write_config(str(d / "t.cfg"))
    head, cu = (d / "t.cfg").read_text().split("NAME = Cu\n", 1)
    assert "DIRICHLET_BOUNDARY = 1\n" in cu and "DIELECTRICITY = 1\n" in cu
    cu = cu.replace("DIELECTRICITY = 1\n", "DIELECTRICITY = 5\n", 1)
    cu = cu.replace("DIRICHLET_BOUNDARY = 1\n", "DIRICHLET_BOUNDARY = 0\n", 1)
    (d / "d.cfg").write_text(head + "NAME = Cu\n" + cu)
    return Mesh.from_files(str(d / "t.nodes"), str(d / "d.cfg"))


@pytest.fixture(scope="module")
def oracle_sequence(dielectric_mesh):
    from oracle import Oracle
    a = dielectric_mesh.arrays()
    o = Oracle(a)
    o.solve(1e-12, 2_000_000, 1.9)
    o.surface_init(0)
    seq, margins, phis = [], [], []
    for _ in range(EVENTS):
        info, _ = o.select()
        seq.append(info.candidate)
        margins.append((info.best - info.second) / info.best)
        o.take_away(info.candidate, 0)
        o.solve(1e-12, 2_000_000, 1.9)
        phis.append(o.phi.copy())
    return a, seq, margins, phis


@pytest.mark.parametrize("preconditioner", [0, 1])
def test_dielectric_removals_match_oracle(dielectric_mesh, oracle_sequence, preconditioner):
    from tapsim_modified_b200.tapsim import Grid
    a, seq, margins, phis = oracle_sequence
    cu = 5
    assert sum(int(a["type"][n]) == cu for n in seq) >= 6  # mostly free cells removed
    g = Grid(dielectric_mesh)
    g.solve(rel_tol=1e-11, max_outer=50, max_inner=20000, preconditioner=preconditioner)
    g.surface_init(0)
    for k, node in enumerate(seq):
        sel = g.select()
        if sel.candidate != node:
            assert margins[k] < NEAR_TIE, f"event {k + 1}: {sel.candidate} vs {node}"
            break
        g.take_away(node)
        info = g.solve(rel_tol=1e-11, max_outer=50, max_inner=20000, warm_start=1, preconditioner=preconditioner)
        # the inner system follows the flips, so one or two outer steps do
        assert info.rel_residual <= 1e-11 and info.outer <= 3, (k, info.outer)
        assert np.abs(g.potentials() - phis[k]).max() <= 1e-8
    g.close()
