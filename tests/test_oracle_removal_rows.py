"""The rows a removal changes.  The device's first residual after removals
(k_residual_rows) recomputes only the flipped cells' rows and their
neighbours' and keeps every other row's residual and Dirichlet part from the
last full pass.  Here the FP64 oracle removes atoms (with detachment, on the
plain Fe tip and on one whose Cu solute is a free dielectric species), and
the per-row residual and Dirichlet part before and after each removal may
differ only on those rows.

The flights' vertex fields in event batches rest on a second premise, checked
the same way: the field of a Dirichlet cell among Dirichlet cells never
changes, and neither does the zero pattern of the couplings."""
import numpy as np
import pytest

from conftest import SMALL_TIP


def _rows(o):
    """Per-row residual and Dirichlet part of the oracle's state, as
    orc_residual sums them (0 on Dirichlet rows)."""
    n = o.n
    rp, col = o.row_ptr, o.col
    row = np.repeat(np.arange(n), np.diff(rp))
    neu = np.array([o.types[int(t)].neumann for t in o.type], bool)
    dir_ = np.array([o.types[int(t)].dirichlet for t in o.type], bool)
    w = np.where(~neu[row] & neu[col], 0.0, o.c)
    s = np.bincount(row, weights=w * o.phi[col], minlength=n)
    d = np.bincount(row, weights=w, minlength=n)
    b = np.bincount(row, weights=np.where(dir_[col], w * o.phi[col], 0.0), minlength=n)
    r = s - d * o.phi - o.q
    b = b - o.q
    r[dir_] = 0.0
    b[dir_] = 0.0
    return r, b


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
def test_removals_change_only_flipped_rows_and_neighbours(kind, tmp_path):
    from oracle import Oracle
    o = Oracle(_mesh(kind, tmp_path).arrays())
    o.solve(1e-10, 2_000_000, 1.9)
    o.surface_init(0)
    changed_total = 0
    for k in range(12):
        info, _ = o.select()
        r0, b0 = _rows(o)
        detached = o.take_away(info.candidate, 0)
        r1, b1 = _rows(o)
        flipped = [info.candidate] + list(detached)
        touched = set(flipped)
        for f in flipped:
            touched.update(o.col[o.row_ptr[f]:o.row_ptr[f + 1]].tolist())
        changed = set(np.nonzero((r1 != r0) | (b1 != b0))[0].tolist())
        assert changed <= touched, (k, sorted(changed - touched)[:10])
        changed_total += len(changed)
        # relax so that the next removal starts from a converged state again
        o.solve(1e-10, 2_000_000, 1.9)
    assert changed_total > 12


@pytest.mark.parametrize("kind", ["fe", "dielectric"])
def test_fields_outside_the_listed_cells_never_change(kind, tmp_path):
    """The flights' vertex fields in event batches are recomputed only for the
    cells that are free or have a free neighbour, a list that removals grow
    by the flipped cells and their neighbours.  The field of every cell left
    off the list must keep its first value, and the zero pattern of the
    couplings (all the fields read of them) must not change."""
    from oracle import Oracle
    o = Oracle(_mesh(kind, tmp_path).arrays())
    o.solve(1e-10, 2_000_000, 1.9)
    o.surface_init(0)
    n = o.n
    row = np.repeat(np.arange(n), np.diff(o.row_ptr))
    free = ~np.array([o.types[int(t)].dirichlet for t in o.type], bool)
    active = free | (np.bincount(row, weights=free[o.col].astype(float), minlength=n) > 0)
    off = np.nonzero(~active)[0]
    assert off.size > 0
    first = {int(i): o.field_o1(int(i)).copy() for i in off}
    pattern = o.c == 0.0
    for k in range(12):
        info, _ = o.select()
        flipped = [info.candidate] + list(o.take_away(info.candidate, 0))
        for f in flipped:
            active[f] = True
            active[o.col[o.row_ptr[f]:o.row_ptr[f + 1]]] = True
        o.solve(1e-10, 2_000_000, 1.9)
        assert np.array_equal(o.c == 0.0, pattern), k
    still = [i for i in first if not active[i]]
    assert len(still) > 0.5 * len(first)
    for i in still:
        assert np.array_equal(o.field_o1(i), first[i]), i
