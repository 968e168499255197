"""tg_field_o1_noalloc (fixed device scratch, no allocation) against
tg_field_o1, both called through the C ABI on the same handle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NODES = 65536  # TG_FIELD_O1_NOALLOC_MAX


@pytest.fixture(scope="module")
def grid(small_mesh):
    from tapsim_modified_b200.tapsim import Grid
    g = Grid(small_mesh)
    g.solve(rel_tol=1e-10)
    g.surface_init(0)
    return g


def _fields(entry, handle, nodes):
    from tapsim_modified_b200 import _native as N
    nd = np.ascontiguousarray(nodes, np.int32)
    out = np.full((len(nd), 3), np.nan)
    rc = getattr(N.lib(), entry)(handle, len(nd), N.ptr(nd), N.ptr(out))
    assert rc == 0, N.lib().tg_last_error(handle)
    return out


def test_noalloc_matches_field_o1_twice(grid):
    surface, _ = grid.surface()
    n = grid.n
    # two calls in a row with different lists: the second must not see the
    # first one's nodes or results
    lists = [np.concatenate([surface, np.arange(0, n, 37)]).astype(np.int32),
             np.arange(n - 1, 0, -53, dtype=np.int32)]
    for nodes in lists:
        ref = _fields("tg_field_o1", grid._h, nodes)
        got = _fields("tg_field_o1_noalloc", grid._h, nodes)
        scale = np.abs(ref).max()
        assert scale > 0
        assert np.abs(got - ref).max() <= 1e-12 * scale


def test_noalloc_rejects_oversized_and_bad_input(grid):
    from tapsim_modified_b200 import _native as N
    lib = N.lib()
    big = np.zeros(MAX_NODES + 1, np.int32)
    out = np.zeros((MAX_NODES + 1, 3))
    assert lib.tg_field_o1_noalloc(grid._h, len(big), N.ptr(big), N.ptr(out)) == 1
    assert b"fixed scratch" in lib.tg_last_error(grid._h)
    bad = np.array([grid.n], np.int32)
    assert lib.tg_field_o1_noalloc(grid._h, 1, N.ptr(bad), N.ptr(out)) == 1
    # the largest allowed list still works afterwards
    nodes = np.arange(MAX_NODES, dtype=np.int32) % grid.n
    got = _fields("tg_field_o1_noalloc", grid._h, nodes)
    ref = _fields("tg_field_o1", grid._h, nodes)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
