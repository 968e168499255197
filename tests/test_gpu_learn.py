"""The learned near-field warm start: sample collection in the solver,
device forward/backward against the CPU oracle (oracle/mpnn.py), training,
and warm_start 2 in the event loop."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

EVENTS = 12


@pytest.fixture(scope="module")
def collected(ref_mesh):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Learner, solve_opts
    g = Grid(ref_mesh)
    g.solve(rel_tol=1e-10)
    L = Learner(hops=6, max_cells=4096, ell_width=64, seed=3)
    L.attach(g, collect=True)
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=1, preconditioner=1))
    recs = ev.run(EVENTS)
    L.attach(g)  # detach
    return g, L, recs


def test_one_sample_per_event(collected):
    g, L, recs = collected
    n, cells = L.samples()
    assert n == EVENTS
    s = L.sample(0)
    k = s["target"].size
    assert 1 < k <= 4096 and cells >= k
    assert s["X"][0, 5] == 1.0                      # the first cell is the removed atom
    assert np.all(s["col"] < k) and np.all(s["col"] >= -1)
    assert np.all(np.isfinite(s["X"])) and np.all(np.isfinite(s["target"]))


@pytest.mark.parametrize("first,count", [(0, 1), (3, 2)])
def test_forward_backward_match_oracle(collected, first, count):
    from oracle import mpnn
    g, L, recs = collected
    p = L.params().astype(np.float64)
    Xs, cols, ws, ts = [], [], [], []
    off = 0
    for k in range(first, first + count):
        s = L.sample(k)
        c = s["col"].copy()
        c[c >= 0] += off
        Xs.append(s["X"]); cols.append(c); ws.append(s["w"]); ts.append(s["target"])
        off += s["target"].size
    X, col, w, t = (np.concatenate(a) for a in (Xs, cols, ws, ts))
    loss_o, g_o, y_o = mpnn.forward_backward(p, X, col, w, t.astype(np.float64), bf16=True)
    loss_d, g_d, y_d = L.gradients(first, count)
    # same BF16 operands; FP32 vs FP64 accumulation order only
    assert np.abs(y_d - y_o).max() <= 1e-3 * max(1.0, np.abs(y_o).max())
    assert abs(loss_d - loss_o) <= 1e-3 * loss_o
    assert np.linalg.norm(g_d - g_o) <= 1e-2 * np.linalg.norm(g_o)


def test_training_fits(collected):
    g, L, recs = collected
    loss0, _, _ = L.gradients(0, EVENTS)
    loss1 = L.train(300, batch=4, lr=2e-3, seed=1)
    loss2, _, _ = L.gradients(0, EVENTS)
    print("loss before", loss0, "after", loss2, "last batches", loss1)
    assert loss2 < 0.5 * loss0


def test_learned_start_keeps_sequence_and_lowers_the_first_residual(ref_mesh):
    """Trained on the removals of another tip (another seed of the same
    generator), the network's near-field prediction on top of the recycled
    far field (warm_start 2, multigrid preconditioner) removes the same cells
    as the plain and recycled starts and ends at the same tolerance; and it
    does what it is trained for: the first residual of each solve is lower
    than the recycled start's alone, on a twin grid that runs the same
    removals.  (Whether that saves inner iterations is measured by bench.py:
    under the multigrid preconditioner it does not, see the design notes.)"""
    from conftest import SMALL_TIP
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, Learner, Mesh, solve_opts
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    tip = dict(SMALL_TIP, seed=23)
    tg = Grid(Mesh.from_tip(**tip))
    tg.solve(rel_tol=1e-10, preconditioner=1)
    L = Learner(hops=6, max_cells=4096, ell_width=64, seed=5)
    L.attach(tg, collect=True)
    Evaporation(tg, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=1, preconditioner=1)).run(120)
    L.attach(tg)
    tg.close()
    n, _ = L.samples()
    hold = n // 10
    before = L.gradients(n - hold, hold)[0]
    L.train(1500, batch=8, lr=1e-3, seed=2, first=0, count=n - hold)
    after = L.gradients(n - hold, hold)[0]
    print("held-out loss before", before, "after", after)
    assert after < 0.05 * before
    runs = {}
    for ws in (0, 1, 2):
        g = Grid(ref_mesh)
        g.solve(rel_tol=1e-10, preconditioner=1)
        if ws == 2:
            L.attach(g, predict=True)
        ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=ws, preconditioner=1))
        runs[ws] = ev.run(24)
        if ws == 2:
            L.attach(g)
        g.close()
    plain, recycled, learned = runs[0], runs[1], runs[2]
    assert [r["node"] for r in learned] == [r["node"] for r in plain] == [r["node"] for r in recycled]
    assert all(r["rel_residual"] <= 1e-10 for r in plain + recycled + learned)
    print("inner iterations over 23 events: plain", sum(r["relax_iterations"] for r in plain[1:]),
          "recycled", sum(r["relax_iterations"] for r in recycled[1:]),
          "learned", sum(r["relax_iterations"] for r in learned[1:]))
    # first residuals: twin grids, the same removals, recycled vs learned
    first = {1: [], 2: []}
    grids = {}
    for ws in (1, 2):
        g = Grid(ref_mesh)
        g.solve(rel_tol=1e-10, preconditioner=1)
        g.surface_init(0)
        grids[ws] = g
    L.attach(grids[2], predict=True)
    for k in range(10):
        node = grids[1].select().candidate
        for ws, g in grids.items():
            assert g.select().candidate == node
            g.take_away(node)
            info = g.solve(rel_tol=1e-10, max_outer=50, max_inner=20000, warm_start=ws, preconditioner=1)
            if k >= 2:
                first[ws].append(info.initial_rel_residual)
    L.attach(grids[2])
    for g in grids.values():
        g.close()
    print("first relative residuals: recycled", np.median(first[1]), "learned", np.median(first[2]))
    assert np.median(first[2]) < 0.5 * np.median(first[1])
