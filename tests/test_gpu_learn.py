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
    ev = Evaporation(g, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=1))
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


def test_training_fits_and_warm_start_2_keeps_sequence(collected, ref_mesh):
    from tapsim_modified_b200.tapsim import EvaporationOptions, Evaporation, Grid, solve_opts
    g, L, recs = collected
    loss0, _, _ = L.gradients(0, EVENTS)
    loss1 = L.train(300, batch=4, lr=2e-3, seed=1)
    loss2, _, _ = L.gradients(0, EVENTS)
    print("loss before", loss0, "after", loss2, "last batches", loss1)
    assert loss2 < 0.5 * loss0
    # the trained network as the near-field start: same sequence, same tolerance
    g2 = Grid(ref_mesh)
    g2.solve(rel_tol=1e-10)
    L.attach(g2, predict=True)
    opts = EvaporationOptions.from_ini(str(GOLDEN / "oracle.ini"))
    ev = Evaporation(g2, opts, relax_mode=1, solve=solve_opts(rel_tol=1e-10, warm_start=2))
    recs2 = ev.run(EVENTS)
    assert [r["node"] for r in recs2] == [r["node"] for r in recs]
    assert all(r["rel_residual"] <= 1e-10 for r in recs2)
    it1 = np.median([r["relax_iterations"] for r in recs[1:]])
    it2 = np.median([r["relax_iterations"] for r in recs2[1:]])
    print("median iterations: recycled far field", it1, "plus learned near field", it2)
