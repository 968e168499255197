"""The network oracle (oracle/mpnn.py) against finite differences."""
import numpy as np

from oracle import mpnn


def _graph(rng, n=40, D=6):
    col = np.full((n, D), -1, np.int32)
    w = np.zeros((n, D), np.float32)
    for i in range(n):
        nb = rng.choice(n, size=rng.integers(1, D + 1), replace=False)
        col[i, :len(nb)] = nb
        w[i, :len(nb)] = rng.random(len(nb)) / len(nb)
    X = rng.standard_normal((n, mpnn.F)).astype(np.float32)
    t = rng.standard_normal(n)
    return X, col, w, t


def _params(rng):
    p = np.zeros(mpnn.NPARAMS)
    for l in range(mpnn.LAYERS):
        fan = mpnn.F if l == 0 else mpnn.CAT
        W = np.zeros((mpnn.CAT, mpnn.HID))
        W[:fan] = rng.standard_normal((fan, mpnn.HID)) * np.sqrt(2.0 / fan)
        p[l * mpnn.LAYER:l * mpnn.LAYER + mpnn.CAT * mpnn.HID] = W.ravel()
        p[l * mpnn.LAYER + mpnn.CAT * mpnn.HID:(l + 1) * mpnn.LAYER] = 0.1 * rng.standard_normal(mpnn.HID)
    p[mpnn.LAYERS * mpnn.LAYER:] = 0.1 * rng.standard_normal(mpnn.HID + 1)
    return p


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    X, col, w, t = _graph(rng)
    p = _params(rng)
    loss, g, _ = mpnn.forward_backward(p, X, col, w, t, bf16=False)
    # a sample of parameters from every block: weights, biases, readout
    idx = [3, 100, 1000, mpnn.CAT * mpnn.HID + 7, mpnn.LAYER + 200, 2 * mpnn.LAYER + 5000,
           3 * mpnn.LAYER + mpnn.CAT * mpnn.HID + 1, 4 * mpnn.LAYER + 8000, mpnn.NPARAMS - 10, mpnn.NPARAMS - 1]
    for k in idx:
        h = 1e-6 * max(1.0, abs(p[k]))
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (mpnn.forward_backward(pp, X, col, w, t, bf16=False)[0] -
              mpnn.forward_backward(pm, X, col, w, t, bf16=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-39], np.float32)
    r = mpnn.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6
    assert r[3] == -2.5
