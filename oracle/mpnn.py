"""CPU restatement of the learned warm start's network (test oracle).

Test infrastructure only: the tests compare the device's forward pass, loss
and gradients (tg_learner_gradients) with this FP64 numpy version.  With
`bf16=True` the GEMM operands are rounded to BF16 exactly where the device
rounds them (the input block, the concatenated [h, A h] blocks, the
activation gradients and the weights), so the two agree to FP32 accumulation
order; with `bf16=False` the math is exact and is checked against finite
differences.

Network (the library has no counterpart in the reference):
    h0 = relu(x W0 + b0)                       x padded to 128 columns
    h_l = h_{l-1} + relu([h_{l-1}, A h_{l-1}] W_l + b_l),   l = 1..4
    y = h4 . w_out + b_out,   loss = mean((y - t)^2)
with A the ELL graph (columns `col`, -1 padding; weights `w`).
Parameters, flat: for l in 0..4 W_l (128 x 64, input x output) then b_l (64);
then w_out (64) and b_out (1).
"""
import numpy as np

F, HID, CAT, LAYERS = 16, 64, 128, 5
LAYER = CAT * HID + HID
NPARAMS = LAYERS * LAYER + HID + 1


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to BF16 (values returned as float64)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    W = [p[l * LAYER:l * LAYER + CAT * HID].reshape(CAT, HID) for l in range(LAYERS)]
    b = [p[l * LAYER + CAT * HID:(l + 1) * LAYER] for l in range(LAYERS)]
    wout = p[LAYERS * LAYER:LAYERS * LAYER + HID]
    bout = p[LAYERS * LAYER + HID]
    return W, b, wout, bout


def _aggregate(h, col, w):
    m = np.zeros_like(h)
    for k in range(col.shape[1]):
        c = col[:, k]
        ok = c >= 0
        m[ok] += w[ok, k:k + 1].astype(np.float64) * h[c[ok]]
    return m


def _aggregate_t(dm, col, w, n):
    out = np.zeros((n, dm.shape[1]))
    for k in range(col.shape[1]):
        c = col[:, k]
        ok = np.nonzero(c >= 0)[0]
        np.add.at(out, c[ok], w[ok, k:k + 1].astype(np.float64) * dm[ok])
    return out


def forward_backward(p, X, col, w, target, bf16=True):
    """Returns (loss, gradient [NPARAMS], outputs y)."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    W, b, wout, bout = unpack(p)
    Wr = [rnd(Wl) for Wl in W]
    n = X.shape[0]
    z0 = np.zeros((n, CAT))
    z0[:, :F] = X
    zs, us, hs = [rnd(z0)], [], []
    u = zs[0] @ Wr[0] + b[0]
    h = np.maximum(u, 0.0)
    us.append(u)
    hs.append(h)
    for l in range(1, LAYERS):
        m = _aggregate(h, col, w)
        z = rnd(np.concatenate([h, m], axis=1))
        u = z @ Wr[l] + b[l]
        h = h + np.maximum(u, 0.0)
        zs.append(z)
        us.append(u)
        hs.append(h)
    y = h @ wout + bout
    e = y - target
    loss = float(np.mean(e * e))
    g = np.zeros(NPARAMS)
    dy = 2.0 * e / n
    g[LAYERS * LAYER:LAYERS * LAYER + HID] = hs[-1].T @ dy
    g[LAYERS * LAYER + HID] = dy.sum()
    dh = np.outer(dy, wout)
    for l in range(LAYERS - 1, -1, -1):
        du = np.where(us[l] > 0.0, dh, 0.0)
        g[l * LAYER + CAT * HID:(l + 1) * LAYER] = du.sum(axis=0)
        dur = rnd(du)
        g[l * LAYER:l * LAYER + CAT * HID] = (zs[l].T @ dur).ravel()
        if l == 0:
            break
        dz = dur @ Wr[l].T
        dh = dh + dz[:, :HID] + _aggregate_t(dz[:, HID:], col, w, n)
    return loss, g, y
