"""NumPy float64 restatement of the precision-tier selector (test infrastructure,
never the product): the 24 per-matrix features and the 24-64-64-4 MLP's forward
pass, class-weighted cross-entropy loss, backward pass and Adam step, with the
same parameter layout as the CUDA kernels
(tinysolverdx-..._b200/csrc/selector.cuh).

The selector has no counterpart in TinySolverDx, so there is no reference output
to pin against; the checker is pinned instead by exact properties: the backward
pass against central finite differences of the loss (tests/test_selector_cpu.py)
and the features against closed forms on matrices where they are known.

Only ``tests/`` import this module.
"""
import numpy as np

N_FEAT, N_HID, N_TIER = 24, 64, 4
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_FEAT * N_HID
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID * N_TIER
N_PARAM = OFF_B3 + N_TIER


def _L(x):
    return np.log10(np.maximum(x, 1e-300))


def _clip(x):
    x = np.asarray(x, np.float64)
    return np.where(np.isnan(x), 0.0, np.clip(x, -30.0, 30.0))


def features(A, kind):
    """(batch, n, n) float64, kind scalar or (batch,) -> (batch, 24) float64."""
    A = np.asarray(A, np.float64)
    b, n, _ = A.shape
    kind = np.broadcast_to(np.asarray(kind), (b,))
    aa = np.abs(A)
    d = np.abs(np.diagonal(A, axis1=1, axis2=2))
    r = aa.sum(2)
    R = r - d
    c = aa.sum(1)
    amax = aa.max((1, 2))
    tri_l = np.tril(np.ones((n, n), bool), -1)
    lo = (A ** 2 * tri_l).sum((1, 2))
    up = (A ** 2 * tri_l.T).sum((1, 2))
    fro = (A ** 2).sum((1, 2))
    g = d - R
    with np.errstate(divide="ignore", invalid="ignore"):
        gn = np.where(r > 0, g / np.where(r > 0, r, 1.0), 0.0)
    fn = float(n)
    dmax, dmin, dmean = d.max(1), d.min(1), d.mean(1)
    ld, lr, lc = _L(d), _L(r), _L(c)

    def std(x):
        return np.sqrt(np.maximum(0.0, (x * x).mean(1) - x.mean(1) ** 2))

    f = np.zeros((b, N_FEAT))
    f[:, 0] = fn / 64.0
    f[:, 1] = (kind != 0).astype(np.float64)
    f[:, 2] = _L(dmax) - _L(dmin)
    f[:, 3] = _L(r.max(1)) - _L(r.min(1))
    f[:, 4] = _L(c.max(1)) - _L(c.min(1))
    f[:, 5] = _L(amax) - _L(dmax)
    f[:, 6] = _L(amax) - _L(dmin)
    f[:, 7] = (d > R).sum(1) / fn
    f[:, 8] = gn.min(1)
    f[:, 9] = gn.sum(1) / fn
    f[:, 10] = _L((d + R).max(1)) - _L(g.min(1))
    f[:, 11] = (g.min(1) <= 0).astype(np.float64)
    f[:, 12] = _L(np.sqrt(fro)) - _L(r.max(1))
    f[:, 13] = _L(dmax) - _L(dmean)
    f[:, 14] = _L(dmean) - _L(dmin)
    f[:, 15] = std(ld)
    f[:, 16] = std(lr)
    f[:, 17] = std(lc)
    f[:, 18] = (lr - ld).max(1)
    f[:, 19] = (lr - ld).mean(1)
    f[:, 20] = _L(np.sqrt(lo)) - _L(np.sqrt(up))
    f[:, 21] = (_L(dmin) - _L(R.sum(1) / (fn * fn - fn))) if n > 1 else 0.0
    f[:, 22] = (d < 1e-8 * dmax[:, None]).sum(1) / fn
    f[:, 23] = (lc - ld).max(1)
    return _clip(f)


def unpack(P):
    P = np.asarray(P, np.float64)
    W1 = P[OFF_W1:OFF_B1].reshape(N_FEAT, N_HID)
    b1 = P[OFF_B1:OFF_W2]
    W2 = P[OFF_W2:OFF_B2].reshape(N_HID, N_HID)
    b2 = P[OFF_B2:OFF_W3]
    W3 = P[OFF_W3:OFF_B3].reshape(N_HID, N_TIER)
    b3 = P[OFF_B3:N_PARAM]
    return W1, b1, W2, b2, W3, b3


def forward(P, norm, X):
    """Returns (logits, cache) for features X (batch, 24)."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    norm = np.asarray(norm, np.float64)
    x = (np.asarray(X, np.float64) - norm[:N_FEAT]) * norm[N_FEAT:]
    z1 = x @ W1 + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0.0)
    logits = h2 @ W3 + b3
    return logits, (x, h1, h2)


def loss_and_grad(P, norm, X, y, class_weight=None):
    """sum_s w_{y_s} CE_s / batch and its gradient with respect to P."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    logits, (x, h1, h2) = forward(P, norm, X)
    y = np.asarray(y, np.int64)
    B = len(y)
    w = np.ones(N_TIER) if class_weight is None else np.asarray(class_weight, np.float64)
    wy = w[y]
    m = logits.max(1, keepdims=True)
    e = np.exp(logits - m)
    z = e.sum(1, keepdims=True)
    p = e / z
    ce = (np.log(z[:, 0]) + m[:, 0]) - logits[np.arange(B), y]
    loss = (wy * ce).sum() / B
    dl = p.copy()
    dl[np.arange(B), y] -= 1.0
    dl *= (wy / B)[:, None]
    dW3 = h2.T @ dl
    db3 = dl.sum(0)
    dh2 = (dl @ W3.T) * (h2 > 0)
    dW2 = h1.T @ dh2
    db2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    dW1 = x.T @ dh1
    db1 = dh1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g


def adam(P, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return P - lr * mh / (np.sqrt(vh) + eps), m, v
