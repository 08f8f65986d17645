"""CPU restatement of the learned selector's arithmetic -- TEST INFRASTRUCTURE ONLY.

Only tests/ may import this module; the engine never calls it.  The reference has no
selector (it runs the formats it is told to), so there is nothing of the reference to pin
here: these are plain numpy statements of the engine's own definitions, used as the oracle
for the CUDA kernels.

* ``features(rp, ci, n)``  -- the 12 structural features of pava_features (float64 here;
  the kernel accumulates the same integer statistics, so they agree to float32 rounding)
* ``mlp_forward`` / ``mlp_loss_grad`` -- the MLP 12-64-64-32 with ReLU and the masked mean
  squared error, forward and backward in float64, for the gradient check of pava_mlp_gradient
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 12, 64, 32
OW1, OB1 = 0, HID * IN
OW2, OB2 = OB1 + HID, OB1 + HID + HID * HID
OW3, OB3 = OB2 + HID, OB2 + HID + OUT * HID
NP = OB3 + OUT


def features(rp, ci, n):
    rp = np.asarray(rp, np.int64)
    ci = np.asarray(ci, np.int64)
    m = len(rp) - 1
    nnz = int(rp[-1])
    L = np.diff(rp)
    M, Z, N = max(m, 1), max(nnz, 1), max(n, 1)
    mean = nnz / M
    var = float((L * L).sum()) / M - mean * mean
    rows = np.repeat(np.arange(m, dtype=np.int64), L)
    d = np.abs(ci - rows)
    first = np.zeros(nnz, bool)
    first[rp[:-1][L > 0]] = True
    sec = ci >> 4
    newline = first.copy()
    newline[1:] |= sec[1:] != sec[:-1]
    nonempty = L > 0
    span = (ci[rp[1:][nonempty] - 1] - ci[rp[:-1][nonempty]] + 1).sum() if nonempty.any() else 0
    ne = int(nonempty.sum())
    f = np.empty(12)
    f[0] = np.log10(M)
    f[1] = np.log10(Z)
    f[2] = np.log10(max(mean, 1e-9))
    f[3] = np.sqrt(max(var, 0.0)) / mean if mean > 0 else 0.0
    f[4] = np.log10(L.max() / mean) if mean > 0 and L.max() > 0 else 0.0
    f[5] = (L == 0).sum() / M
    f[6] = L[L > 64].sum() / Z
    f[7] = ((L >= 1) & (L <= 4)).sum() / M
    f[8] = np.log10(d.sum() / Z / N + 1e-7)
    f[9] = (d <= 64).sum() / Z
    f[10] = newline.sum() / Z
    f[11] = np.log10((span / ne if ne else 0.0) / N + 1e-7)
    return f


def unpack(P):
    P = np.asarray(P, np.float64)
    return (P[OW1:OB1].reshape(HID, IN), P[OB1:OW2], P[OW2:OB2].reshape(HID, HID), P[OB2:OW3],
            P[OW3:OB3].reshape(OUT, HID), P[OB3:NP])


def mlp_forward(P, X):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    Z1 = X @ W1.T + b1
    H1 = np.maximum(Z1, 0)
    Z2 = H1 @ W2.T + b2
    H2 = np.maximum(Z2, 0)
    return H2 @ W3.T + b3, (Z1, H1, Z2, H2)


def mlp_loss_grad(P, X, T, mask=None):
    """Masked MSE = sum(mask (O - T)^2) / sum(mask) and its gradient (float64)."""
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    mask = np.ones_like(T) if mask is None else np.asarray(mask, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(P)
    O, (Z1, H1, Z2, H2) = mlp_forward(P, X)
    cnt = mask.sum()
    loss = float((mask * (O - T) ** 2).sum() / cnt)
    dO = 2.0 * mask * (O - T) / cnt
    gW3 = dO.T @ H2
    gb3 = dO.sum(0)
    dZ2 = (dO @ W3) * (Z2 > 0)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * (Z1 > 0)
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
