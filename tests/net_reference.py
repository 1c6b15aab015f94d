"""FP64 numpy restatement of the warm-start network of lceqcd_b200/csrc/lce_net.cu
(test infrastructure: the checker of the CUDA forward and backward passes).

Sites are in the parity-split order of the fields (flat i = eo * V/2 + s, s
the half-row index of f/adresses.f).  Parameters per layer: weights
[27][16 out][16 in] then 16 biases; offset k = 9 (dx+1) + 3 (dy+1) + (dz+1).
With bf16=True the BF16 roundings of the CUDA path (input features, weights,
hidden activations, the loss gradient and the back-propagated activation
gradients) are applied at the same points, in FP64 arithmetic otherwise.
"""
from __future__ import annotations

import numpy as np

C, K, LAYERS, OUT = 16, 27, 4, 4
WL = K * C * C
PL = WL + C
NPARAM = LAYERS * PL


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) via float32, returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def coords(L):
    """(x, y, z) of every flat site."""
    L1, L2, L3 = L
    nh = L1 * L2 * L3 // 2
    hx, nxy = L1 // 2, L1 * L2 // 2
    i = np.arange(2 * nh)
    eo, s = i // nh, i % nh
    z, r = s // nxy, s % nxy
    y, xh = r // hx, r % hx
    x = 2 * xh + ((eo + y + z) & 1)
    return x, y, z


def flat_index(L, x, y, z):
    L1, L2, L3 = L
    nh = L1 * L2 * L3 // 2
    x, y, z = x % L1, y % L2, z % L3
    return ((x + y + z) & 1) * nh + z * (L1 * L2 // 2) + y * (L1 // 2) + x // 2


def neighbours(L):
    """nbr[k][i]: flat index of site i shifted by offset k."""
    x, y, z = coords(L)
    out = np.empty((K, x.size), np.int64)
    for k in range(K):
        dx, dy, dz = k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1
        out[k] = flat_index(L, x + dx, y + dy, z + dz)
    return out


def split(w):
    w = np.asarray(w, np.float64)
    Ws, bs = [], []
    for l in range(LAYERS):
        Ws.append(w[l * PL:l * PL + WL].reshape(K, C, C))
        bs.append(w[l * PL + WL:(l + 1) * PL])
    return Ws, bs


def conv(x, W, b, nbr):
    """y[i][co] = b[co] + sum_k sum_ci x[nbr_k(i)][ci] W[k][co][ci]."""
    y = np.zeros((x.shape[0], C)) if b is None else np.tile(b, (x.shape[0], 1))
    for k in range(K):
        y += x[nbr[k]] @ W[k].T
    return y


def forward_backward(w, feat, target, L, bf16_path: bool = True):
    """(output [V][4], loss, gradient [NPARAM]) of the network with parameters w."""
    r = bf16 if bf16_path else (lambda a: np.asarray(a, np.float64))
    nbr = neighbours(L)
    Ws, bs = split(w)
    Wq = [r(W) for W in Ws]
    xs = [r(feat)]
    for l in range(LAYERS - 1):
        xs.append(r(np.maximum(conv(xs[l], Wq[l], bs[l], nbr), 0.0)))
    o = conv(xs[-1], Wq[-1], bs[-1], nbr)[:, :OUT]
    t = np.asarray(target, np.float64)
    N = o.shape[0]
    n = np.sqrt((o * o).sum(1)) + 1e-12
    q = o / n[:, None]
    qt = (q * t).sum(1)
    loss = float(np.mean(1.0 - qt))
    gz = np.zeros((N, C))
    gz[:, :OUT] = -(t - qt[:, None] * q) / (n[:, None] * N)
    gz = r(gz)
    grad = np.zeros(NPARAM)
    for l in range(LAYERS - 1, -1, -1):
        gW = np.empty((K, C, C))
        for k in range(K):
            gW[k] = gz.T @ xs[l][nbr[k]]
        grad[l * PL:l * PL + WL] = gW.ravel()
        grad[l * PL + WL:(l + 1) * PL] = gz.sum(0)
        if l > 0:
            gx = np.zeros((N, C))
            for k in range(K):
                np.add.at(gx, nbr[k], gz @ Wq[l][k])
            gz = r(gx * (xs[l] > 0))
    grad[(LAYERS - 1) * PL:(LAYERS - 1) * PL + WL].reshape(K, C, C)[:, OUT:, :] = 0.0
    grad[(LAYERS - 1) * PL + WL + OUT:] = 0.0
    return o, loss, grad


def loss_only(w, feat, target, L):
    return forward_backward(w, feat, target, L, bf16_path=False)[1]
