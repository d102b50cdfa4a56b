"""CPU FP64 oracle of the learned split (test infrastructure only: the library
never calls it).  The reference has no learned part; this is the
specification the GPU training kernels are checked against.

A split function of one tree level is an MLP d -> 64 -> 1,

    z = W1 bf16 . x + b1,   a = tanh(z),   f = w2 bf16 . a + b2,

whose weights are rounded to BF16 (round to nearest even) in the forward
pass; gradients are taken with respect to the rounded weights and applied to
FP32 master weights.  Its loss on a sample whose points are grouped into the
level's nodes, with neighbour pairs (i, j), j among the k nearest of i:

    L = (1 / P) * sum_n (1 / V_n) * sum_{(i, j) in n} (f_i - f_j)^2

over the P ordered pairs whose two points share a node, V_n the population
variance of f over node n plus eps.  The loss is small when neighbours get
close values while each node's values spread out, so a median split of f
separates few neighbours.
"""
from __future__ import annotations

import numpy as np

HIDDEN = 64
EPS = 1e-6


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def forward(X, W1, b1, w2, b2, rounded: bool = True):
    """X (m x d); W1 (64 x d), b1 (64), w2 (64), b2 scalar.  Returns (A, f).
    rounded=False skips the BF16 rounding (for finite-difference checks)."""
    rnd = bf16_round if rounded else (lambda a: np.asarray(a, np.float64))
    W1r = np.asarray(rnd(W1), np.float64)
    w2r = np.asarray(rnd(w2), np.float64)
    Z = X.astype(np.float64) @ W1r.T + b1.astype(np.float64)
    A = np.tanh(Z)
    f = A @ w2r + float(b2)
    return A, f


def loss_and_grad(X, W1, b1, w2, b2, node, nbr, rounded: bool = True):
    """node (m,): node id of every sample point; nbr (m x k): sample-local ids
    of each point's neighbours (-1 = none).  Returns (L, dW1, db1, dw2, db2)."""
    A, f = forward(X, W1, b1, w2, b2, rounded)
    m = len(f)
    nodes = np.unique(node)
    mu = np.zeros(node.max() + 1)
    V = np.zeros(node.max() + 1)
    cnt = np.zeros(node.max() + 1)
    for n in nodes:
        sel = node == n
        cnt[n] = sel.sum()
        mu[n] = f[sel].mean()
        V[n] = ((f[sel] - mu[n]) ** 2).mean() + EPS
    ii = np.repeat(np.arange(m), nbr.shape[1])
    jj = nbr.reshape(-1)
    keep = (jj >= 0)
    ii, jj = ii[keep], jj[keep]
    same = node[ii] == node[jj]
    ii, jj = ii[same], jj[same]
    P = max(len(ii), 1)
    diff = f[ii] - f[jj]
    S = np.zeros_like(V)
    np.add.at(S, node[ii], diff * diff)
    L = float(np.sum(S[nodes] / V[nodes]) / P)
    g = np.zeros(m)
    w = 2.0 * diff / (P * V[node[ii]])
    np.add.at(g, ii, w)
    np.add.at(g, jj, -w)
    g -= 2.0 * S[node] * (f - mu[node]) / (P * V[node] ** 2 * cnt[node])
    w2r = np.asarray(bf16_round(w2) if rounded else w2, np.float64)
    db2 = g.sum()
    dw2 = A.T @ g
    dZ = (g[:, None] * w2r[None, :]) * (1.0 - A * A)
    db1 = dZ.sum(0)
    dW1 = dZ.T @ X.astype(np.float64)
    return L, dW1, db1, dw2, db2
