"""CPU oracle of the learned scheduler (test infrastructure only: imported by tests/ as the
checker of the device kernels, never by the package).

The scheduler has no counterpart in the reference (its BFS/CC strategy is fixed by
constants: scout_bfs.cu:475-476, scout_cc.cu:68-69 and 469, core/local_repair.h:13-26), so
this oracle restates the project's own specification in float64 numpy:

* the cost model: a 24-64-64-4 ReLU perceptron over one flat parameter vector
  W1[64][24] b1[64] W2[64][64] b2[64] W3[4][64] b3[4] (6,020 values), masked mean squared
  error and its gradient by hand-written backpropagation (pinned against central finite
  differences in the CPU tests);
* the 24 per-batch features the device computes between the merge and the repair.

Parity with the device: gradients within a relative 1e-4 of this float64 restatement
(fp32 arithmetic with atomically summed tiles), features within 1e-5 absolute.
"""
from __future__ import annotations

import math

import numpy as np

IN, H, OUT = 24, 64, 4
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT * H
NPARAM = OFF_B3 + OUT


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    assert w.size == NPARAM
    return (w[OFF_W1:OFF_B1].reshape(H, IN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(H, H),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3].reshape(OUT, H), w[OFF_B3:NPARAM])


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, dtype=np.float64).reshape(-1, IN)
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3.T + b3


def loss(w, x, t, m):
    y = forward(w, x)
    m = np.asarray(m, dtype=np.float64).reshape(-1, OUT)
    d = y - np.asarray(t, dtype=np.float64).reshape(-1, OUT)
    return float((m * d * d).sum() / m.sum())


def loss_grad(w, x, t, m):
    """Masked MSE and its gradient with respect to the flat parameter vector."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, dtype=np.float64).reshape(-1, IN)
    t = np.asarray(t, dtype=np.float64).reshape(-1, OUT)
    m = np.asarray(m, dtype=np.float64).reshape(-1, OUT)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ W3.T + b3
    norm = m.sum()
    d = y - t
    L = float((m * d * d).sum() / norm)
    dy = 2.0 * m * d / norm
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = (dy.T @ h2).ravel()
    g[OFF_B3:NPARAM] = dy.sum(0)
    d2 = (dy @ W3) * (h2 > 0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return L, g


def finite_diff_grad(w, x, t, m, idx, eps=1e-6):
    """Central differences of the loss at the parameter indices idx."""
    w = np.asarray(w, dtype=np.float64).copy()
    out = np.zeros(len(idx))
    for i, k in enumerate(idx):
        o = w[k]
        w[k] = o + eps
        lp = loss(w, x, t, m)
        w[k] = o - eps
        lm = loss(w, x, t, m)
        w[k] = o
        out[i] = (lp - lm) / (2 * eps)
    return out


def targets(variant_ms, changed):
    """Training targets and mask of one probed batch: log2(1 + repair microseconds) / 4 per
    variant (mask 0 where the problem lacks the variant), log2(1 + changed) / 24."""
    t = np.zeros(OUT, dtype=np.float32)
    mk = np.zeros(OUT, dtype=np.float32)
    for v in range(3):
        if variant_ms[v] >= 0:
            t[v] = math.log2(1.0 + 1000.0 * variant_ms[v]) / 4.0
            mk[v] = 1.0
    t[3] = math.log2(1.0 + changed) / 24.0
    mk[3] = 1.0
    return t, mk


def features(off, adj, edges, problem, level=None, prev_ms=0.0):
    """The 24 scheduler features of one toggle batch applied to the CSR (off, adj) as it
    stood before the batch. The batch must hold distinct, valid pairs (u != v); level are
    the BFS levels before the repair (BFS only)."""
    off = np.asarray(off, dtype=np.int64)
    adj = np.asarray(adj, dtype=np.int64)
    n = len(off) - 1
    rows = [set(adj[off[v]:off[v + 1]].tolist()) for v in range(n)] if n <= 1 << 16 else None
    deg = np.diff(off).astype(np.int64)
    ins = dele = 0
    dels = []
    aff = set()
    for u, v in np.asarray(edges).tolist():
        present = (v in rows[u]) if rows is not None else bool(np.any(adj[off[u]:off[u + 1]] == v))
        if present:
            dele += 1
            deg[u] -= 1
            deg[v] -= 1
            dels += [(u, v), (v, u)]
        else:
            ins += 1
            deg[u] += 1
            deg[v] += 1
        aff.add(u)
        aff.add(v)
    ed = ins + dele
    nnz = int(deg.sum())
    f = np.zeros(IN, dtype=np.float64)
    f[0] = math.log2(1 + ed) / 24
    f[1] = ins / ed if ed else 0.0
    f[2] = dele / ed if ed else 0.0
    na = len(aff)
    for a in aff:
        b = min(15, int(math.floor(math.log2(deg[a] + 1))))
        f[3 + b] += 1.0 / na
    f[19] = math.log2(1 + n) / 32
    f[20] = math.log2(1 + nnz / max(1, n)) / 8
    f[21] = math.log2(1 + na) / math.log2(2 + n)
    hit = 0
    for x, y in dels:
        if problem == "bfs":
            hit += int(level[x] >= 0 and level[y] == level[x] + 1)
        else:
            hit += int(deg[y] <= 2)
    f[22] = hit / len(dels) if dels else 0.0
    f[23] = math.log2(1 + 1000.0 * prev_ms) / 16
    return f
