"""NumPy restatement of the order model's network — TEST INFRASTRUCTURE ONLY.

An independent float64 forward pass and hand-derived backward pass of the
message-passing network in matrixgraph_b200/csrc/mg_order_model.cu, used by
tests/ to check the CUDA gradients (analytically and by finite differences).
"""
from __future__ import annotations

import numpy as np

MF, MH = 8, 64
SHAPES = [("W1x", (MH, MF)), ("W1m", (MH, MF + 1)), ("b1", (MH,)), ("W2h", (MH, MH)),
          ("W2m", (MH, MH)), ("b2", (MH,)), ("Wr", (MH, MH)), ("br", (MH,)), ("wo", (MH,)),
          ("bo", (1,))]


def unpack(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    assert o == len(p)
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SHAPES])


def forward(P, x, e, adj, mask, cache=False):
    nodes = [u for u in range(16) if (mask >> u) & 1]
    xs = np.array([x[u] for u in nodes], dtype=np.float64)
    for a, u in enumerate(nodes):
        xs[a, 5] = bin(int(adj[u]) & mask).count("1") * 0.125
    A = np.array([[1.0 if (int(adj[u]) >> w) & 1 else 0.0 for w in nodes] for u in nodes])
    E = np.array([[e[u][w] if (int(adj[u]) >> w) & 1 else 0.0 for w in nodes] for u in nodes])
    a1 = np.concatenate([A @ xs, E.sum(axis=1, keepdims=True)], axis=1)
    p1 = xs @ P["W1x"].T + a1 @ P["W1m"].T + P["b1"]
    h1 = np.maximum(p1, 0)
    a2 = A @ h1
    p2 = h1 @ P["W2h"].T + a2 @ P["W2m"].T + P["b2"]
    h2 = np.maximum(p2, 0)
    z = h2.sum(axis=0)
    pr = P["Wr"] @ z + P["br"]
    r = np.maximum(pr, 0)
    y = float(P["wo"] @ r + P["bo"][0])
    if not cache:
        return y
    return y, dict(xs=xs, A=A, a1=a1, p1=p1, h1=h1, a2=a2, p2=p2, h2=h2, z=z, pr=pr, r=r)


def loss_and_grad(params, samples, feats):
    """Mean squared error over samples (q, mask, target) and its gradient."""
    P = unpack(params)
    G = {k: np.zeros_like(v) for k, v in P.items()}
    loss = 0.0
    n = len(samples)
    for q, mask, t in samples:
        x, e, adj = feats[q]
        y, c = forward(P, x, e, adj, int(mask), cache=True)
        d = y - t
        loss += d * d / n
        dy = 2 * d / n
        G["bo"][0] += dy
        G["wo"] += dy * c["r"]
        dr = dy * P["wo"] * (c["pr"] > 0)
        G["br"] += dr
        G["Wr"] += np.outer(dr, c["z"])
        dz = P["Wr"].T @ dr
        dp2 = dz[None, :] * (c["p2"] > 0)
        G["b2"] += dp2.sum(axis=0)
        G["W2h"] += dp2.T @ c["h1"]
        G["W2m"] += dp2.T @ c["a2"]
        dh1 = dp2 @ P["W2h"] + c["A"].T @ (dp2 @ P["W2m"])
        dp1 = dh1 * (c["p1"] > 0)
        G["b1"] += dp1.sum(axis=0)
        G["W1x"] += dp1.T @ c["xs"]
        G["W1m"] += dp1.T @ c["a1"]
    return loss, pack(G)


def loss_only(params, samples, feats):
    P = unpack(params)
    return sum((forward(P, *feats[q], int(m)) - t) ** 2 for q, m, t in samples) / len(samples)
