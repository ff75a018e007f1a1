"""The numpy restatement of the order network: backward pass vs finite differences."""
import numpy as np

from oracle import mpnn_ref as R


def _random_case(rng, nq=3):
    feats = []
    for _ in range(nq):
        k = int(rng.integers(3, 7))
        x = rng.random((16, 8))
        e = np.zeros((16, 16))
        adj = np.zeros(16, dtype=np.uint32)
        for j in range(1, k):
            p = int(rng.integers(0, j))
            adj[j] |= 1 << p
            adj[p] |= 1 << j
        for u in range(k):
            for w in range(k):
                if (int(adj[u]) >> w) & 1:
                    e[u][w] = rng.random()
        feats.append((x, e, adj))
    samples = []
    for qi, (x, e, adj) in enumerate(feats):
        k = int(max(np.nonzero(adj)[0])) + 1
        mask = 0
        for v in range(k):
            mask |= 1 << v
            samples.append((qi, mask, float(rng.random() * 5)))
    return feats, samples


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    feats, samples = _random_case(rng)
    n = sum(int(np.prod(s)) for _, s in R.SHAPES)
    p = rng.normal(0, 0.2, n)
    loss, g = R.loss_and_grad(p, samples, feats)
    assert abs(loss - R.loss_only(p, samples, feats)) < 1e-12
    idx = rng.choice(n, 40, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (R.loss_only(pp, samples, feats) - R.loss_only(pm, samples, feats)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), (i, fd, g[i])
