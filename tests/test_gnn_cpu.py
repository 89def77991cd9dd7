"""The learned preconditioner's CPU restatement: gradients against finite differences, and the
package's feature builder against it (no GPU)."""
import numpy as np

from oracle import gnn_oracle as G
from parallel_admm_b200 import gnn


def _graph(n=12, seed=0):
    rng = np.random.default_rng(seed)
    pairs = set()
    for i in range(n):
        for j in rng.choice(n, 3, replace=False):
            if i != j:
                pairs.add((i, j))
                pairs.add((j, i))
    pairs = sorted(pairs)
    start = np.zeros(n + 1, np.int64)
    col = []
    for i, j in pairs:
        start[i + 1] += 1
        col.append(j)
    start = np.cumsum(start)
    col = np.array(col)
    vals = {}
    for i, j in pairs:
        vals[(i, j)] = vals.get((j, i), -rng.uniform(0.1, 1.0))
    val = np.array([vals[p] for p in pairs])
    rows = np.repeat(np.arange(n), np.diff(start))
    adiag = np.zeros(n)
    np.add.at(adiag, rows, np.abs(val))
    adiag += 1.0
    return start, col, val, adiag, rng


def test_oracle_gradient_matches_finite_differences():
    start, col, val, adiag, rng = _graph()
    n = len(adiag)
    x, ef = G.features(start, col, val, adiag, rng.uniform(1, 2, n), rng.uniform(0, 1, n), rng.normal(size=(n, 3)))
    theta = G.init_params(1) + rng.normal(scale=0.05, size=G.n_params())
    R = rng.normal(size=(2, n, 3))
    _, g = G.loss_and_grad(theta, x, ef, start, col, val, adiag, R)
    idx = np.concatenate([rng.choice(G.n_params(), 40, replace=False), np.arange(G.n_params() - 390, G.n_params(), 37)])
    eps = 1e-6
    for k in idx:
        t1, t2 = theta.copy(), theta.copy()
        t1[k] += eps
        t2[k] -= eps
        fd = (G.loss_and_grad(t1, x, ef, start, col, val, adiag, R)[0]
              - G.loss_and_grad(t2, x, ef, start, col, val, adiag, R)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * (abs(fd) + abs(g[k])) + 1e-9, (k, fd, g[k])


def test_zero_head_is_the_jacobi_preconditioner():
    start, col, val, adiag, rng = _graph(seed=2)
    n = len(adiag)
    x, ef = G.features(start, col, val, adiag, np.ones(n), np.zeros(n), rng.normal(size=(n, 3)))
    B, _ = G.forward(G.init_params(4), x, ef, start, col, adiag)
    np.testing.assert_allclose(B, np.eye(3)[None] / adiag[:, None, None], rtol=1e-12)


def test_package_features_match_the_restatement():
    start, col, val, adiag, rng = _graph(seed=3)
    n = len(adiag)
    mass, wc, pos = rng.uniform(1, 2, n), rng.uniform(0, 1, n), rng.normal(size=(n, 3))
    sysm = gnn.System(start, col, val, adiag)
    x, ef = gnn.features(sysm, mass, wc, pos)
    xo, efo = G.features(start, col, val.astype(np.float32).astype(np.float64),
                         adiag.astype(np.float32).astype(np.float64), mass, wc, pos)
    np.testing.assert_allclose(x, xo, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(ef, efo, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(gnn.init_params(7), G.init_params(7).astype(np.float32))
