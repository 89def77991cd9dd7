"""The learned preconditioner's CPU restatement: gradients against finite differences, and the
package's feature builder against it (no GPU)."""
import numpy as np
import pytest

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


def _samples(start, col, val, adiag, rng, k=2):
    """(b, x_c, x_l, x*) samples with x* = A^-1 b (dense solve of the small system)."""
    n = len(adiag)
    A = np.diag(adiag)
    rows = np.repeat(np.arange(n), np.diff(start))
    A[rows, col] = val
    out = []
    for _ in range(k):
        xs = rng.normal(size=(n, 3))
        b = A @ xs
        xc = xs + rng.normal(scale=0.3, size=(n, 3))
        xl = xc + rng.normal(scale=0.1, size=(n, 3))
        out.append((b, xc, xl, np.linalg.solve(A, b)))
    return out


@pytest.mark.parametrize("mu", [0.0, 0.7])
def test_learned_step_adjoint_matches_finite_differences(mu):
    """Gradients of the unrolled learned sweeps (omega, beta, m, theta) by the adjoint
    recursion against central differences of the FP64 loss, without and with the residual
    term mu |b - A x_K|^2 / |b - A x_c|^2."""
    start, col, val, adiag, rng = _graph(n=14, seed=5)
    n = len(adiag)
    K = 5
    omega = rng.uniform(0.6, 1.4, K)
    beta = rng.uniform(0.0, 0.4, K)
    m = rng.uniform(0.7, 1.3, n) / adiag
    th = rng.uniform(-0.5, 0.8, n)
    S = _samples(start, col, val, adiag, rng)
    loss, go, gb, gm, gt = G.sweeps_loss_grad(m, th, omega, beta, start, col, val, adiag, S, mu=mu)
    assert loss > 0
    eps = 1e-6

    def f(o=omega, b=beta, mm=m, t=th):
        return G.sweeps_loss_grad(mm, t, o, b, start, col, val, adiag, S, mu=mu)[0]

    for k in range(K):
        for arr, grad in ((omega, go), (beta, gb)):
            if arr is beta and k == 0:
                assert grad[0] == 0.0  # beta_0 is not used
                continue
            a1, a2 = arr.copy(), arr.copy()
            a1[k] += eps
            a2[k] -= eps
            fd = ((f(o=a1) - f(o=a2)) if arr is omega else (f(b=a1) - f(b=a2))) / (2 * eps)
            assert abs(fd - grad[k]) <= 1e-5 * (abs(fd) + abs(grad[k])) + 1e-9, (k, fd, grad[k])
    for i in rng.choice(n, 5, replace=False):
        for arr, grad in ((m, gm), (th, gt)):
            a1, a2 = arr.copy(), arr.copy()
            h = eps * max(1.0, abs(arr[i]))
            a1[i] += h
            a2[i] -= h
            fd = ((f(mm=a1) - f(mm=a2)) if arr is m else (f(t=a1) - f(t=a2))) / (2 * h)
            assert abs(fd - grad[i]) <= 1e-5 * (abs(fd) + abs(grad[i])) + 1e-9, (i, fd, grad[i])


def test_learned_step_network_gradient_matches_finite_differences():
    """Through the network: m = trace(B) / 3 and theta = clip(o_6) from the head."""
    start, col, val, adiag, rng = _graph(n=12, seed=6)
    n = len(adiag)
    x, ef = G.features(start, col, val, adiag, rng.uniform(1, 2, n), rng.uniform(0, 1, n), rng.normal(size=(n, 3)))
    theta = G.init_params(2) + rng.normal(scale=0.05, size=G.n_params())
    K = 4
    omega, beta = rng.uniform(0.8, 1.2, K), rng.uniform(0.0, 0.3, K)
    S = _samples(start, col, val, adiag, rng)
    _, g, _, _ = G.learned_loss_grad(theta, omega, beta, x, ef, start, col, val, adiag, S)
    P = G.n_params()
    idx = np.concatenate([rng.choice(P, 25, replace=False), np.arange(P - 455, P, 23)])
    eps = 1e-6
    for k in idx:
        t1, t2 = theta.copy(), theta.copy()
        t1[k] += eps
        t2[k] -= eps
        fd = (G.learned_loss_grad(t1, omega, beta, x, ef, start, col, val, adiag, S)[0]
              - G.learned_loss_grad(t2, omega, beta, x, ef, start, col, val, adiag, S)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * (abs(fd) + abs(g[k])) + 1e-9, (k, fd, g[k])


def test_zero_head_learned_step_is_jacobi():
    """An all-zero head, omega = 1, beta = 0: the learned step is the Jacobi sweep."""
    start, col, val, adiag, rng = _graph(n=10, seed=7)
    n = len(adiag)
    x, ef = G.features(start, col, val, adiag, np.ones(n), np.zeros(n), rng.normal(size=(n, 3)))
    m, th, _ = G.outputs(G.init_params(3), x, ef, start, col, adiag)
    np.testing.assert_allclose(m, 1.0 / adiag, rtol=1e-12)
    assert np.all(th == 0.0)
    (b, xc, xl, _), = _samples(start, col, val, adiag, rng, k=1)
    X, _ = G.sweeps(m, th, np.ones(3), np.zeros(3), start, col, val, adiag, b, xc, xl)
    xj = xc.copy()
    for _ in range(3):
        xj = (b - (G.spmv(start, col, val, adiag, xj) - adiag[:, None] * xj)) / adiag[:, None]
    np.testing.assert_allclose(X[3], xj, rtol=1e-10, atol=1e-12)
