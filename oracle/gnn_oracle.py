"""CPU restatement (FP64 numpy) of the learned block preconditioner's network, its loss
and its gradients.

TEST INFRASTRUCTURE: only the tests use this module, as the checker of the CUDA forward
and backward kernels in parallel_admm_b200/csrc/gnn.cu.  The network has no counterpart
in the reference (an addition beyond it).

Graph: the dynamic vertices, with the off-diagonal pattern of the global-step matrix A as
directed edges (row i, column j: message j -> i).  Parameters, in this order (each weight
stored row-major [out][in]):

    W0 [64 x 6],  b0 [64]                          node embedding
    for l in 0..2:
        We_l [64 x 130], be_l [64]                 edge MLP on [h_i, h_j, e_ij]
        Wn_l [64 x 128], bn_l [64]                 node MLP on [h_i, mean_j m_ij]
    Wo [7 x 64],  bo [7]                           head

Forward:  h = relu(W0 x + b0);  per layer  m_ij = relu(We [h_i; h_j; e_ij] + be),
a_i = (1 / deg_i) sum_j m_ij (row order), h_i += relu(Wn [h_i; a_i] + bn);  o = Wo h + bo.
Block:  L_i lower triangular with diagonal exp(clamp(o_i0..2, -8, 8)) and (1,0), (2,0),
(2,1) entries o_i3..5;  B_i = L_i L_i^T / a_ii  (symmetric positive definite; o = 0 gives
diag(A)^-1).  Node features are standardised per graph (columns 0-4, zero mean, unit
variance), so the network sees every system at the same scale.
Loss for residual samples r (K x n x 3):  mean_k |A (B r_k) - r_k|^2 / |r_k|^2.

Outputs for the learned global step: m_i = trace(B_i) / 3 and the warm-start coefficient
theta_i = clip(o_i6, -1, 1).  Its loss over samples (b, x_c, x_l, x*) of K unrolled sweeps

    x_0 = x_c + theta (x_c - x_l),
    x_{k+1} = x_k + omega_k m (b - A x_k) + beta_k (x_k - x_{k-1})    (beta_0 = 0)

is the mean of |x_K - x*|_A^2 / |x_c - x*|_A^2 (sweeps_loss_grad, with the adjoint
recursion written out there).
"""
import numpy as np

H = 64
F_IN = 6
F_E = 2


def param_shapes():
    shapes = [(H, F_IN), (H,)]
    for _ in range(3):
        shapes += [(H, 2 * H + F_E), (H,), (H, 2 * H), (H,)]
    shapes += [(7, H), (7,)]
    return shapes


def n_params():
    return int(sum(np.prod(s) for s in param_shapes()))


def unpack(theta):
    out, k = [], 0
    for s in param_shapes():
        n = int(np.prod(s))
        out.append(theta[k:k + n].reshape(s))
        k += n
    return out


def init_params(seed=0):
    """Small random weights; the head starts at zero, so B starts as diag(A)^-1."""
    rng = np.random.default_rng(seed)
    parts = []
    for s in param_shapes():
        if len(s) == 2:
            w = rng.normal(scale=1.0 / np.sqrt(s[1]), size=s)
        else:
            w = np.zeros(s)
        parts.append(w)
    parts[-2][:] = 0.0
    return np.concatenate([p.ravel() for p in parts])


def relu(x):
    return np.maximum(x, 0.0)


def forward(theta, x, ef, start, col, adiag):
    """Returns (blocks [n x 3 x 3], cache)."""
    P = unpack(theta)
    n = x.shape[0]
    rows = np.repeat(np.arange(n), np.diff(start))
    z0 = x @ P[0].T + P[1]
    h = relu(z0)
    cache = {"z0": z0, "h": [h], "layers": []}
    for l in range(3):
        We, be, Wn, bn = P[2 + 4 * l: 6 + 4 * l]
        inp = np.concatenate([h[rows], h[col], ef], 1)
        zm = inp @ We.T + be
        m = relu(zm)
        agg = np.zeros((n, H))
        np.add.at(agg, rows, m)
        agg = agg / np.maximum(np.diff(start), 1)[:, None]
        zn = np.concatenate([h, agg], 1) @ Wn.T + bn
        h_new = h + relu(zn)
        cache["layers"].append({"inp": inp, "zm": zm, "agg": agg, "zn": zn, "h_in": h})
        h = h_new
        cache["h"].append(h)
    o = h @ P[-2].T + P[-1]
    Lm = np.zeros((n, 3, 3))
    oc = np.clip(o[:, :3], -8.0, 8.0)
    Lm[:, 0, 0], Lm[:, 1, 1], Lm[:, 2, 2] = np.exp(oc[:, 0]), np.exp(oc[:, 1]), np.exp(oc[:, 2])
    Lm[:, 1, 0], Lm[:, 2, 0], Lm[:, 2, 1] = o[:, 3], o[:, 4], o[:, 5]
    B = np.einsum("nij,nkj->nik", Lm, Lm) / adiag[:, None, None]
    cache.update(o=o, L=Lm, rows=rows)
    return B, cache


def spmv(start, col, val, adiag, v):
    n = len(adiag)
    rows = np.repeat(np.arange(n), np.diff(start))
    out = adiag[:, None] * v
    np.add.at(out, rows, val[:, None] * v[col])
    return out


def head_grad(c, adiag, gB, gth=None):
    """dL/do from dL/dB (and dL/dtheta_i for the seventh output)."""
    n = gB.shape[0]
    G = gB / adiag[:, None, None]
    gL = np.einsum("nij,njk->nik", G + np.transpose(G, (0, 2, 1)), c["L"])
    go = np.zeros((n, 7))
    inside = np.abs(c["o"][:, :3]) < 8.0
    go[:, 0] = gL[:, 0, 0] * c["L"][:, 0, 0] * inside[:, 0]
    go[:, 1] = gL[:, 1, 1] * c["L"][:, 1, 1] * inside[:, 1]
    go[:, 2] = gL[:, 2, 2] * c["L"][:, 2, 2] * inside[:, 2]
    go[:, 3], go[:, 4], go[:, 5] = gL[:, 1, 0], gL[:, 2, 0], gL[:, 2, 1]
    if gth is not None:
        go[:, 6] = gth * (np.abs(c["o"][:, 6]) < 1.0)
    return go


def backward(theta, x, start, col, c, go):
    """Parameter gradient from dL/do (the network's backward pass)."""
    P = unpack(theta)
    grads = [np.zeros_like(p) for p in P]
    h = c["h"][-1]
    grads[-2] = go.T @ h
    grads[-1] = go.sum(0)
    gh = go @ P[-2]
    rows = c["rows"]
    for l in reversed(range(3)):
        L_ = c["layers"][l]
        We, be, Wn, bn = P[2 + 4 * l: 6 + 4 * l]
        gzn = gh * (L_["zn"] > 0)
        nin = np.concatenate([L_["h_in"], L_["agg"]], 1)
        grads[4 + 4 * l] = gzn.T @ nin
        grads[5 + 4 * l] = gzn.sum(0)
        gnin = gzn @ Wn
        gh_in = gh + gnin[:, :H]
        gagg = gnin[:, H:] / np.maximum(np.diff(start), 1)[:, None]
        gm = gagg[rows]
        gzm = gm * (L_["zm"] > 0)
        grads[2 + 4 * l] = gzm.T @ L_["inp"]
        grads[3 + 4 * l] = gzm.sum(0)
        ginp = gzm @ We
        np.add.at(gh_in, rows, ginp[:, :H])
        np.add.at(gh_in, col, ginp[:, H:2 * H])
        gh = gh_in
    gz0 = gh * (c["z0"] > 0)
    grads[0] = gz0.T @ x
    grads[1] = gz0.sum(0)
    return np.concatenate([g.ravel() for g in grads])


def loss_and_grad(theta, x, ef, start, col, val, adiag, R):
    """Loss (mean over samples) and its gradient with respect to theta."""
    B, c = forward(theta, x, ef, start, col, adiag)
    K = R.shape[0]
    loss = 0.0
    gB = np.zeros_like(B)
    for k in range(K):
        r = R[k]
        z = np.einsum("nij,nj->ni", B, r)
        res = spmv(start, col, val, adiag, z) - r
        nr = np.sum(r * r)
        loss += np.sum(res * res) / nr / K
        gz = 2.0 * spmv(start, col, val, adiag, res) / nr / K   # A symmetric
        gB += np.einsum("ni,nj->nij", gz, r)
    go = head_grad(c, adiag, gB)
    return loss, backward(theta, x, start, col, c, go)


def outputs(theta, x, ef, start, col, adiag):
    """(m, theta_v, cache): m_i = trace(B_i) / 3, theta_v = clip(o_6, -1, 1)."""
    B, c = forward(theta, x, ef, start, col, adiag)
    m = np.trace(B, axis1=1, axis2=2) / 3.0
    return m, np.clip(c["o"][:, 6], -1.0, 1.0), c


def sweeps(m, th, omega, beta, start, col, val, adiag, b, xc, xl):
    """The K iterates x_0 .. x_K and residuals r_0 .. r_{K-1} of the learned global step."""
    X = [xc + th[:, None] * (xc - xl)]
    Rs = []
    for k in range(len(omega)):
        r = b - spmv(start, col, val, adiag, X[k])
        Rs.append(r)
        bk = beta[k] if k > 0 else 0.0
        prev = X[k - 1] if k > 0 else X[0]
        X.append(X[k] + omega[k] * m[:, None] * r + bk * (X[k] - prev))
    return X, Rs


def sweeps_loss_grad(m, th, omega, beta, start, col, val, adiag, samples, mu=0.0):
    """Mean over samples (b, x_c, x_l, x*) of |x_K - x*|_A^2 / |x_c - x*|_A^2
    + mu |b - A x_K|^2 / |b - A x_c|^2 and its gradients (omega, beta, m, theta).  The second
    term (the residual that the judge checks; b - A x = -A (x - x*)) is off by default.
    Adjoint (A symmetric):
        g_K = 2 A (x_K - x*) / E_c + mu 2 A A (x_K - x*) / R_c,
        g_k = (1 + beta_k) g_{k+1} - omega_k A (m g_{k+1}) - beta_{k+1} g_{k+2},
        dL/domega_k = g_{k+1} . m r_k,  dL/dbeta_k = g_{k+1} . (x_k - x_{k-1}) (k >= 1),
        dL/dm_i = sum_k omega_k g_{k+1,i} . r_{k,i},  dL/dtheta_i = g_{0,i} . (x_c - x_l)_i."""
    K = len(omega)
    n = len(adiag)
    loss = 0.0
    go, gb, gm, gt = np.zeros(K), np.zeros(K), np.zeros(n), np.zeros(n)
    S = len(samples)
    for (b, xc, xl, xs) in samples:
        ec = xc - xs
        Aec = spmv(start, col, val, adiag, ec)
        Ec = np.sum(ec * Aec)
        if not Ec > 0:
            continue
        Rc = np.sum(Aec * Aec)
        X, Rs = sweeps(m, th, omega, beta, start, col, val, adiag, b, xc, xl)
        eK = X[K] - xs
        AeK = spmv(start, col, val, adiag, eK)
        loss += np.sum(eK * AeK) / Ec / S
        g = [None] * (K + 2)
        g[K] = 2.0 * AeK / Ec / S
        if mu > 0.0 and Rc > 0.0:
            loss += mu * np.sum(AeK * AeK) / Rc / S
            g[K] = g[K] + mu * 2.0 * spmv(start, col, val, adiag, AeK) / Rc / S
        for k in range(K - 1, -1, -1):
            bk = beta[k] if k > 0 else 0.0
            gk = (1.0 + bk) * g[k + 1] - omega[k] * spmv(start, col, val, adiag, m[:, None] * g[k + 1])
            if k + 2 <= K:
                gk = gk - beta[k + 1] * g[k + 2]
            g[k] = gk
            go[k] += np.sum(g[k + 1] * m[:, None] * Rs[k])
            if k > 0:
                gb[k] += np.sum(g[k + 1] * (X[k] - X[k - 1]))
            gm += omega[k] * np.sum(g[k + 1] * Rs[k], 1)
        gt += np.sum(g[0] * (xc - xl), 1)
    return loss, go, gb, gm, gt


def learned_loss_grad(theta, omega, beta, x, ef, start, col, val, adiag, samples):
    """The learned global step's loss and its gradients with respect to the network's
    parameters and the per-sweep coefficients."""
    m, th, c = outputs(theta, x, ef, start, col, adiag)
    loss, go, gb, gm, gt = sweeps_loss_grad(m, th, omega, beta, start, col, val, adiag, samples)
    n = len(adiag)
    gB = np.zeros((n, 3, 3))
    for d in range(3):
        gB[:, d, d] = gm / 3.0
    gout = head_grad(c, adiag, gB, gt)
    return loss, backward(theta, x, start, col, c, gout), go, gb


def features(start, col, val, adiag, mass, wc_dt2, pos):
    """Node features [log a_ii, log m_i, h^2 w_c / a_ii, degree / 16, sum_j |a_ij| / a_ii, 1]
    (the first five standardised) and edge features [a_ij / sqrt(a_ii a_jj),
    |p_i - p_j| / mean edge length]."""
    n = len(adiag)
    rows = np.repeat(np.arange(n), np.diff(start))
    deg = np.diff(start).astype(np.float64)
    off = np.zeros(n)
    np.add.at(off, rows, np.abs(val))
    x = np.stack([np.log(adiag), np.log(np.maximum(mass, 1e-30)), wc_dt2 / adiag, deg / 16.0, off / adiag,
                  np.ones(n)], 1)
    mu, sd = x[:, :5].mean(0), x[:, :5].std(0)
    x[:, :5] = (x[:, :5] - mu) / np.where(sd > 0, sd, 1.0)
    d = np.linalg.norm(pos[rows] - pos[col], axis=1)
    ef = np.stack([val / np.sqrt(adiag[rows] * adiag[col]), d / max(d.mean(), 1e-30)], 1)
    return x, ef
