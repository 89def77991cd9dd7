"""Learned per-vertex block preconditioner for the PCG global step (global_solver 2).

An addition with no counterpart in the reference.  The network (3 message-passing
layers of width 64 over the graph of the global matrix A) and its training run on the GPU in
the library's own kernels (csrc/gnn.cu, C ABI ``admm_gnn_*``); this module builds the inputs,
drives training and hands the predicted blocks to a solver handle:

    sysm = system(handle)                       # A of the handle (CSR + diagonal)
    net = LearnedPreconditioner()
    net.fit([(sysm, feats, residuals), ...])   # (system, residual samples) from plain runs
    handle.set_preconditioner(net.blocks(sysm, feats))

Node features per dynamic vertex: [log a_ii, log m_i, h^2 w_c,i / a_ii, degree / 16,
sum_j |a_ij| / a_ii, 1], the first five standardised per system; edge features per
off-diagonal entry: [a_ij / sqrt(a_ii a_jj),
|p_i - p_j| / mean edge length].  Block i = L_i L_i^T / a_ii with L_i lower triangular from
the network's 6 outputs (exp of the outputs clamped to [-8, 8] on the diagonal); messages are
averaged over a vertex's neighbours; all-zero outputs give diag(A)^-1, the plain
Jacobi preconditioner the network starts from and falls back to.
"""
import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import backend as B

_i = ctypes.POINTER(ctypes.c_int32)
_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p


def _lib():
    L = B.lib()
    if not getattr(L, "_gnn_sigs", False):
        sig = {
            "admm_gnn_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp)]),
            "admm_gnn_set_graph": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _i, _i, _f, _f, _f, _f]),
            "admm_gnn_destroy": (None, [vp]),
            "admm_gnn_num_params": (ctypes.c_int, []),
            "admm_gnn_set_params": (ctypes.c_int, [vp, _f, ctypes.c_int]),
            "admm_gnn_get_params": (ctypes.c_int, [vp, _f, ctypes.c_int]),
            "admm_gnn_forward": (ctypes.c_int, [vp, _f]),
            "admm_gnn_loss_grad": (ctypes.c_int, [vp, _f, ctypes.c_int, _d, _f]),
            "admm_gnn_adam": (ctypes.c_int, [vp, ctypes.c_float]),
            "admm_b200_system": (ctypes.c_int, [vp, _i, _i, _f, _f]),
            "admm_gnn_outputs": (ctypes.c_int, [vp, _f, _f]),
            "admm_gnn_backward": (ctypes.c_int, [vp, _f, _f, _f]),
            "admm_learn_create": (ctypes.c_int, [ctypes.c_int, _i, _i, _f, _f, ctypes.POINTER(vp)]),
            "admm_learn_destroy": (None, [vp]),
            "admm_learn_loss_grad": (ctypes.c_int, [vp, ctypes.c_int, _f, _f, _f, _f, ctypes.c_int, _f, _f, _f, _f,
                                                    _d, _f, _f, _f, _f]),
            "admm_learn_solve": (ctypes.c_int, [vp, _f, _f, ctypes.c_double, ctypes.c_int, _i]),
            "admm_learn_set_residual_weight": (ctypes.c_int, [vp, ctypes.c_double]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L._gnn_sigs = True
    return L


def _p(a, ct):
    return a.ctypes.data_as(ct)


class System:
    """The global matrix A of a handle: off-diagonal CSR (sorted columns) and diagonal, FP32."""

    def __init__(self, start, col, val, diag):
        self.start = np.ascontiguousarray(start, np.int32)
        self.col = np.ascontiguousarray(col, np.int32)
        self.val = np.ascontiguousarray(val, np.float32)
        self.diag = np.ascontiguousarray(diag, np.float32)
        self.n = len(self.diag)

    def matvec(self, v: np.ndarray) -> np.ndarray:
        """A v for v of shape (n, 3), FP64 on the host (data generation, evaluation)."""
        rows = np.repeat(np.arange(self.n), np.diff(self.start))
        out = self.diag[:, None].astype(np.float64) * v
        np.add.at(out, rows, self.val[:, None].astype(np.float64) * v[self.col])
        return out


def system(h: "B.Handle") -> System:
    L = _lib()
    nnz = L.admm_b200_system(h.h, None, None, None, None)
    start = np.zeros(h.n_dyn + 1, np.int32)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float32)
    diag = np.zeros(h.n_dyn, np.float32)
    rc = L.admm_b200_system(h.h, _p(start, _i), _p(col, _i), _p(val, _f), _p(diag, _f))
    if rc < 0:
        raise B.AdmmError(rc, "admm_b200_system")
    return System(start, col[:nnz], val[:nnz], diag)


def features(sysm: System, mass: np.ndarray, wc_dt2: np.ndarray, pos: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Node features [n x 6] and edge features [nnz x 2] (see the module docstring)."""
    n = sysm.n
    a = sysm.diag.astype(np.float64)
    val = sysm.val.astype(np.float64)
    rows = np.repeat(np.arange(n), np.diff(sysm.start))
    deg = np.diff(sysm.start).astype(np.float64)
    off = np.zeros(n)
    np.add.at(off, rows, np.abs(val))
    x = np.stack([np.log(a), np.log(np.maximum(mass[:n].astype(np.float64), 1e-30)), wc_dt2[:n] / a, deg / 16.0,
                  off / a, np.ones(n)], 1)
    mu, sd = x[:, :5].mean(0), x[:, :5].std(0)
    x[:, :5] = (x[:, :5] - mu) / np.where(sd > 0, sd, 1.0)
    d = np.linalg.norm(pos[rows].astype(np.float64) - pos[sysm.col].astype(np.float64), axis=1)
    ef = np.stack([val / np.sqrt(a[rows] * a[sysm.col]), d / max(d.mean() if len(d) else 1.0, 1e-30)], 1)
    return x.astype(np.float32), ef.astype(np.float32)


def scene_features(sc, sysm: System) -> Tuple[np.ndarray, np.ndarray]:
    """Features of a scene's system at its rest positions."""
    wc_dt2 = np.zeros(sysm.n)
    surf = np.zeros(sc.n_vert, bool)
    surf[sc.surf_verts] = True
    wc = sc.contact_w.astype(np.float64) * sc.params.dt * sc.params.dt
    wc_dt2[:] = np.where(surf[:sysm.n], wc[:sysm.n], 0.0)
    return features(sysm, sc.mass, wc_dt2, sc.verts[:sysm.n])


def global_residuals(h: "B.Handle", sysm: System, frames: int) -> np.ndarray:
    """Residual samples r = b - A x of the global step after the plain solve, one per frame
    (the handle steps `frames` substeps)."""
    out = []
    for _ in range(frames):
        h.step(1, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        b = h.read(B.BUF_B)[:sysm.n].astype(np.float64)
        x = h.read(B.BUF_X)[:sysm.n].astype(np.float64)
        r = b - sysm.matvec(x)
        if np.linalg.norm(r) > 0:
            out.append(r.astype(np.float32))
    return np.array(out, np.float32).reshape(-1, sysm.n, 3)


def pcg_iterations(sysm: System, blocks: Optional[np.ndarray], b: np.ndarray, tol: float = 1e-4,
                   maxit: int = 2000) -> int:
    """Preconditioned CG iterations to |r| <= tol |b| (FP64 on the host; blocks None = diag(A))."""
    if blocks is None:
        apply = lambda r: r / sysm.diag[:, None].astype(np.float64)
    else:
        Bk = blocks.reshape(-1, 3, 3).astype(np.float64)
        apply = lambda r: np.einsum("nij,nj->ni", Bk, r)
    x = np.zeros_like(b, np.float64)
    r = b.astype(np.float64).copy()
    u = apply(r)
    p = u.copy()
    rz = np.sum(r * u)
    r0 = np.linalg.norm(r)
    for k in range(maxit):
        if np.linalg.norm(r) <= tol * r0:
            return k
        q = sysm.matvec(p)
        a = rz / np.sum(p * q)
        x += a * p
        r -= a * q
        u = apply(r)
        rzn = np.sum(r * u)
        if not rzn > 0:
            return maxit
        p = u + (rzn / rz) * p
        rz = rzn
    return maxit


class LearnedPreconditioner:
    """The network (parameters, Adam state) on the GPU; one system at a time."""

    def __init__(self, bf16: bool = True, seed: int = 0):
        L = _lib()
        self.bf16 = bool(bf16)
        self.g = vp()
        rc = L.admm_gnn_create(int(bf16), ctypes.byref(self.g))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_create")
        self.P = L.admm_gnn_num_params()
        self.set_params(init_params(seed))
        self._bound = None

    def close(self):
        if self.g:
            _lib().admm_gnn_destroy(self.g)
            self.g = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bind(self, sysm: System, x: np.ndarray, ef: np.ndarray):
        key = (id(sysm), id(x))
        if self._bound == key:
            return
        self._keep = (sysm, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(ef, np.float32))
        s, xx, ee = self._keep
        rc = _lib().admm_gnn_set_graph(self.g, s.n, len(s.col), _p(s.start, _i), _p(s.col, _i), _p(s.val, _f),
                                       _p(s.diag, _f), _p(xx, _f), _p(ee, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_set_graph")
        self._bound = key

    def set_params(self, theta: np.ndarray):
        th = np.ascontiguousarray(theta, np.float32)
        assert th.size == self.P
        rc = _lib().admm_gnn_set_params(self.g, _p(th, _f), self.P)
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_set_params")

    def params(self) -> np.ndarray:
        th = np.zeros(self.P, np.float32)
        _lib().admm_gnn_get_params(self.g, _p(th, _f), self.P)
        return th

    def blocks(self, sysm: System, x: np.ndarray, ef: np.ndarray) -> np.ndarray:
        self.bind(sysm, x, ef)
        out = np.zeros((sysm.n, 9), np.float32)
        rc = _lib().admm_gnn_forward(self.g, _p(out, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_forward")
        return out

    def blocks_or_fallback(self, sysm: System, x: np.ndarray, ef: np.ndarray, probe: np.ndarray,
                           tol: float = 1e-4) -> Tuple[np.ndarray, bool, float]:
        """The learned blocks for a system, judged by plain diag(A): on the probe residuals,
        PCG with the learned blocks must need fewer iterations than with diag(A), else
        diag(A) as 3x3 blocks is returned.  Returns (blocks, learned_used, iteration ratio
        learned / diag(A))."""
        blk = self.blocks(sysm, x, ef)
        it_l = np.mean([pcg_iterations(sysm, blk, r.astype(np.float64), tol) for r in probe])
        it_j = np.mean([pcg_iterations(sysm, None, r.astype(np.float64), tol) for r in probe])
        ratio = float(it_l / max(it_j, 1e-30))
        if it_l < it_j:
            return blk, True, ratio
        diag = np.zeros((sysm.n, 9), np.float32)
        diag[:, 0] = diag[:, 4] = diag[:, 8] = 1.0 / sysm.diag
        return diag, False, ratio

    def loss_grad(self, sysm: System, x: np.ndarray, ef: np.ndarray, R: np.ndarray):
        self.bind(sysm, x, ef)
        RR = np.ascontiguousarray(R, np.float32)
        loss = ctypes.c_double()
        grad = np.zeros(self.P, np.float32)
        rc = _lib().admm_gnn_loss_grad(self.g, _p(RR, _f), RR.shape[0], ctypes.byref(loss), _p(grad, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_loss_grad")
        return loss.value, grad

    def outputs(self, sysm: System, x: np.ndarray, ef: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """(m, theta) per vertex for the learned global step (global_solver 3)."""
        self.bind(sysm, x, ef)
        m = np.zeros(sysm.n, np.float32)
        th = np.zeros(sysm.n, np.float32)
        rc = _lib().admm_gnn_outputs(self.g, _p(m, _f), _p(th, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_outputs")
        return m, th

    def backward(self, sysm: System, x: np.ndarray, ef: np.ndarray, gm: np.ndarray, gth: np.ndarray) -> np.ndarray:
        """Parameter gradient from the gradients with respect to (m, theta); Adam applies it."""
        self.bind(sysm, x, ef)
        gm = np.ascontiguousarray(gm, np.float32)
        gth = np.ascontiguousarray(gth, np.float32)
        grad = np.zeros(self.P, np.float32)
        rc = _lib().admm_gnn_backward(self.g, _p(gm, _f), _p(gth, _f), _p(grad, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_backward")
        return grad

    def step(self, lr: float):
        rc = _lib().admm_gnn_adam(self.g, ctypes.c_float(lr))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_gnn_adam")

    def fit(self, data: Sequence[Tuple[System, np.ndarray, np.ndarray, np.ndarray]], epochs: int = 20,
            lr: float = 1e-3, batch: int = 8, seed: int = 0) -> List[float]:
        """Adam on the mean loss over (system, node features, edge features, residuals) items;
        returns the loss per epoch."""
        rng = np.random.default_rng(seed)
        hist = []
        for _ in range(epochs):
            tot = 0.0
            for k in rng.permutation(len(data)):
                sysm, x, ef, R = data[k]
                sel = rng.choice(len(R), min(batch, len(R)), replace=False)
                loss, _ = self.loss_grad(sysm, x, ef, R[sel])
                self.step(lr)
                tot += loss / len(data)
            hist.append(tot)
        return hist


class SweepTrainer:
    """GPU context of the learned global step's training on one system (learn.cu)."""

    def __init__(self, sysm: System, residual_weight: float = 0.0):
        self.sysm = sysm
        self.L = vp()
        rc = _lib().admm_learn_create(sysm.n, _p(sysm.start, _i), _p(sysm.col, _i), _p(sysm.val, _f),
                                      _p(sysm.diag, _f), ctypes.byref(self.L))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_learn_create")
        if residual_weight:
            rc = _lib().admm_learn_set_residual_weight(self.L, float(residual_weight))
            if rc != B.OK:
                raise B.AdmmError(rc, "admm_learn_set_residual_weight")

    def close(self):
        if self.L:
            _lib().admm_learn_destroy(self.L)
            self.L = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, b: np.ndarray, x0: np.ndarray, tol: float = 1e-6, maxit: int = 20000) -> Tuple[np.ndarray, int]:
        """The converged solution of A x = b (conjugate gradients from x0)."""
        bb = np.ascontiguousarray(b, np.float32)
        x = np.array(x0, np.float32, copy=True, order="C")
        it = ctypes.c_int32()
        rc = _lib().admm_learn_solve(self.L, _p(bb, _f), _p(x, _f), tol, maxit, ctypes.byref(it))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_learn_solve")
        return x, it.value

    def loss_grad(self, omega, beta, m, theta, b, xc, xl, xs):
        """Mean |x_K - x*|_A^2 / |x_c - x*|_A^2 (+ residual_weight |b - A x_K|^2 / |b - A x_c|^2)
        over the samples and its gradients (omega, beta, m, theta)."""
        K = len(omega)
        om = np.ascontiguousarray(omega, np.float32)
        be = np.ascontiguousarray(beta, np.float32)
        mm = np.ascontiguousarray(m, np.float32)
        th = np.ascontiguousarray(theta, np.float32)
        arrs = [np.ascontiguousarray(a, np.float32) for a in (b, xc, xl, xs)]
        S = arrs[0].shape[0]
        loss = ctypes.c_double()
        go, gb = np.zeros(K, np.float32), np.zeros(K, np.float32)
        gm, gt = np.zeros(self.sysm.n, np.float32), np.zeros(self.sysm.n, np.float32)
        rc = _lib().admm_learn_loss_grad(self.L, K, _p(om, _f), _p(be, _f), _p(mm, _f), _p(th, _f), S,
                                         *[_p(a, _f) for a in arrs], ctypes.byref(loss), _p(go, _f), _p(gb, _f),
                                         _p(gm, _f), _p(gt, _f))
        if rc != B.OK:
            raise B.AdmmError(rc, "admm_learn_loss_grad")
        return loss.value, go, gb, gm, gt


def global_samples(h: "B.Handle", trainer: SweepTrainer, count: int, iterations: Sequence[int],
                   tol: float = 1e-6, max_substeps: Optional[int] = None) -> Tuple[np.ndarray, ...]:
    """(b, x_c, x_l, x*) samples of the global step from plain substeps: substep f records
    global step iterations[f % len(iterations)] (every recording is one substep of the
    simulation); x* by conjugate gradients on the GPU.  A sample whose x_c is already the
    solution to FP32 precision (max |x_c - x*| <= 20 eps32 max(1, max |x*|), e.g. a free-fall
    frame) carries no error to learn from and is dropped; recording continues until `count`
    samples or max_substeps (default 3 count) substeps."""
    bs, xcs, xls, xss = [], [], [], []
    limit = 3 * count if max_substeps is None else max_substeps
    eps = 20.0 * float(np.finfo(np.float32).eps)
    f = 0
    while len(bs) < count and f < limit:
        it = int(iterations[f % len(iterations)])
        f += 1
        b, xc, xl = h.record_global(it, allow=(B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW))
        xs, _ = trainer.solve(b, xc, tol)
        if np.abs(xc - xs).max() <= eps * max(1.0, float(np.abs(xs).max())):
            continue
        bs.append(b)
        xcs.append(xc)
        xls.append(xl)
        xss.append(xs)
    n = trainer.sysm.n
    if not bs:
        z = np.zeros((0, n, 3), np.float32)
        return z, z.copy(), z.copy(), z.copy()
    return tuple(np.array(a, np.float32) for a in (bs, xcs, xls, xss))


def chebyshev_coefficients(K: int, lo: float, hi: float) -> Tuple[np.ndarray, np.ndarray]:
    """(omega, beta) of K steps of the three-term Chebyshev iteration for the spectrum
    [lo, hi] of the preconditioned matrix (Saad, Iterative Methods, Alg. 12.1)."""
    theta = (hi + lo) / 2.0
    delta = (hi - lo) / 2.0
    sigma = theta / delta
    rho = 1.0 / sigma
    om, be = [1.0 / theta], [0.0]
    for _ in range(1, K):
        rn = 1.0 / (2.0 * sigma - rho)
        om.append(2.0 * rn / delta)
        be.append(rn * rho)
        rho = rn
    return np.array(om, np.float32), np.array(be, np.float32)


def jacobi_spectrum_top(sysm: System, iters: int = 60, seed: int = 0) -> float:
    """Largest eigenvalue of D^-1 A by the power method (host, FP64)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(sysm.n, 1))
    d = sysm.diag.astype(np.float64)
    lam = 1.0
    for _ in range(iters):
        w = sysm.matvec(np.repeat(v, 3, 1))[:, :1] / d[:, None]
        lam = float(np.linalg.norm(w) / max(np.linalg.norm(v), 1e-300))
        v = w / max(np.linalg.norm(w), 1e-300)
    return lam


class LearnedGlobalStep:
    """The learned global step: the network (per-vertex m and warm-start theta) and the
    per-sweep coefficients (omega, beta), trained together on the error after K sweeps.

    Starts as plain Jacobi at the network's side (zero head: m = 1 / a_ii, theta = 0);
    the coefficients start as K steps of Chebyshev on [lo_frac * lam_max, lam_max] of
    D^-1 A (omega = 1, beta = 0 with chebyshev=False)."""

    def __init__(self, K: int = 10, bf16: bool = True, seed: int = 0):
        self.K = K
        self.net = LearnedPreconditioner(bf16=bf16, seed=seed)
        self.omega = np.ones(K, np.float32)
        self.beta = np.zeros(K, np.float32)
        self._m = np.zeros(2 * K)
        self._v = np.zeros(2 * K)
        self._t = 0

    def init_chebyshev(self, lam_max: float, lo_frac: float = 0.1):
        self.omega, self.beta = chebyshev_coefficients(self.K, lo_frac * lam_max, 1.02 * lam_max)

    def outputs(self, sysm: System, x: np.ndarray, ef: np.ndarray):
        return self.net.outputs(sysm, x, ef)

    def fit(self, data, epochs: int = 5, batch: int = 8, lr: float = 1e-3, lr_coef: float = 2e-3,
            seed: int = 0) -> List[float]:
        """data: list of (sysm, node feats, edge feats, SweepTrainer, (b, xc, xl, xs) arrays).
        Adam on the network (GPU) and on the coefficients (host) with the GPU gradients;
        returns the mean loss per epoch."""
        rng = np.random.default_rng(seed)
        hist = []
        for _ in range(epochs):
            tot, cnt = 0.0, 0
            for k in rng.permutation(len(data)):
                sysm, x, ef, tr, S = data[k]
                order = rng.permutation(S[0].shape[0])
                for j in range(0, len(order), batch):
                    sel = order[j:j + batch]
                    m, th = self.net.outputs(sysm, x, ef)
                    loss, go, gb, gm, gt = tr.loss_grad(self.omega, self.beta, m, th, *(a[sel] for a in S))
                    self.net.backward(sysm, x, ef, gm, gt)
                    self.net.step(lr)
                    self._adam_coef(go, gb, lr_coef)
                    tot += loss
                    cnt += 1
            hist.append(tot / max(cnt, 1))
        return hist

    def _adam_coef(self, go, gb, lr, b1=0.9, b2=0.999, eps=1e-8):
        g = np.concatenate([go, gb]).astype(np.float64)
        g[self.K] = 0.0  # beta_0 is not used
        self._t += 1
        self._m = b1 * self._m + (1 - b1) * g
        self._v = b2 * self._v + (1 - b2) * g * g
        step = lr * (self._m / (1 - b1 ** self._t)) / (np.sqrt(self._v / (1 - b2 ** self._t)) + eps)
        self.omega = (self.omega - step[:self.K]).astype(np.float32)
        self.beta = (self.beta - step[self.K:]).astype(np.float32)
        self.beta[0] = 0.0

    def evaluate(self, tr: SweepTrainer, m, th, S) -> float:
        return tr.loss_grad(self.omega, self.beta, m, th, *S)[0]

    def apply(self, h: "B.Handle", sysm: System, x: np.ndarray, ef: np.ndarray):
        """Hand the learned step to a handle created with global_solver 3."""
        m, th = self.net.outputs(sysm, x, ef)
        h.set_learned(self.omega, self.beta, m, th)
        return m, th

    def save(self, path: str):
        np.savez(path, params=self.net.params(), omega=self.omega, beta=self.beta, K=self.K,
                 bf16=int(self.net.bf16))

    @classmethod
    def load(cls, path: str, bf16: Optional[bool] = None) -> "LearnedGlobalStep":
        """A saved model; bf16 None: the precision it was trained in."""
        d = np.load(path)
        if bf16 is None:
            bf16 = bool(int(d["bf16"])) if "bf16" in d else True
        obj = cls(K=int(d["K"]), bf16=bf16)
        obj.net.set_params(d["params"])
        obj.omega = d["omega"].astype(np.float32)
        obj.beta = d["beta"].astype(np.float32)
        return obj


def init_params(seed: int = 0) -> np.ndarray:
    """Scaled normal weights, zero biases, zero head (the network starts as diag(A)^-1)."""
    rng = np.random.default_rng(seed)
    H, F_IN, F_E = 64, 6, 2
    shapes = [(H, F_IN), (H,)]
    for _ in range(3):
        shapes += [(H, 2 * H + F_E), (H,), (H, 2 * H), (H,)]
    shapes += [(7, H), (7,)]
    parts = []
    for s in shapes:
        parts.append(rng.normal(scale=1.0 / np.sqrt(s[1]), size=s) if len(s) == 2 else np.zeros(s))
    parts[-2][:] = 0.0
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)
