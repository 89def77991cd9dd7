"""ctypes front-end of the oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``liboracle_admm.so``, built from ``oracle/admm_oracle.cpp``) is a CPU
restatement of the reference's GPU ADMM substep.  It is the checker of the CUDA
library: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module.  ``ref_pin`` exposes the reference's own
``svd_fast3.cuh`` / ``dist_g.cuh`` compiled on the host (``oracle/_ref``), when it
has been built, for pinning the oracle.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_admm.so")
REF_PIN_PATH = os.path.join(HERE, "_ref", "libref_pin.so")

_lib = None
_ref = None

_f = ctypes.POINTER(ctypes.c_float)
_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int32)


def build(force: bool = False) -> None:
    """Compile the oracle (and the reference pin library if the reference tree is present)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "OCXX=g++"], check=True)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, _d, _i]
        L.orc_reset.argtypes = [ctypes.c_void_p]
        L.orc_read.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, ctypes.c_int]
        L.orc_write.argtypes = [ctypes.c_void_p, ctypes.c_int, _d, ctypes.c_int]
        for fn in ("orc_local_step", "orc_pre_integration", "orc_rhs", "orc_contact_step"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.orc_jacobi.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_pcg.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_system.restype = ctypes.c_int
        L.orc_set_preconditioner.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.orc_set_learned.argtypes = [ctypes.c_void_p, ctypes.c_int, _f, _f, _f, _f]
        L.orc_learned_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
        L.orc_detect.restype = ctypes.c_int
        L.orc_detect.argtypes = [ctypes.c_void_p]
        L.orc_contacts.restype = ctypes.c_int
        L.orc_contacts.argtypes = [ctypes.c_void_p, _i, _d, _d, _d, _d, ctypes.c_int]
        L.orc_dcd.restype = ctypes.c_int
        L.orc_dcd.argtypes = [_f, ctypes.c_int, _i, ctypes.c_int, _i, ctypes.c_int, _i, ctypes.c_int,
                              ctypes.c_float, _i, _f, ctypes.c_int]
        L.orc_svd3_d.argtypes = [_d, _d, _d, _d]
        for fn in ("orc_prox_tet_d", "orc_prox_tri_d"):
            getattr(L, fn).argtypes = [_d]
        for fn in ("orc_prox_tet_f", "orc_prox_tri_f"):
            getattr(L, fn).argtypes = [_f]
        L.orc_dcd_pt_f.argtypes = [_f, _f, _f, _f, _f]
        L.orc_dcd_ee_f.argtypes = [_f, _f, _f, _f, _f]
        L.orc_gt_pt_f.argtypes = [_f, _f, _f, _f, _f]
        L.orc_gt_ee_f.argtypes = [_f, _f, _f, _f, _f]
        L.orc_dcd2.restype = ctypes.c_int
        L.orc_dcd2.argtypes = [_f, ctypes.c_int, _i, ctypes.c_int, _i, ctypes.c_int, _i, ctypes.c_int,
                               ctypes.c_float, _i, _f, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_pin():
    """The reference's own SVD / narrow phase compiled on the host, or None."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PIN_PATH):
            return None
        R = ctypes.CDLL(REF_PIN_PATH)
        R.ref_svd3.argtypes = [_f, _f, _f, _f]
        R.ref_dcd_pt_f.argtypes = [_f, _f, _f, _f, _f]
        R.ref_dcd_ee_f.argtypes = [_f, _f, _f, _f, _f]
        R.ref_gt_pt_f.argtypes = [_f, _f, _f, _f, _f]
        R.ref_gt_ee_f.argtypes = [_f, _f, _f, _f, _f]
        _ref = R
    return _ref


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(ct)


class Oracle:
    """Stateful oracle over the same scene description as the CUDA library."""

    def __init__(self, desc_holder, double: bool = True):
        self._holder = desc_holder  # keeps the numpy arrays behind the desc alive
        self.h = lib().orc_create(ctypes.byref(desc_holder.desc), 1 if double else 0)
        self.n_vert = desc_holder.desc.n_vert
        self.n_dyn = desc_holder.desc.n_dyn
        self.n_rows = desc_holder.desc.n_rows

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        pr = ctypes.c_double()
        du = ctypes.c_double()
        nc = ctypes.c_int32()
        it = lib().orc_step(self.h, n, ctypes.byref(pr), ctypes.byref(du), ctypes.byref(nc))
        return {"iters": it, "primal": pr.value, "dual": du.value, "n_contacts": nc.value}

    def reset(self):
        lib().orc_reset(self.h)

    def rows(self, which: int) -> int:
        from parallel_admm_b200 import backend as B
        return {B.BUF_UC: self.n_dyn, B.BUF_B: self.n_dyn, B.BUF_UE: self.n_rows,
                B.BUF_Z: self.n_rows}.get(which, self.n_vert)

    def read(self, which: int) -> np.ndarray:
        n = self.rows(which)
        out = np.zeros((n, 3), np.float64)
        if lib().orc_read(self.h, which, _p(out, _d), n) != 0:
            raise ValueError("bad buffer")
        return out

    def write(self, which: int, a: np.ndarray):
        n = self.rows(which)
        a = np.ascontiguousarray(a, np.float64).reshape(n, 3)
        if lib().orc_write(self.h, which, _p(a, _d), n) != 0:
            raise ValueError("bad buffer")

    def set_learned(self, omega, beta, m=None, theta=None):
        """Learned global step (global_solver 3), the same arguments as the CUDA library's."""
        om = np.ascontiguousarray(omega, np.float32).ravel()
        be = np.ascontiguousarray(beta, np.float32).ravel()
        mm = None if m is None else np.ascontiguousarray(m, np.float32).ravel()
        th = None if theta is None else np.ascontiguousarray(theta, np.float32).ravel()
        lib().orc_set_learned(self.h, len(om), _p(om, _f), _p(be, _f), None if mm is None else _p(mm, _f),
                              None if th is None else _p(th, _f))
        self._learned_keep = (om, be, mm, th)

    def learned_stats(self):
        out = (ctypes.c_longlong * 4)()
        lib().orc_learned_stats(self.h, out)
        return {"substeps": out[0], "fallbacks": out[1], "solves": out[2], "failed_solves": out[3]}

    def local_step(self):
        lib().orc_local_step(self.h)

    def pre_integration(self):
        lib().orc_pre_integration(self.h)

    def rhs(self):
        lib().orc_rhs(self.h)

    def jacobi(self, sweeps: int):
        lib().orc_jacobi(self.h, sweeps)

    def system(self):
        """The constant global-step matrix A as a scipy CSR (nd x nd, FP64 oracle only)."""
        import scipy.sparse as sp
        nnz = lib().orc_system(self.h, None, None, None, None)
        if nnz < 0:
            raise ValueError("system() needs the FP64 oracle")
        start = np.zeros(self.n_dyn + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz, np.float64)
        diag = np.zeros(self.n_dyn, np.float64)
        lib().orc_system(self.h, start.ctypes.data, col.ctypes.data, val.ctypes.data, diag.ctypes.data)
        off = sp.csr_matrix((val, col, start), shape=(self.n_dyn, self.n_dyn))
        return (off + sp.diags(diag)).tocsr()

    def pcg(self, iters: int):
        lib().orc_pcg(self.h, iters)

    def set_preconditioner(self, blocks: np.ndarray):
        blk = np.ascontiguousarray(blocks, np.float32).reshape(-1, 9)
        lib().orc_set_preconditioner(self.h, blk.ctypes.data, blk.shape[0])

    def contact_step(self):
        lib().orc_contact_step(self.h)

    def detect(self) -> int:
        return lib().orc_detect(self.h)

    def contacts(self):
        nc = lib().orc_contacts(self.h, None, None, None, None, None, 0)
        pairs = np.zeros((max(nc, 1), 4), np.int32)
        bary = np.zeros((max(nc, 1), 4))
        nrm = np.zeros((max(nc, 1), 3))
        pt = np.zeros((max(nc, 1), 3))
        gap = np.zeros(max(nc, 1))
        lib().orc_contacts(self.h, _p(pairs, _i), _p(bary, _d), _p(nrm, _d), _p(pt, _d), _p(gap, _d), nc)
        return {"pairs": pairs[:nc], "bary": bary[:nc], "normal": nrm[:nc], "point": pt[:nc], "gap": gap[:nc]}


def dcd(x: np.ndarray, surf_verts, surf_tris, surf_edges, thickness: float, cap: Optional[int] = None,
        semantics: int = 0, static_begin: Optional[int] = None):
    """All contact pairs (int4) on float32 positions, in the oracle's order.  semantics 0: the GPU
    backend's predicates; 1: the CPU backend's (static_begin = first static vertex)."""
    x = np.ascontiguousarray(x, np.float32)
    sv = np.ascontiguousarray(surf_verts, np.int32)
    st = np.ascontiguousarray(surf_tris, np.int32)
    se = np.ascontiguousarray(surf_edges, np.int32)
    sb = len(x) if static_begin is None else int(static_begin)
    L = lib()
    args = (_p(x, _f), len(x), _p(sv, _i), len(sv), _p(st, _i), len(st), _p(se, _i), len(se), float(thickness))
    n = L.orc_dcd2(*args, None, None, 0, int(semantics), sb)
    pairs = np.zeros((max(n, 1), 4), np.int32)
    dist = np.zeros(max(n, 1), np.float32)
    L.orc_dcd2(*args, _p(pairs, _i), _p(dist, _f), n, int(semantics), sb)
    return pairs[:n], dist[:n]


def gt_pt(p, t0, t1, t2, ref: bool = False) -> np.ndarray:
    """The CPU backend's point-triangle closest points (11 floats as dcd_pt)."""
    out = np.zeros(11, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (p, t0, t1, t2)]
    fn = ref_pin().ref_gt_pt_f if ref else lib().orc_gt_pt_f
    fn(*[_p(a, _f) for a in args], _p(out, _f))
    return out


def gt_ee(p0, p1, q0, q1, ref: bool = False) -> np.ndarray:
    """The CPU backend's segment-segment closest points (parameters in slots 2-3)."""
    out = np.zeros(11, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (p0, p1, q0, q1)]
    fn = ref_pin().ref_gt_ee_f if ref else lib().orc_gt_ee_f
    fn(*[_p(a, _f) for a in args], _p(out, _f))
    return out


def dcd_pt(p, t0, t1, t2, ref: bool = False) -> np.ndarray:
    out = np.zeros(11, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (p, t0, t1, t2)]
    fn = ref_pin().ref_dcd_pt_f if ref else lib().orc_dcd_pt_f
    fn(*[_p(a, _f) for a in args], _p(out, _f))
    return out


def dcd_ee(p0, p1, q0, q1, ref: bool = False) -> np.ndarray:
    out = np.zeros(11, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (p0, p1, q0, q1)]
    fn = ref_pin().ref_dcd_ee_f if ref else lib().orc_dcd_ee_f
    fn(*[_p(a, _f) for a in args], _p(out, _f))
    return out


def svd3_ref(F: np.ndarray):
    F = np.ascontiguousarray(F, np.float32).reshape(9)
    U = np.zeros(9, np.float32)
    S = np.zeros(3, np.float32)
    V = np.zeros(9, np.float32)
    ref_pin().ref_svd3(_p(F, _f), _p(U, _f), _p(S, _f), _p(V, _f))
    return U.reshape(3, 3), S, V.reshape(3, 3)


def svd3(F: np.ndarray):
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    U = np.zeros(9)
    S = np.zeros(3)
    V = np.zeros(9)
    lib().orc_svd3_d(_p(F, _d), _p(U, _d), _p(S, _d), _p(V, _d))
    return U.reshape(3, 3), S, V.reshape(3, 3)


def prox_tet(z9, double: bool = True) -> np.ndarray:
    if double:
        a = np.ascontiguousarray(z9, np.float64).copy()
        lib().orc_prox_tet_d(_p(a, _d))
    else:
        a = np.ascontiguousarray(z9, np.float32).copy()
        lib().orc_prox_tet_f(_p(a, _f))
    return a


def prox_tri(z6, double: bool = True) -> np.ndarray:
    if double:
        a = np.ascontiguousarray(z6, np.float64).copy()
        lib().orc_prox_tri_d(_p(a, _d))
    else:
        a = np.ascontiguousarray(z6, np.float32).copy()
        lib().orc_prox_tri_f(_p(a, _f))
    return a


def num_threads() -> int:
    return lib().orc_num_threads()


# --- per-contact / per-row pieces (FP32), pinned to the reference's kernels ---
REF_SOLVER_PATH = os.path.join(HERE, "_ref", "libref_solver.so")
_ref_solver = None


def ref_solver():
    """The reference's contact and Jacobi kernels run on the host (oracle/ref_pin_solver.cpp), or None."""
    global _ref_solver
    if _ref_solver is None:
        if not os.path.exists(REF_SOLVER_PATH):
            return None
        _ref_solver = ctypes.CDLL(REF_SOLVER_PATH)
    return _ref_solver


def _c(a, dt):
    return np.ascontiguousarray(a, dt)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def contact_lists(v4: np.ndarray, nv: int):
    """Per-vertex contact counts and CSR starts of a contact set (v4: nc x 4)."""
    cnt = np.bincount(np.asarray(v4, np.int64).ravel(), minlength=nv).astype(np.int32)
    start = np.zeros(nv + 1, np.int32)
    start[1:] = np.cumsum(cnt)
    return cnt, start


def scc(v4, bary4, gap, normal3, w, winv, eps, gam, dt_inv, ref: bool = False):
    """S_c / Gamma_c / K_c of every contact (GPU-backend form, with per-vertex counts).
    Returns (Gamma [nc x 4], K_c [nc x 3]) and, for the reference, also its per-vertex
    lists (involved contact, Gamma_i) in CSR order."""
    v4, bary4, normal3 = _c(v4, np.int32), _c(bary4, np.float32), _c(normal3, np.float32)
    gap, w, winv = _c(gap, np.float32), _c(w, np.float32), _c(winv, np.float32)
    nc, nv = len(v4), len(w)
    cnt, start = contact_lists(v4, nv)
    G = np.zeros((nc, 4), np.float32)
    K = np.zeros((nc, 3), np.float32)
    f = ctypes.c_float
    if ref:
        R = ref_solver()
        inv = np.zeros(max(int(start[-1]), 1), np.int32)
        gi = np.zeros(max(int(start[-1]), 1), np.float32)
        R.ref_scc_f(ctypes.c_int(nc), _ptr(v4), _ptr(bary4), _ptr(start), _ptr(cnt), _ptr(w), _ptr(winv), _ptr(gap),
                    _ptr(normal3), f(gam), f(eps), f(dt_inv), ctypes.c_int(nv), _ptr(G), _ptr(K), _ptr(inv), _ptr(gi))
        return G, K, inv[:start[-1]], gi[:start[-1]]
    lib().orc_scc_f(ctypes.c_int(nc), _ptr(v4), _ptr(bary4), _ptr(gap), _ptr(normal3), _ptr(cnt), _ptr(w), _ptr(winv),
                    f(eps), f(gam), f(dt_inv), _ptr(G), _ptr(K))
    return G, K


def cone_step(mu: float, v4, bary4, normal3, p, Kc3, rc3, ref: bool = False):
    """One friction-cone projection of every contact: (du [nc x 3], r_c after)."""
    v4, bary4, normal3 = _c(v4, np.int32), _c(bary4, np.float32), _c(normal3, np.float32)
    p, Kc3 = _c(p, np.float32), _c(Kc3, np.float32)
    rc = np.array(rc3, np.float32, copy=True, order="C")
    nc = len(v4)
    du = np.zeros((nc, 3), np.float32)
    if ref:
        ref_solver().ref_delta_u_f(ctypes.c_int(nc), ctypes.c_float(mu), _ptr(v4), _ptr(bary4), _ptr(p), _ptr(Kc3),
                                   _ptr(normal3), _ptr(du), _ptr(rc))
    else:
        mus = np.full(nc, mu, np.float32)
        lib().orc_cone_step_f(ctypes.c_int(nc), _ptr(mus), _ptr(v4), _ptr(bary4), _ptr(normal3), _ptr(p), _ptr(Kc3),
                              _ptr(rc), _ptr(du))
    return du, rc


def gather_p(v4, Gam4, du3, p, ref_lists=None):
    """p + the per-vertex gather of du Gamma over each vertex's contacts (contact order).
    ref_lists = (involved, Gamma_i) runs the reference's update_p on its own lists."""
    v4, Gam4, du3 = _c(v4, np.int32), _c(Gam4, np.float32), _c(du3, np.float32)
    out = np.array(p, np.float32, copy=True, order="C")
    nv = len(out) // 3 if out.ndim == 1 else len(out)
    cnt, start = contact_lists(v4, nv)
    if ref_lists is not None:
        inv, gi = _c(ref_lists[0], np.int32), _c(ref_lists[1], np.float32)
        ref_solver().ref_gather_p_f(ctypes.c_int(nv), _ptr(inv), _ptr(start), _ptr(gi), _ptr(du3), _ptr(out))
        return out
    # the oracle's list: entries 4 c + k in contact order
    vlist = np.zeros(max(int(start[-1]), 1), np.int32)
    fill = start[:-1].copy()
    for c in range(len(v4)):
        for k in range(4):
            v = v4[c, k]
            vlist[fill[v]] = 4 * c + k
            fill[v] += 1
    lib().orc_gather_p_f(ctypes.c_int(nv), _ptr(start), _ptr(vlist), _ptr(Gam4), _ptr(du3), _ptr(out))
    return out


def jacobi_sweep(start, col, val, diag, b, x, ref: bool = False):
    """One Jacobi sweep over CSR rows (off-diagonal part), FP32."""
    start, col = _c(start, np.int32), _c(col, np.int32)
    val, diag, b, x = _c(val, np.float32), _c(diag, np.float32), _c(b, np.float32), _c(x, np.float32)
    rows = len(diag)
    xn = np.zeros((rows, 3), np.float32)
    fn = ref_solver().ref_jacobi_sweep_f if ref else lib().orc_jacobi_sweep_f
    fn(ctypes.c_int(rows), _ptr(start), _ptr(col), _ptr(val), _ptr(diag), _ptr(b), _ptr(x), _ptr(xn))
    return xn
