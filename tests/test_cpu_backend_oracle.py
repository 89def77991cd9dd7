"""The oracle's restatement of the reference's CPU backend (ADMMImplCPU::step_fast,
admm_impl_cpu.cpp:264-359): its exact global solve (FP64 envelope Cholesky of the damped
system) against conjugate gradients run to convergence, its damping against a hand-built
damping matrix, and its substeps in FP64 against FP32 (no GPU)."""
import numpy as np
import scipy.sparse as sp

from oracle import oracle as O
from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene


def _system(o, nd):
    L = O.lib()
    nnz = L.orc_system(o.h, None, None, None, None)
    st = np.zeros(nd + 1, np.int32)
    col = np.zeros(nnz, np.int32)
    val = np.zeros(nnz)
    dg = np.zeros(nd)
    L.orc_system(o.h, st.ctypes.data, col.ctypes.data, val.ctypes.data, dg.ctypes.data)
    return sp.csr_matrix((val, col, st), shape=(nd, nd)) + sp.diags(dg)


def test_exact_solve_equals_converged_cg_without_damping():
    """With the damping off and no contact, a CPU-backend substep (exact solve) equals a
    GPU-backend substep whose global step is CG run to convergence."""
    sc = scene.cloth_on_box(12, seed=1)
    sc.params.enable_contact = False
    sc.params.damp_k_L = 0.0
    a = sc.params
    a.backend_semantics = 1
    oc = O.Oracle(B.DescHolder(sc), double=True)
    a.backend_semantics = 0
    a.global_solver = 1
    a.pcg_iter = 400
    og = O.Oracle(B.DescHolder(sc), double=True)
    for _ in range(5):
        oc.step(1)
        og.step(1)
    xc, xg = oc.read(B.BUF_X0), og.read(B.BUF_X0)
    assert np.abs(xc - xg).max() <= 1e-9, np.abs(xc - xg).max()


def test_damped_matrix_is_a_plus_damping():
    """A_damp - A = dt damp_k_L sum_rows w D_r^T D_r over the triangle and bending rows (pins
    excluded) + dt damp_k_M M, built here from the D rows of the scene."""
    sc = scene.cloth_on_box(8, seed=2)
    nd = sc.n_dyn
    sc.params.damp_k_L, sc.params.damp_k_M = 3e-3, 0.7
    sc.params.backend_semantics = 0
    A0 = _system(O.Oracle(B.DescHolder(sc), double=True), nd)
    sc.params.backend_semantics = 1
    A1 = _system(O.Oracle(B.DescHolder(sc), double=True), nd)
    Dm = np.zeros((nd, nd))
    h = sc.params.dt
    for c in range(len(sc.tri_inds)):
        Bm = sc.tri_binv[c].astype(np.float64).reshape(2, 2)
        for r in range(2):
            row = np.zeros(nd)
            ids = sc.tri_inds[c]
            row[ids[0]] += -(Bm[0, r] + Bm[1, r])
            row[ids[1]] += Bm[0, r]
            row[ids[2]] += Bm[1, r]
            Dm += h * 3e-3 * float(sc.tri_w[c]) * np.outer(row, row)
    for c in range(len(sc.bend_w)):
        row = np.zeros(nd)
        for k in range(sc.bend_offsets[c], sc.bend_offsets[c + 1]):
            row[sc.bend_inds[k]] += float(sc.bend_coeffs[k])
        Dm += h * 3e-3 * float(sc.bend_w[c]) * np.outer(row, row)
    Dm += np.diag(h * 0.7 * sc.mass[:nd].astype(np.float64))
    diff = (A1 - A0).toarray()
    assert np.abs(diff - Dm).max() <= 1e-6 * np.abs(Dm).max()


def test_cpu_backend_substeps_fp64_against_fp32():
    """The pinned cloth over the box in the CPU backend's semantics (exact solves, serial
    Gauss-Seidel contact), 40 frames: every FP32 substep, started from the FP64 state, agrees
    with the FP64 substep within 2e-5 m.  (Free-running, the two drift apart by ~1e-4 m per
    frame: the pinned cloth is stiff, kappa(D^-1 A) ~ 700, and converged solves amplify the FP32
    rounding of the reference's own float arithmetic.)"""
    sc = scene.cloth_on_box(16, seed=0)
    sc.params.backend_semantics = 1
    holder = B.DescHolder(sc)
    o64 = O.Oracle(holder, double=True)
    o32 = O.Oracle(holder, double=False)
    worst = 0.0
    for _ in range(40):
        for buf in (B.BUF_X0, B.BUF_X, B.BUF_V, B.BUF_UE, B.BUF_UC):
            o32.write(buf, o64.read(buf).astype(np.float32).astype(np.float64))
        o64.step(1)
        o32.step(1)
        worst = max(worst, np.abs(o64.read(B.BUF_X0) - o32.read(B.BUF_X0)).max())
    assert worst <= 2e-5, worst
