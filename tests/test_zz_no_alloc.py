"""admm_b200_jacobi_noalloc: the Jacobi solve for callers that cannot allocate device memory.

Such callers (their device memory is owned by their own pool allocator, or cudaMalloc's
latency and implicit synchronisation are not acceptable in their loop) pass the matrix,
right-hand side and positions in their own device buffers; the entry point's scratch is a
static device array.  Checked through the C ABI against the handle path
(admm_b200_jacobi on the same system) on two calls in a row, within the 1e-5 relative
tolerance of the other solver tests.  This file is collected last (test_zz_*).
"""
import ctypes

import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _system_matrix(sc):
    """A = M + h^2 D^T W^2 D + h^2 W_c (off-diagonal CSR + diagonal), assembled in float64."""
    h2 = float(sc.params.dt) ** 2
    rows_i, rows_v, rows_w = [], [], []
    for c in range(len(sc.tet_inds)):
        Bm = sc.tet_binv[c].astype(np.float64).reshape(3, 3)
        for r in range(3):
            rows_i.append(sc.tet_inds[c])
            rows_v.append([-(Bm[0, r] + Bm[1, r] + Bm[2, r]), Bm[0, r], Bm[1, r], Bm[2, r]])
            rows_w.append(float(sc.tet_w[c]))
    for c in range(len(sc.tri_inds)):
        Bm = sc.tri_binv[c].astype(np.float64).reshape(2, 2)
        for r in range(2):
            rows_i.append(sc.tri_inds[c])
            rows_v.append([-(Bm[0, r] + Bm[1, r]), Bm[0, r], Bm[1, r]])
            rows_w.append(float(sc.tri_w[c]))
    for c in range(len(sc.bend_w)):
        a, b = sc.bend_offsets[c], sc.bend_offsets[c + 1]
        rows_i.append(sc.bend_inds[a:b])
        rows_v.append(sc.bend_coeffs[a:b].astype(np.float64))
        rows_w.append(float(sc.bend_w[c]))
    for c in range(len(sc.pin_inds)):
        rows_i.append([sc.pin_inds[c]])
        rows_v.append([1.0])
        rows_w.append(float(sc.pin_w[c]))
    nd = sc.n_dyn
    acc = {}
    diag = sc.mass[:nd].astype(np.float64).copy()
    if sc.params.enable_contact:
        surf = np.zeros(sc.n_vert, bool)
        surf[sc.surf_verts] = True
        cw32 = (h2 * sc.contact_w[:nd].astype(np.float64)).astype(np.float32).astype(np.float64)
        diag += np.where(surf[:nd], cw32, 0.0)
    for ids, vals, w in zip(rows_i, rows_v, rows_w):
        s = w * w * h2
        for ia, va in zip(ids, vals):
            for ib, vb in zip(ids, vals):
                if ia == ib:
                    diag[ia] += s * va * vb
                else:
                    acc[(int(ia), int(ib))] = acc.get((int(ia), int(ib)), 0.0) + s * va * vb
    keys = sorted(acc)
    start = np.zeros(nd + 1, np.int32)
    for (i, _j) in keys:
        start[i + 1] += 1
    start = np.cumsum(start).astype(np.int32)
    cols = np.array([j for (_i, j) in keys], np.int32)
    vals = np.array([acc[k] for k in keys], np.float32)
    return start, cols, vals, diag.astype(np.float32)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_jacobi_matches_handle_path_twice():
    import torch
    torch.cuda.set_device(0)
    sc = scene.cube_on_ground(8)
    nd = sc.n_dyn
    h = B.Handle(sc)
    start, cols, vals, diag = _system_matrix(sc)
    dev = torch.device("cuda:0")
    t_start = torch.from_numpy(start).to(dev)
    t_cols = torch.from_numpy(cols).to(dev)
    t_vals = torch.from_numpy(vals).to(dev)
    t_diag = torch.from_numpy(diag).to(dev)
    rng = np.random.default_rng(0)
    for call, sweeps in enumerate((20, 7)):
        b = rng.normal(size=(nd, 3)).astype(np.float32) * np.float32(0.1)
        x = sc.verts[:nd] + rng.normal(scale=1e-3, size=(nd, 3)).astype(np.float32)
        # the existing entry point: admm_b200_jacobi on the handle's copy of A
        xh = np.zeros((sc.n_vert, 3), np.float32)
        xh[:nd] = x
        xh[nd:] = sc.verts[nd:]
        h.write(B.BUF_X, xh)
        h.write(B.BUF_B, b)
        h.jacobi(sweeps)
        ref = h.read(B.BUF_X)[:nd]
        # the allocation-free entry point on caller-owned buffers
        t_b = torch.from_numpy(b).to(dev)
        t_x = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        t_out = torch.empty_like(t_x)
        stream = torch.cuda.current_stream().cuda_stream
        rc = B.lib().admm_b200_jacobi_noalloc(nd, _ptr(t_start), _ptr(t_cols), _ptr(t_vals), _ptr(t_diag),
                                             _ptr(t_b), _ptr(t_x), _ptr(t_out), sweeps, ctypes.c_void_p(stream))
        assert rc == B.OK, (call, rc)
        torch.cuda.synchronize()
        got = t_out.cpu().numpy()
        err = np.abs(got - ref).max() / max(1.0, np.abs(ref).max())
        assert err <= TOL, (call, sweeps, err)
    # in place (x_out == x_in): no sweep (nothing to do), one sweep (through the scratch, then a
    # copy back) and two sweeps, each against the handle path
    for sweeps in (0, 1, 2):
        b = rng.normal(size=(nd, 3)).astype(np.float32) * np.float32(0.1)
        x = sc.verts[:nd] + rng.normal(scale=1e-3, size=(nd, 3)).astype(np.float32)
        xh = np.zeros((sc.n_vert, 3), np.float32)
        xh[:nd] = x
        xh[nd:] = sc.verts[nd:]
        h.write(B.BUF_X, xh)
        h.write(B.BUF_B, b)
        if sweeps:
            h.jacobi(sweeps)
        ref = h.read(B.BUF_X)[:nd]
        t_b = torch.from_numpy(b).to(dev)
        t_x = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        stream = torch.cuda.current_stream().cuda_stream
        rc = B.lib().admm_b200_jacobi_noalloc(nd, _ptr(t_start), _ptr(t_cols), _ptr(t_vals), _ptr(t_diag),
                                             _ptr(t_b), _ptr(t_x), _ptr(t_x), sweeps, ctypes.c_void_p(stream))
        assert rc == B.OK, ("in place", sweeps, rc)
        torch.cuda.synchronize()
        got = t_x.cpu().numpy()
        err = np.abs(got - ref).max() / max(1.0, np.abs(ref).max())
        assert err <= TOL, ("in place", sweeps, err)
    # sizes beyond the static scratch are rejected, nothing is launched
    rc = B.lib().admm_b200_jacobi_noalloc(262145, _ptr(t_start), _ptr(t_cols), _ptr(t_vals), _ptr(t_diag),
                                         _ptr(t_b), _ptr(t_x), _ptr(t_out), 1, None)
    assert rc == B.ERR_INVALID
