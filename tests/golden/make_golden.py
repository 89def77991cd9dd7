"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs the reference's ``src/mutils/svd_fast3.cuh`` (3x3 SVD) and
``src/mutils/dist_g.cuh`` (dcdPT / dcdEE narrow phase), compiled for the host by
``oracle/Makefile`` into ``oracle/_ref/libref_pin.so`` from the reference tree, and its
contact and Jacobi kernels (``src/solver/contact_solver.cu``, ``jacobi_solver.cu``, run on
the host from ``oracle/_ref/libref_solver.so``), on seeded inputs, and stores inputs and
outputs as small .npz fixtures.  The tests
compare the oracle against these files, so they need neither the reference tree
nor the host build at test time.

Usage (in a checkout that has the reference tree and the built oracle):
    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def narrow_phase_cases(rng):
    """Random PT/EE configurations plus hand-placed ones on region boundaries."""
    pts = []
    # random, scaled so that a sizeable fraction lands in region 0
    for _ in range(3000):
        pts.append(rng.normal(size=(4, 3)).astype(np.float32) * np.float32(0.1))
    # near-degenerate / boundary: point above triangle edges and vertices, parallel edges
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    for p in [[0.25, 0.25, 1e-3], [0.5, 0.5, 1e-3], [0.0, 0.3, 1e-3], [0.3, 0.0, 1e-3], [1.0, 0.0, 1e-3],
              [0.5, 0.5 + 1e-7, 1e-4], [0.2, 0.2, 0.0], [-1e-7, 0.5, 1e-3], [0.4999999, 0.5, 2e-3]]:
        pts.append(np.vstack([np.array(p, np.float32), tri]))
    segs = [
        [[0, 0, 0], [1, 0, 0], [0.5, -0.5, 1e-3], [0.5, 0.5, 1e-3]],   # crossing, interior
        [[0, 0, 0], [1, 0, 0], [0, 1e-3, 0], [1, 1e-3, 0]],          # parallel
        [[0, 0, 0], [1, 0, 0], [1, -0.5, 1e-3], [1, 0.5, 1e-3]],      # at an endpoint
        [[0, 0, 0], [1, 0, 0], [0.5, 0, 1e-3], [0.5, 1, 1e-3]],       # T-junction
        [[0, 0, 0], [1, 0, 0], [0.5, -0.5, 0.0], [0.5, 0.5, 0.0]],    # intersecting
    ]
    for s in segs:
        pts.append(np.array(s, np.float32))
    # jittered copies of the boundary cases
    base = list(pts[-14:])
    for b in base:
        for _ in range(20):
            pts.append((b + rng.normal(scale=1e-6, size=b.shape)).astype(np.float32))
    return np.stack(pts)


def main():
    if O.ref_pin() is None:
        raise SystemExit("oracle/_ref/libref_pin.so is missing: build it with `make -C oracle` next to the reference tree")
    rng = np.random.default_rng(20261203)
    X = narrow_phase_cases(rng)
    pt = np.stack([O.dcd_pt(*x, ref=True) for x in X])
    ee = np.stack([O.dcd_ee(*x, ref=True) for x in X])
    np.savez_compressed(os.path.join(HERE, "ref_narrow_phase.npz"), inputs=X, pt=pt, ee=ee)

    F = [rng.normal(size=(3, 3)).astype(np.float32) for _ in range(400)]
    # well-conditioned deformation gradients: R diag(s) Q with s in [0.5, 2]
    for _ in range(400):
        q1 = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        q2 = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        F.append((q1 @ np.diag(rng.uniform(0.5, 2.0, 3)) @ q2).astype(np.float32))
    # triangle-style [F 0] inputs: rank 2, rank 1 and zero
    for _ in range(200):
        a = np.zeros((3, 3), np.float32)
        a[:, :2] = rng.normal(size=(3, 2))
        F.append(a)
    for _ in range(50):
        a = np.zeros((3, 3), np.float32)
        u = rng.normal(size=3)
        a[:, 0] = u
        a[:, 1] = 0.5 * u
        F.append(a.astype(np.float32))
    F.append(np.zeros((3, 3), np.float32))
    F = np.stack(F)
    U, S, V = zip(*[O.svd3_ref(f) for f in F])
    np.savez_compressed(os.path.join(HERE, "ref_svd3.npz"), F=F, U=np.stack(U), S=np.stack(S), V=np.stack(V))
    print("wrote", len(X), "narrow-phase cases and", len(F), "SVD cases")
    if O.ref_solver() is None:
        raise SystemExit("oracle/_ref/libref_solver.so is missing: build it with `make -C oracle` next to the reference tree")
    np.savez_compressed(os.path.join(HERE, "ref_contact_jacobi.npz"), **contact_jacobi_cases(rng))
    print("wrote the contact and Jacobi cases")


def contact_jacobi_cases(rng):
    """Inputs and the reference kernels' outputs for S_c / Gamma / K_c (compute_Scc_kernel),
    the friction-cone projection (get_delta_u_kernel), the per-vertex gather (update_p) and
    one Jacobi sweep (JacobiFunctor): random contacts over 300 vertices (the last 50 static,
    w = 1e8), normals of unit length, p and r_c spread so that separating, sticking and
    sliding contacts all occur; a random sparse symmetric system of 500 rows."""
    nv, nd, nc = 300, 250, 1000
    v4 = np.stack([rng.choice(nv, 4, replace=False) for _ in range(nc)]).astype(np.int32)
    bary = rng.normal(size=(nc, 4)).astype(np.float32)
    nrm = rng.normal(size=(nc, 3))
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    gap = rng.uniform(-1e-3, 1e-3, nc).astype(np.float32)
    w = rng.uniform(10.0, 1000.0, nv).astype(np.float32)
    w[nd:] = 1e8
    winv = (1.0 / w).astype(np.float32)
    eps, gam, dt_inv, mu = np.float32(1e-6), np.float32(0.5), np.float32(100.0), np.float32(0.4)
    G, K, inv, gi = O.scc(v4, bary, gap, nrm, w, winv, eps, gam, dt_inv, ref=True)
    p = rng.normal(size=(nv, 3)).astype(np.float32)
    rc = rng.normal(scale=0.5, size=(nc, 3)).astype(np.float32)
    # the first 600 contacts: r_c chosen so that u* = u - r_c is compressive with a tangential
    # part well inside (sticking) or well outside (sliding) the cone
    u = np.einsum("ck,ckj->cj", bary.astype(np.float64), p[v4].astype(np.float64)) + K
    t = rng.normal(size=(nc, 3))
    t -= np.einsum("cj,cj->c", t, nrm)[:, None] * nrm
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    a = rng.uniform(0.1, 1.0, nc)[:, None]
    scale = np.where(np.arange(nc) < 300, 0.3, 3.0)[:, None] * float(mu)
    target = -a * nrm + scale * a * t
    rc[:600] = (u - target)[:600].astype(np.float32)
    du, rc_after = O.cone_step(float(mu), v4, bary, nrm, p, K, rc, ref=True)
    p_after = O.gather_p(v4, G, du, p, ref_lists=(inv, gi))
    rows = 500
    pairs = {(int(a), int(b)) for a, b in rng.integers(0, rows, size=(3000, 2)) if a != b}
    pairs |= {(b, a) for a, b in pairs}
    pairs = sorted(pairs)
    start = np.zeros(rows + 1, np.int32)
    np.add.at(start, np.array([a for a, _ in pairs]) + 1, 1)
    start = np.cumsum(start).astype(np.int32)
    col = np.array([b for _, b in pairs], np.int32)
    val = (-rng.uniform(0.0, 1.0, len(col))).astype(np.float32)
    diag = rng.uniform(20.0, 40.0, rows).astype(np.float32)
    b = rng.normal(size=(rows, 3)).astype(np.float32)
    x = rng.normal(size=(rows, 3)).astype(np.float32)
    xn = O.jacobi_sweep(start, col, val, diag, b, x, ref=True)
    return dict(v4=v4, bary=bary, normal=nrm, gap=gap, w=w, winv=winv, eps=eps, gam=gam, dt_inv=dt_inv, mu=mu,
                Gamma=G, Kc=K, involved=inv, gamma_i=gi, p=p, rc=rc, du=du, rc_after=rc_after, p_after=p_after,
                start=start, col=col, val=val, diag=diag, b=b, x=x, xn=xn)


if __name__ == "__main__":
    main()
