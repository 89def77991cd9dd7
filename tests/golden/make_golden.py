"""Generate the golden vectors in tests/golden/ from the reference's own code.

Runs the reference's ``src/mutils/svd_fast3.cuh`` (3x3 SVD) and
``src/mutils/dist_g.cuh`` (dcdPT / dcdEE narrow phase), compiled for the host by
``oracle/Makefile`` into ``oracle/_ref/libref_pin.so`` from the reference tree, on
seeded inputs, and stores inputs and outputs as small .npz fixtures.  The tests
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


if __name__ == "__main__":
    main()
