"""The learned global step's safety rules on the CPU oracle (no GPU).

The learned step trained on the dropped-cube family, applied to bodies of the batch it never
saw: its warm start overshoots there (theta about 1, a residual up to 3.5x the received
iterate's).  Judged against the residual of the iterate each global step received, with the
warm start switched off for the rest of a substep once it raised the residual, the substeps
stay bounded and no solve needs replacing.  (Judged against the warm start itself, the same
run grew the ADMM iterate by a factor of about 2.5 per iteration and reached 1e6 m within
one frame.)"""
import os

import numpy as np

from oracle import gnn_oracle as G
from oracle import oracle as O
from parallel_admm_b200 import backend as B
from parallel_admm_b200 import gnn, scene

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "parallel_admm_b200", "weights",
                       "learned_step_cube.npz")


def test_cube_model_on_batch_bodies_stays_bounded():
    sc = scene.batch_bodies(256, seed=0, only=list(range(8)))
    sc.params.global_solver = 3
    hold = B.DescHolder(sc)
    o64 = O.Oracle(hold, double=True)
    A = o64.system()
    o64.close()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    off = A.indices != rows
    start = np.zeros(A.shape[0] + 1, np.int32)
    np.add.at(start, rows[off] + 1, 1)
    sysm = gnn.System(np.cumsum(start).astype(np.int32), A.indices[off], A.data[off], A.diagonal())
    x, ef = gnn.scene_features(sc, sysm)
    d = np.load(WEIGHTS)
    m, th, _ = G.outputs(d["params"].astype(np.float64), x.astype(np.float64), ef.astype(np.float64), sysm.start,
                         sysm.col, sysm.diag.astype(np.float64))
    assert np.percentile(th, 50) > 0.5  # the overshooting warm start
    o = O.Oracle(hold, double=False)
    o.set_learned(d["omega"], d["beta"], m.astype(np.float32), th.astype(np.float32))
    x_init = o.read(B.BUF_X0)[:sc.n_dyn].copy()
    ext0 = np.ptp(x_init, axis=0).max()
    for _ in range(2):
        o.step(1)
        xs = o.read(B.BUF_X0)[:sc.n_dyn]
        assert np.isfinite(xs).all()
        assert np.ptp(xs, axis=0).max() <= 1.01 * ext0
        assert xs[:, 1].min() > -0.01
    st = o.learned_stats()
    assert st["substeps"] == 2 and st["solves"] == 2 * sc.params.admm_max_iter, st
    assert st["fallbacks"] == st["failed_solves"]
