"""The learned global step (global_solver 3) on the GPU, through the C ABI: the untrained
step is the Jacobi sweep, the substep matches the oracle's restatement, the judge falls back
to the plain Jacobi substep, the training kernels (unrolled sweeps and their adjoint, the
network's outputs and backward pass) match the FP64 restatement, and what training gains.

Tolerances: a substep against the FP64 oracle 1e-5 relative (free fall) and against the
FP32 oracle 1e-4 (contact frames, one substep at a time); losses 1e-4 relative; gradients
2e-3 in relative norm (FP32 accumulation against FP64)."""
import numpy as np
import pytest

from oracle import gnn_oracle as G
from parallel_admm_b200 import backend as B
from parallel_admm_b200 import gnn, scene

pytestmark = pytest.mark.gpu

ALLOW = (B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def _pin(sc):
    sc.params.ell_lanes = 4
    sc.params.jacobi_mode = 1
    return sc


def _schedule(sysm, K=8, seed=0):
    rng = np.random.default_rng(seed)
    om, be = gnn.chebyshev_coefficients(K, 0.1 * 1.6, 1.7)
    m = (rng.uniform(0.9, 1.1, sysm.n) / sysm.diag).astype(np.float32)
    th = rng.uniform(0.0, 0.6, sysm.n).astype(np.float32)
    return om, be, m, th


def test_untrained_learned_step_is_the_jacobi_sweep():
    sc = _pin(scene.cube_on_ground(8))
    hj = B.Handle(sc)
    hl = B.Handle(sc, global_solver=3)
    for _ in range(5):
        hj.step(1, allow=ALLOW)
        hl.step(1, allow=ALLOW)
        assert _rel(hl.get_state()[0], hj.get_state()[0]) <= 1e-5
    st = hl.learned_stats()
    assert st["substeps"] == 5 and st["solves"] == 5 * sc.params.admm_max_iter
    hj.close()
    hl.close()


def test_learned_substep_matches_the_oracle_free_fall():
    from oracle import oracle as O
    sc = _pin(scene.cube_on_ground(8))
    h = B.Handle(sc, global_solver=3)
    sysm = gnn.system(h)
    om, be, m, th = _schedule(sysm)
    h.set_learned(om, be, m, th)
    o = O.Oracle(h.holder, double=True)
    o.set_learned(om, be, m, th)
    for f in range(4):
        h.step(1, allow=ALLOW)
        o.step(1)
        err = _rel(h.get_state()[0], o.read(B.BUF_X0))
        assert err <= 1e-5, (f, err)
    sg, so = h.learned_stats(), o.learned_stats()
    assert sg == so, (sg, so)
    h.close()


def test_learned_substep_matches_the_oracle_with_contact():
    """Bodies released just above the ground: every substep has contacts; each substep is
    started from the GPU's state and compared with the FP32 oracle."""
    from oracle import oracle as O
    sc = _pin(scene.batch_bodies(4, seed=1, vmin=300, vmax=900))
    h = B.Handle(sc, global_solver=3)
    sysm = gnn.system(h)
    om, be, m, th = _schedule(sysm, seed=1)
    h.set_learned(om, be, m, th)
    o = O.Oracle(h.holder, double=False)
    o.set_learned(om, be, m, th)
    seen = 0
    for f in range(6):
        x, v = h.get_state()
        for buf, a in ((B.BUF_X0, x), (B.BUF_X, x), (B.BUF_V, v), (B.BUF_UE, h.read(B.BUF_UE)),
                       (B.BUF_UC, h.read(B.BUF_UC))):
            o.write(buf, a.astype(np.float64))
        st = h.step(1, allow=ALLOW)
        ro = o.step(1)
        seen += st["n_contacts"] > 0
        assert st["n_contacts"] == ro["n_contacts"], (f, st["n_contacts"], ro["n_contacts"])
        err = _rel(h.get_state()[0], o.read(B.BUF_X0))
        assert err <= 1e-4, (f, err)
    assert seen >= 4
    h.close()


def test_judge_falls_back_to_plain_jacobi():
    """A schedule that steps slightly backwards (one sweep with omega = -0.05: the residual
    grows a little, the positions stay near the inertial prediction) fails the judge on a
    deformed cube: every solve is replaced on the device (the IF node of the substep graph)
    by the plain one from the iterate it received, so the substeps are the plain handle's bit
    for bit (lanes per row and the global-step mode pinned, so that both handles sum the
    right-hand side and the sweeps in the same order)."""
    sc = _pin(scene.cube_on_ground(8))
    sc.params.ell_lanes = 4
    sc.params.jacobi_mode = 1
    # one ADMM iteration per substep: its global solve starts from the prediction, whose
    # residual lies far above the judge's FP32 noise floor (1e-5 |b|), so every solve fails;
    # later iterations of a converging substep may start below the floor, where any solve passes
    sc.params.admm_max_iter = 1
    hj = B.Handle(sc)
    hl = B.Handle(sc, global_solver=3)
    rng = np.random.default_rng(0)
    x = sc.verts.copy()
    x[:sc.n_dyn] += rng.normal(scale=2e-3, size=(sc.n_dyn, 3)).astype(np.float32)
    hj.set_state(x)
    hl.set_state(x)
    hl.set_learned(np.full(1, -0.05, np.float32), np.zeros(1, np.float32))
    for _ in range(3):
        hj.step(1, allow=ALLOW)
        hl.step(1, allow=ALLOW)
        xj, vj = hj.get_state()
        xl, vl = hl.get_state()
        assert np.array_equal(xj, xl) and np.array_equal(vj, vl), np.abs(xj - xl).max()
    st = hl.learned_stats()
    assert st["substeps"] == 3 and st["solves"] == 3, st
    assert st["fallbacks"] == st["failed_solves"] == 3, st
    hj.close()
    hl.close()


def _impact_cube(n, seed=0):
    """A cube 3 cm above the ground at the speed of a 1 m drop: contact from the first frame,
    so the plain global solves leave real errors (free-fall solves converge to FP32 noise)."""
    sc = _pin(scene.cube_on_ground(n, seed=seed, drop=0.0))
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8 * 1.0)
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.03
    return sc, x0, v0


def _samples(h, sysm, tr, count=3, iters=(3, 7, 12)):
    S = gnn.global_samples(h, tr, count, iters)
    assert S[0].shape[0] == count
    A = lambda v: sysm.matvec(v.astype(np.float64))
    for b, xs in zip(S[0], S[3]):
        assert np.linalg.norm(A(xs) - b) <= 1e-4 * np.linalg.norm(b)
    return S


@pytest.mark.parametrize("mu", [0.0, 0.5])
def test_training_gradients_match_the_restatement(mu):
    """The GPU loss and gradients of the unrolled sweeps (learn.cu) against the FP64
    restatement, without and with the residual term of weight mu."""
    sc, x0, v0 = _impact_cube(6, seed=2)
    h = B.Handle(sc)
    h.set_state(x0, v0)
    sysm = gnn.system(h)
    tr = gnn.SweepTrainer(sysm, residual_weight=mu)
    S = _samples(h, sysm, tr)
    assert np.abs(S[1] - S[2]).max() > 0  # x_cur and x_last differ
    om, be, m, th = _schedule(sysm, K=6, seed=3)
    loss, go, gb, gm, gt = tr.loss_grad(om, be, m, th, *S)
    d = lambda a: np.asarray(a, np.float64)
    samples = [tuple(d(a[k]) for a in S) for k in range(S[0].shape[0])]
    lo, go_, gb_, gm_, gt_ = G.sweeps_loss_grad(d(m), d(th), d(om), d(be), sysm.start, sysm.col, d(sysm.val),
                                                d(sysm.diag), samples, mu=mu)
    assert abs(loss - lo) <= 1e-3 * abs(lo), (loss, lo)
    for a, b_ in ((go, go_), (gb, gb_), (gm, gm_), (gt, gt_)):
        assert np.linalg.norm(a - b_) <= 2e-3 * np.linalg.norm(b_), np.linalg.norm(a - b_) / np.linalg.norm(b_)
    tr.close()
    h.close()


def test_network_outputs_and_backward_match_the_restatement():
    sc = scene.cube_on_ground(5, seed=4)
    h = B.Handle(sc)
    sysm = gnn.system(h)
    x, ef = gnn.scene_features(sc, sysm)
    rng = np.random.default_rng(6)
    theta = G.init_params(2) + rng.normal(scale=0.03, size=G.n_params())
    net = gnn.LearnedPreconditioner(bf16=False)
    net.set_params(theta.astype(np.float32))
    m, th = net.outputs(sysm, x, ef)
    th32 = theta.astype(np.float32).astype(np.float64)
    d = lambda a: np.asarray(a, np.float64)
    mo, tho, c = G.outputs(th32, d(x), d(ef), sysm.start, sysm.col, d(sysm.diag))
    assert np.abs(m - mo).max() <= 1e-4 * np.abs(mo).max()
    assert np.abs(th - tho).max() <= 1e-4
    gm = rng.normal(size=sysm.n).astype(np.float32)
    gt = rng.normal(size=sysm.n).astype(np.float32)
    grad = net.backward(sysm, x, ef, gm, gt)
    gB = np.zeros((sysm.n, 3, 3))
    for k in range(3):
        gB[:, k, k] = d(gm) / 3.0
    ref = G.backward(th32, d(x), sysm.start, sysm.col, c, G.head_grad(c, d(sysm.diag), gB, d(gt)))
    assert np.linalg.norm(grad - ref) <= 2e-3 * np.linalg.norm(ref), np.linalg.norm(grad - ref) / np.linalg.norm(ref)
    net.close()
    h.close()


def test_training_gains_over_jacobi():
    """Train the learned step (network + schedule, K = 10) on samples of plain runs of cubes
    (E, drop and rotation per seed), then on held-out cubes of the same family compare its
    own error after its 10 sweeps (|x_K - x*|_A^2 / |x_c - x*|_A^2 of the global step, no
    fallback involved) with 10 plain Jacobi sweeps (the same kernel count) and report the
    untrained solver (zero head, Chebyshev schedule) and the reference's 20 Jacobi sweeps."""
    K = 10

    def family(seed):
        rng = np.random.default_rng(1000 + seed)
        return _pin(scene.cube_on_ground(6, seed=seed, drop=float(rng.uniform(0.05, 0.3)), rotate=True))

    data = []
    for seed in range(6):
        sc = family(seed)
        h = B.Handle(sc)
        sysm = gnn.system(h)
        x, ef = gnn.scene_features(sc, sysm)
        h.step(3, allow=ALLOW)
        tr = gnn.SweepTrainer(sysm)
        data.append((sysm, x, ef, tr, gnn.global_samples(h, tr, 16, (1, 2, 4, 8, 15, 25), max_substeps=60)))
        h.close()
    model = gnn.LearnedGlobalStep(K=K)
    model.init_chebyshev(gnn.jacobi_spectrum_top(data[0][0]))
    om0, be0 = model.omega.copy(), model.beta.copy()
    hist = model.fit(data, epochs=6, batch=8, lr=5e-4, lr_coef=5e-4)
    assert hist[-1] < hist[0], hist
    res = {"learned": [], "untrained": [], "jacobi_same_sweeps": [], "jacobi20": [], "fallbacks": []}
    for seed in (100, 101, 102, 103):
        sc = family(seed)
        h = B.Handle(sc)
        sysm = gnn.system(h)
        x, ef = gnn.scene_features(sc, sysm)
        h.step(3, allow=ALLOW)
        tr = gnn.SweepTrainer(sysm)
        S = gnn.global_samples(h, tr, 8, (2, 5, 10, 20), max_substeps=40)
        assert S[0].shape[0] > 0
        m, th = model.outputs(sysm, x, ef)
        jm = (1.0 / sysm.diag).astype(np.float32)
        z = np.zeros(sysm.n, np.float32)
        res["learned"].append(tr.loss_grad(model.omega, model.beta, m, th, *S)[0])
        res["untrained"].append(tr.loss_grad(om0, be0, jm, z, *S)[0])
        res["jacobi_same_sweeps"].append(tr.loss_grad(np.ones(K, np.float32), np.zeros(K, np.float32), jm, z, *S)[0])
        res["jacobi20"].append(tr.loss_grad(np.ones(20, np.float32), np.zeros(20, np.float32), jm, z, *S)[0])
        # the trained step in a substep: finite, judged
        sc.params.global_solver = 3
        h3 = B.Handle(sc)
        model.apply(h3, gnn.system(h3), x, ef)
        h3.step(3, allow=ALLOW)
        assert np.isfinite(h3.get_state()[0]).all()
        res["fallbacks"].append(h3.learned_stats()["fallbacks"])
        h3.close()
        tr.close()
        h.close()
    mean = {k: float(np.mean(v)) for k, v in res.items()}
    print("training loss per epoch", [f"{v:.3e}" for v in hist], "held-out A-norm error ratio after the solve:",
          {k: f"{v:.3e}" for k, v in mean.items()})
    assert mean["learned"] < mean["jacobi_same_sweeps"]
    for _, _, _, tr, _ in data:
        tr.close()
    model.net.close()


def test_training_script_end_to_end(tmp_path):
    """The training script that makes the committed weights, at a tiny scale: it trains the
    models of every sweep count, evaluates held-out seeds with fallback counts, writes the
    chosen model and a JSON summary, and the written model loads and runs in a substep."""
    import json
    import os
    import subprocess
    import sys
    out = tmp_path / "w.npz"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-m", "parallel_admm_b200.train_learned", "--out", str(out), "--n", "6",
                        "--train-seeds", "3", "--samples", "8", "--eval-seeds", "10", "--eval-samples", "2",
                        "--eval-substeps", "3", "--sweeps", "6,10"], cwd=root, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    summary = json.loads(r.stdout.strip().splitlines()[-1])
    assert summary["train"]["triples"] > 0 and summary["eval"]["evaluated_seeds"] > 0
    assert summary["chosen_sweeps"] in (6, 10)
    for K in ("6", "10"):
        assert summary["models"][K]["judged"]["substeps"] > 0
    model = gnn.LearnedGlobalStep.load(str(out))
    sc = _pin(scene.cube_on_ground(6, drop=0.02))
    sc.params.global_solver = 3
    h = B.Handle(sc)
    sysm = gnn.system(h)
    model.apply(h, sysm, *gnn.scene_features(sc, sysm))
    h.step(2, allow=ALLOW)
    assert np.isfinite(h.get_state()[0]).all()
    model.net.close()
