"""The learned block preconditioner on the GPU: forward and gradients against the FP64
restatement, BF16 weights, training, and what the trained network gains in the PCG solve."""
import numpy as np
import pytest

from oracle import gnn_oracle as G
from parallel_admm_b200 import backend as B
from parallel_admm_b200 import gnn, scene

pytestmark = pytest.mark.gpu


def _cube_system(n=5, seed=0, **kw):
    sc = scene.cube_on_ground(n, seed=seed, **kw)
    h = B.Handle(sc)
    sysm = gnn.system(h)
    x, ef = gnn.scene_features(sc, sysm)
    return sc, h, sysm, x, ef


def test_gradient_matches_the_restatement():
    sc, h, sysm, x, ef = _cube_system(5)
    rng = np.random.default_rng(0)
    theta = G.init_params(1) + rng.normal(scale=0.02, size=G.n_params())
    R = rng.normal(size=(3, sysm.n, 3))
    net = gnn.LearnedPreconditioner(bf16=False)
    net.set_params(theta.astype(np.float32))
    loss, grad = net.loss_grad(sysm, x, ef, R.astype(np.float32))
    th32 = theta.astype(np.float32).astype(np.float64)
    lo, go = G.loss_and_grad(th32, x.astype(np.float64), ef.astype(np.float64), sysm.start, sysm.col,
                             sysm.val.astype(np.float64), sysm.diag.astype(np.float64), R.astype(np.float32).astype(np.float64))
    assert abs(loss - lo) <= 1e-4 * abs(lo), (loss, lo)
    assert np.linalg.norm(grad - go) <= 2e-3 * np.linalg.norm(go), np.linalg.norm(grad - go) / np.linalg.norm(go)
    Bg = net.blocks(sysm, x, ef).reshape(-1, 3, 3)
    Bo, _ = G.forward(th32, x.astype(np.float64), ef.astype(np.float64), sysm.start, sysm.col,
                      sysm.diag.astype(np.float64))
    assert np.abs(Bg - Bo).max() <= 1e-4 * np.abs(Bo).max()
    net.close()


def _bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), kept as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def test_tensor_core_layers_match_the_restatement():
    """With BF16 weights the 64-output layers run on the tensor cores (tcgen05, TF32 operands,
    FP32 accumulation in tensor memory): the blocks agree with the FP64 restatement evaluated
    with the same BF16-rounded weights, within the TF32 rounding of the activations."""
    sc, h, sysm, x, ef = _cube_system(6, seed=4)
    rng = np.random.default_rng(5)
    theta = (G.init_params(7) + rng.normal(scale=0.05, size=G.n_params())).astype(np.float32)
    net = gnn.LearnedPreconditioner(bf16=True)
    net.set_params(theta)
    Bg = net.blocks(sysm, x, ef).reshape(-1, 3, 3)
    net.close()
    # the restatement with the weights (not the biases) rounded to BF16
    parts, k = [], 0
    for shp in G.param_shapes():
        n = int(np.prod(shp))
        blk = theta[k:k + n]
        parts.append(_bf16(blk) if len(shp) == 2 else blk)
        k += n
    th = np.concatenate(parts).astype(np.float64)
    Bo, _ = G.forward(th, x.astype(np.float64), ef.astype(np.float64), sysm.start, sysm.col,
                      sysm.diag.astype(np.float64))
    err = np.abs(Bg - Bo).max() / np.abs(Bo).max()
    assert err <= 1e-2, err


def test_bf16_weights_stay_close():
    sc, h, sysm, x, ef = _cube_system(5, seed=1)
    rng = np.random.default_rng(2)
    theta = (G.init_params(3) + rng.normal(scale=0.02, size=G.n_params())).astype(np.float32)
    out = []
    for bf in (False, True):
        net = gnn.LearnedPreconditioner(bf16=bf)
        net.set_params(theta)
        out.append(net.blocks(sysm, x, ef))
        net.close()
    assert np.abs(out[0] - out[1]).max() <= 3e-2 * np.abs(out[0]).max()


def test_training_and_what_it_gains():
    """Train on residuals of plain runs of cubes with different E, drops and rotations, then
    count PCG iterations to 1e-4 on held-out cubes: learned blocks against diag(A).  On these
    systems A = (M + h^2 D^T W^2 D + h^2 W_c) (x) I3 is isotropic, so a per-vertex block has
    little room beyond diag(A) and the trained network does not beat it; plain diag(A) judges
    every system and stays in use when the learned blocks are not better (the fallback).  The
    test requires the training loss to fall, the chosen preconditioner never to be worse than
    diag(A), the handle to run with the chosen blocks, and prints the ratios and fallbacks."""
    data = []
    for seed in range(6):
        sc, h, sysm, x, ef = _cube_system(6, seed=seed, drop=float(0.5 + 0.3 * seed), rotate=True)
        R = gnn.global_residuals(h, sysm, 12)
        data.append((sysm, x, ef, R))
        h.close()
    net = gnn.LearnedPreconditioner(bf16=True)
    hist = net.fit(data, epochs=15, lr=2e-3, batch=6)
    assert hist[-1] < hist[0], hist
    ratios, fallbacks = [], 0
    for seed in (100, 101, 102):
        sc, h, sysm, x, ef = _cube_system(6, seed=seed, drop=1.2, rotate=True)
        R = gnn.global_residuals(h, sysm, 6)
        blk, learned, ratio = net.blocks_or_fallback(sysm, x, ef, R[:3])
        ratios.append(ratio)
        fallbacks += 0 if learned else 1
        it_j = np.mean([gnn.pcg_iterations(sysm, None, r.astype(np.float64)) for r in R[:3]])
        it_c = np.mean([gnn.pcg_iterations(sysm, blk, r.astype(np.float64)) for r in R[:3]])
        assert it_c <= it_j
        sc.params.global_solver = 2
        h2 = B.Handle(sc)
        h2.set_preconditioner(blk)
        h2.step(3)
        assert np.isfinite(h2.get_state()[0]).all()
        h2.close()
        h.close()
    print("loss per epoch", [round(v, 5) for v in hist], "PCG iterations learned / diag(A):",
          [round(r, 3) for r in ratios], "fallbacks to diag(A):", fallbacks, "of", len(ratios))
    net.close()
