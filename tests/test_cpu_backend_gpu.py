"""The CUDA substep in the semantics of the reference's CPU backend (backend_semantics 1:
damped system, exact-enough global solve, S_c without contact counts, serial Gauss-Seidel
contact, CPU contact predicates) against the FP64 restatement of that backend
(ADMMImplCPU::step_fast, admm_impl_cpu.cpp:264-359; exact envelope-Cholesky solve of the
damped A, as SimplicialLLT in linear_solver_cpu.h:16-23), on the 32x32 cloth pinned at two
corners over the unit box (the CPU-runnable configuration, 100 frames of dt = 1/200).

Per substep, from the oracle's state: within 1e-4 m on frames where both sides see the
same contacts (the GPU's 150 FP32 conjugate-gradient iterations against the exact FP64
factorisation of a system with kappa(D^-1 A) ~ 700: the FP32 restatement with the exact
solve is 2e-5 m from FP64 per substep).  Over 100 free-running frames the FP32 GPU path drifts from the FP64
oracle by about as much as the FP32 restatement of the same algorithm does (the pinned
cloth is stiff, kappa(D^-1 A) ~ 700, and its converged solves amplify FP32 rounding: the
FP32 and FP64 restatements are 4e-3 apart after 40 frames), so the long run is checked
against that drift, not against 1e-3."""
import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene

pytestmark = pytest.mark.gpu

ALLOW = (B.ERR_CONTACT_OVERFLOW, B.ERR_STACK_OVERFLOW)


def _cloth():
    sc = scene.cloth_on_box(32, seed=0)
    sc.params.backend_semantics = 1
    sc.params.global_solver = 1
    sc.params.pcg_iter = 150
    sc.params.ell_lanes = 4
    return sc


def test_cpu_backend_substeps_match_the_fp64_cpu_oracle():
    from oracle import oracle as O
    sc = _cloth()
    h = B.Handle(sc)
    o = O.Oracle(h.holder, double=True)
    errs, contacts = [], 0
    for f in range(100):
        x0, v0 = o.read(B.BUF_X0), o.read(B.BUF_V)
        h.set_state(x0.astype(np.float32), v0.astype(np.float32))
        h.write(B.BUF_UE, o.read(B.BUF_UE).astype(np.float32))
        h.write(B.BUF_UC, o.read(B.BUF_UC).astype(np.float32))
        sg = h.step(1, allow=ALLOW)
        so = o.step(1)
        contacts += sg["n_contacts"] > 0 or so["n_contacts"] > 0
        errs.append((np.abs(h.get_state()[0] - o.read(B.BUF_X0)).max(), sg["n_contacts"] == so["n_contacts"]))
    same = [e for e, eq in errs if eq]
    print(f"CPU-backend semantics, per substep from the FP64 oracle's state: median {np.median(same):.2e}, "
          f"max {max(same):.2e} over {len(same)} frames with equal contact counts; frames with contact {contacts}")
    assert len(same) >= 90
    assert max(same) <= 1e-4, max(same)


def test_cpu_backend_100_frames_drift_is_the_fp32_drift():
    from oracle import oracle as O
    sc = _cloth()
    h = B.Handle(sc)
    o64 = O.Oracle(h.holder, double=True)
    o32 = O.Oracle(h.holder, double=False)
    dg, do = 0.0, 0.0
    for f in range(100):
        h.step(1, allow=ALLOW)
        o64.step(1)
        o32.step(1)
        ref = o64.read(B.BUF_X0)
        dg = max(dg, np.abs(h.get_state()[0] - ref).max())
        do = max(do, np.abs(o32.read(B.BUF_X0) - ref).max())
    print(f"CPU-backend semantics, 100 frames: GPU FP32 vs FP64 oracle {dg:.2e} m, FP32 oracle vs FP64 oracle {do:.2e} m")
    assert np.isfinite(dg)
    assert dg <= 2.0 * do + 1e-3, (dg, do)
