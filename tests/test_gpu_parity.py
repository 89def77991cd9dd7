"""Parity of the CUDA substep (through the C ABI) against the oracle.

Tolerances (FP32 kernels against the FP64 oracle, on the same inputs):
* local step z, global step x, contact p: max |err| <= 1e-5 * max(1, max|ref|)
  (the per-step bound of the spec);
* one full substep: positions within 1e-5 relative (max |dx| / extent of the body);
* 20 substeps with contact: within 1e-3 relative;
* contact pair sets on identical float positions: identical (bit-exact integer sets).
"""
import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-5
TOL_LONG = 1e-3


def _setup(sc, **over):
    from oracle import oracle as O
    h = B.Handle(sc, **over)
    o = O.Oracle(h.holder, double=True)
    return h, o


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def _perturbed(sc, amp, seed=0):
    rng = np.random.default_rng(seed)
    x = sc.verts.astype(np.float64).copy()
    x[:sc.n_dyn] += rng.normal(scale=amp, size=(sc.n_dyn, 3))
    return x


def _crumpled_cloth(nx=24, seed=3):
    """A cloth folded onto itself so that PT and EE contacts exist."""
    sc = scene.cloth_on_box(nx, seed=seed)
    x = sc.verts.astype(np.float64).copy()
    n = sc.n_dyn
    u = x[:n, 0] - x[:n, 0].min()
    # fold along x: second half lifted and mirrored over the first half
    fold = u > 0.5 * u.max()
    x[:n, 0] = np.where(fold, x[:n, 0].min() + u.max() - u, x[:n, 0])
    x[:n, 1] = np.where(fold, x[:n, 1] + sc.params.thickness * 0.6, x[:n, 1])
    rng = np.random.default_rng(seed)
    x[:n] += rng.normal(scale=sc.params.thickness * 0.2, size=(n, 3))
    return sc, x.astype(np.float32)


@pytest.mark.parametrize("name", ["cloth", "cube"])
def test_local_step_parity(name):
    sc = scene.cloth_on_box(32) if name == "cloth" else scene.cube_on_ground(12)
    h, o = _setup(sc)
    x = _perturbed(sc, 2e-3, seed=1)
    rng = np.random.default_rng(2)
    ue = rng.normal(scale=1e-2, size=(sc.n_rows, 3))
    for tgt in (h, o):
        tgt.write(B.BUF_X, x)
        tgt.write(B.BUF_UE, ue)
        tgt.local_step()
    zg = h.read(B.BUF_Z)
    zo = o.read(B.BUF_Z)
    assert np.isfinite(zg).all()
    assert _rel(zg, zo) <= TOL_STEP, _rel(zg, zo)


@pytest.mark.parametrize("name", ["cloth", "cube"])
def test_global_step_parity(name):
    sc = scene.cloth_on_box(32) if name == "cloth" else scene.cube_on_ground(12)
    h, o = _setup(sc)
    o.pre_integration()
    o.write(B.BUF_X, _perturbed(sc, 1e-3, seed=4) + (o.read(B.BUF_X) - sc.verts))
    o.local_step()
    rng = np.random.default_rng(5)
    o.write(B.BUF_UC, rng.normal(scale=1e-3, size=(sc.n_dyn, 3)))
    p = np.zeros((sc.n_vert, 3))
    p[:sc.n_dyn] = rng.normal(scale=0.1, size=(sc.n_dyn, 3))
    o.write(B.BUF_P, p)
    for b in (B.BUF_X, B.BUF_X0, B.BUF_V, B.BUF_P, B.BUF_UC, B.BUF_UE, B.BUF_Z, B.BUF_MXT):
        h.write(b, o.read(b))
    h.global_step()
    o.rhs()
    o.jacobi(sc.params.jacobi_iter)
    assert _rel(h.read(B.BUF_B), o.read(B.BUF_B)) <= TOL_STEP
    assert _rel(h.read(B.BUF_X), o.read(B.BUF_X)) <= TOL_STEP


def _pairset(pairs, canon=True):
    out = set()
    for p in np.asarray(pairs):
        out.add(tuple(int(v) for v in p))
    return out


def _dcd_case(case):
    if case == "layers_stack":
        # 40 small sheets stacked within one thickness: every query has dozens of
        # partners (more than the count pass records, so the write pass walks again)
        v, f = scene.grid_cloth(6, 0.1)
        bodies = [scene._Body(v + np.array([0.0, 0.5 + 1e-4 * l, 0.0]), f, np.zeros((0, 4), np.int32),
                              0.1, 1e3, 1e-3) for l in range(40)]
        sc = scene.assemble("stack", bodies, [], scene.SolverParams(thickness=5e-3, max_contacts=1_000_000))
        return sc, np.ascontiguousarray(sc.verts, np.float32)
    if case == "cloth_fold":
        sc, x = _crumpled_cloth()
    elif case == "cube_squeezed":
        sc = scene.cube_on_ground(10)
        x = sc.verts.copy()
        # squash the cube into the ground so that PT and EE contacts appear
        x[:sc.n_dyn, 1] = (x[:sc.n_dyn, 1] - x[:sc.n_dyn, 1].min()) * 0.5 - 0.25 * sc.params.thickness
        rng = np.random.default_rng(7)
        x[:sc.n_dyn] += rng.normal(scale=0.2 * sc.params.thickness, size=(sc.n_dyn, 3)).astype(np.float32)
    else:
        sc = scene.cloth_on_box(32)
        x = sc.verts.copy()
        x[:sc.n_dyn, 1] = 0.5 + 0.5 * sc.params.thickness  # lying on the box top
    return sc, np.ascontiguousarray(x, np.float32)


@pytest.mark.parametrize("broad,lanes", [(1, 0), (2, 8), (2, 16), (2, 32)],
                         ids=["lbvh", "grid8", "grid16", "grid32"])
@pytest.mark.parametrize("case", ["cloth_fold", "cube_squeezed", "cloth_flat_on_box", "layers_stack"])
def test_dcd_pairs_bitexact(case, broad, lanes):
    from oracle import oracle as O
    sc, x = _dcd_case(case)
    sc.params.broad_phase = broad
    sc.params.query_lanes = lanes
    h = B.Handle(sc)
    n = h.detect(x)
    ref_pairs, _ = O.dcd(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, sc.params.thickness)
    assert n == len(ref_pairs)
    assert n > 0
    got = h.contacts()
    # identical multisets (a point-triangle tuple can equal an edge-edge tuple)
    assert sorted(map(tuple, got["pairs"].tolist())) == sorted(map(tuple, ref_pairs.tolist()))


@pytest.mark.parametrize("case", ["cloth_fold", "cube_squeezed", "layers_stack"])
def test_grid_query_lanes_same_contact_list(case):
    """The lanes per grid query change only the schedule: the contact list (queries in order,
    each query's partners ascending) and every contact field are identical bit for bit."""
    sc, x = _dcd_case(case)
    sc.params.broad_phase = 2
    out = []
    for lanes in (8, 16, 32):
        sc.params.query_lanes = lanes
        h = B.Handle(sc)
        assert h.detect(x) > 0
        out.append(h.contacts())
        h.close()
    for other in out[1:]:
        for k in out[0]:
            assert np.array_equal(out[0][k], other[k]), k


def test_contact_conversion_and_step_parity():
    sc, x = _crumpled_cloth()
    h, o = _setup(sc)
    x64 = x.astype(np.float64)
    rng = np.random.default_rng(11)
    uc = rng.normal(scale=1e-4, size=(sc.n_dyn, 3))
    for tgt in (h, o):
        tgt.write(B.BUF_X, x64)
        tgt.write(B.BUF_UC, uc)
    n = h.detect()
    assert n == o.detect() and n > 0
    gc, oc = h.contacts(), o.contacts()
    # align by pair tuple
    gi = {tuple(p): i for i, p in enumerate(gc["pairs"].tolist())}
    perm = np.array([gi[tuple(p)] for p in oc["pairs"].tolist()])
    assert np.abs(gc["bary"][perm] - oc["bary"]).max() <= 1e-5
    assert np.abs(gc["normal"][perm] - oc["normal"]).max() <= 1e-4
    assert np.abs(gc["gap"][perm] - oc["gap"]).max() <= 1e-6
    h.contact_step()
    o.contact_step()
    pg, po = h.read(B.BUF_P), o.read(B.BUF_P)
    assert _rel(pg[:sc.n_dyn], po[:sc.n_dyn]) <= 1e-4


def test_full_step_cloth_parity():
    sc = scene.cloth_on_box(32)
    h, o = _setup(sc)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    for k in range(3):
        h.step(1)
        o.step(1)
        xg, _ = h.get_state()
        xo = o.read(B.BUF_X0)
        err = np.abs(xg - xo).max() / ext
        assert err <= TOL_STEP * (k + 1), (k, err)


def test_full_step_cube_contact_parity():
    """The cube right at impact (1 m drop speed).

    Frames 0-2 run free against the FP64 oracle (1e-5 per step).  From frame 3 on, contacts
    at the edge of the thickness band decide differently in FP64 and FP32 (the narrow phase
    is FP32 on both sides of the reference), so frames 3-9 are compared one substep at a time,
    from the oracle's state (positions, velocities, both duals), against the FP32 oracle:
    identical contact counts and positions within 1e-4 relative."""
    from oracle import oracle as O
    sc = scene.cube_on_ground(10, drop=0.0)
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8 * 1.0)
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.03
    h, o = _setup(sc)
    o32 = O.Oracle(h.holder, double=False)
    h.set_state(x0, v0)
    for orc in (o, o32):
        orc.write(B.BUF_X0, x0)
        orc.write(B.BUF_V, v0)
        orc.write(B.BUF_X, x0)
    ext = np.ptp(x0[:sc.n_dyn], axis=0).max()
    ncs = []
    for k in range(3):
        sg = h.step(1)
        so = o.step(1)
        o32.step(1)
        ncs.append((sg["n_contacts"], so["n_contacts"]))
        err = np.abs(h.get_state()[0] - o.read(B.BUF_X0)).max() / ext
        assert err <= TOL_STEP * (k + 1), (k, err, ncs)
    for k in range(3, 10):
        h.set_state(o32.read(B.BUF_X0), o32.read(B.BUF_V))
        h.write(B.BUF_UE, o32.read(B.BUF_UE))
        h.write(B.BUF_UC, o32.read(B.BUF_UC))
        sg = h.step(1)
        so = o32.step(1)
        ncs.append((sg["n_contacts"], so["n_contacts"]))
        assert sg["n_contacts"] == so["n_contacts"], (k, ncs)
        err = np.abs(h.get_state()[0] - o32.read(B.BUF_X0)).max() / ext
        assert err <= 1e-4, (k, err, ncs)
    assert min(c[0] for c in ncs) > 0


def test_long_run_cloth_1e3():
    sc = scene.cloth_on_box(16)
    h, o = _setup(sc)
    h.step(20)
    o.step(20)
    xg, _ = h.get_state()
    xo = o.read(B.BUF_X0)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    assert np.abs(xg - xo).max() / ext <= TOL_LONG


def test_residuals_match_oracle():
    """FP64 residual reductions agree with the oracle above the FP32 noise floor of the state.

    D x - z is formed from FP32 x and z, so relative residuals below ~1e-6 are rounding
    noise (2e-6 absolute allowance); with contact at impact they are far above it.
    """
    sc = scene.cloth_on_box(16)
    h, o = _setup(sc)
    sg = h.step(2)
    so = o.step(2)
    for key in ("primal", "dual"):
        assert np.isfinite(sg[key])
        assert abs(sg[key] - so[key]) <= 0.05 * abs(so[key]) + 2e-6, (key, sg[key], so[key])
    sc = scene.cube_on_ground(8, drop=0.0)
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8)
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.02
    h, o = _setup(sc)
    h.set_state(x0, v0)
    for b, a in ((B.BUF_X0, x0), (B.BUF_X, x0), (B.BUF_V, v0)):
        o.write(b, a)
    sg = h.step(1)
    so = o.step(1)
    assert so["primal"] > 1e-4 and so["n_contacts"] > 0
    for key in ("primal", "dual"):
        assert abs(sg[key] - so[key]) <= 0.05 * abs(so[key]) + 2e-6, (key, sg[key], so[key])


def test_determinism_and_reset():
    sc, _ = _crumpled_cloth(16)
    h1 = B.Handle(sc)
    h2 = B.Handle(sc)
    h1.step(5)
    h2.step(5)
    a, _ = h1.get_state()
    b, _ = h2.get_state()
    assert np.array_equal(a, b)
    h1.reset()
    h1.step(5)
    c, _ = h1.get_state()
    assert np.array_equal(a, c)


def test_contact_overflow_is_reported_and_clamped():
    sc, x = _crumpled_cloth(16)
    sc.params.max_contacts = 8
    h = B.Handle(sc)
    cnt = h.detect(x, allow=(B.ERR_CONTACT_OVERFLOW,))
    assert cnt > 8
    c = h.contacts()
    assert len(c["pairs"]) == 8
    st = h.step(1, allow=(B.ERR_CONTACT_OVERFLOW,))
    assert st["n_contacts"] <= 8
    assert np.isfinite(h.get_state()[0]).all()


def test_no_contact_scene_and_contact_disabled():
    sc = scene.cloth_on_box(8)
    sc.params.enable_contact = False
    h, o = _setup(sc)
    h.step(2)
    o.step(2)
    assert np.abs(h.get_state()[0] - o.read(B.BUF_X0)).max() <= 1e-5


def test_backend_contract_call_order():
    sc = scene.cloth_on_box(8)
    be = B.ADMMBackendB200()
    be.apply_config(admm_max_iter=10)
    be.add_constraints(sc)
    be.addPins([0])
    be.set_constraint_dim(sc.n_rows)
    be.finalize_constraints()
    be.init(sc.verts, sc.mass, sc.params.dt)
    be.set_sync_to_host(False)
    for _ in range(3):
        be.step()
    assert len(be.step_metrics) == 3
    assert be.step_metrics[-1]["admm_iters"] == 10
    v = be.getVertices()
    assert v.shape == (sc.n_vert, 3) and np.isfinite(v).all()
    det = be.collision_detector()
    det.detect(be.getVertices())
    assert det.points().shape == (det.max_slots(), 3)
    be.reset()
    assert np.allclose(be.getVertices(), sc.verts)


def test_refit_rebuild_and_grid_give_the_same_motion():
    """Refitting the BVH between DCDs of a substep changes only traversal cost and the
    order of contacts within a query (so the summation order): one impact substep agrees
    to 1e-5 with the same contact count; three substeps at impact (where rounding can flip
    borderline pairs) agree to the contact tolerance 1e-3."""
    sc = scene.cube_on_ground(8, drop=0.0)
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8)
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.02
    ext = np.ptp(x0[:sc.n_dyn], axis=0).max()
    for nsteps, tol in ((1, TOL_STEP), (3, TOL_LONG)):
        out = []
        for broad, refit in ((1, 0), (1, 1), (2, 0)):
            sc.params.bvh_refit = bool(refit)
            sc.params.broad_phase = broad
            h = B.Handle(sc)
            h.set_state(x0, v0)
            st = h.step(nsteps)
            out.append((h.get_state()[0], st["n_contacts"]))
        assert out[0][1] > 0
        for k in (1, 2):
            if nsteps == 1:
                assert out[0][1] == out[k][1]
            assert np.abs(out[0][0] - out[k][0]).max() / ext <= tol


def test_autotuner_choice_is_valid():
    h = B.Handle(scene.cube_on_ground(12))
    t = h.tuning()
    assert t["jacobi_lanes"] in (1, 2, 4, 8) and t["rhs_lanes"] in (1, 2, 4, 8)
    assert 0 < t["jacobi_ms"] < 10 and 0 < t["rhs_ms"] < 10


@pytest.mark.parametrize("name,tol", [("cloth", 1e-4), ("cube_impact", 1e-4)])
def test_tolerance_mode_matches_oracle(name, tol):
    """residual_tol > 0: chunks of dcd_interval iterations until both relative residuals are
    <= tol (device-side WHILE node); same iteration counts and positions as the oracle."""
    if name == "cloth":
        sc = scene.cloth_on_box(16)
        x0 = v0 = None
    else:
        sc = scene.cube_on_ground(8, drop=0.0)
        v0 = np.zeros_like(sc.verts)
        v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8)
        x0 = sc.verts.copy()
        x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.02
    sc.params.admm_max_iter = 60
    h, o = _setup(sc, residual_tol=tol)
    if x0 is not None:
        h.set_state(x0, v0)
        for b, a in ((B.BUF_X0, x0), (B.BUF_X, x0), (B.BUF_V, v0)):
            o.write(b, a)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    for k in range(2):
        sg = h.step(1)
        so = o.step(1)
        assert sg["iters"] % sc.params.dcd_interval == 0 and 0 < sg["iters"] <= 60
        assert sg["iters"] == so["iters"], (k, sg, so)
        if sg["iters"] < 60:
            assert sg["primal"] <= tol and sg["dual"] <= tol
        xg, _ = h.get_state()
        assert np.abs(xg - o.read(B.BUF_X0)).max() / ext <= TOL_LONG


def test_tolerance_mode_eager_matches_graph():
    """The eager (profiling) path of residual_tol mode takes the same decisions on the host as
    the conditional graph node on the device, and the launch count follows the chunks run."""
    sc = scene.cloth_on_box(16)
    sc.params.admm_max_iter = 40
    hg = B.Handle(sc, residual_tol=1e-4)
    he = B.Handle(sc, residual_tol=1e-4)
    he.set_profiling(True)
    k_min = hg.kernels_per_step()
    for _ in range(3):
        sg = hg.step(1)
        se = he.step(1)
        assert sg["iters"] == se["iters"]
        xg, _ = hg.get_state()
        xe, _ = he.get_state()
        np.testing.assert_array_equal(xg, xe)
        chunks = sg["iters"] // sc.params.dcd_interval
        k = hg.kernels_per_step()
        assert (k > k_min) == (chunks > 1)
    hg.close()
    he.close()


def _cube_at_impact(n=8):
    sc = scene.cube_on_ground(n, drop=0.0)
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -np.sqrt(2 * 9.8)
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.02
    return sc, x0, v0


@pytest.mark.parametrize("mode", [2, 3], ids=["persistent", "tiled"])
@pytest.mark.parametrize("case", ["cloth", "cube_impact", "cube_impact_tol"])
def test_persistent_global_step_bitwise(case, mode):
    """jacobi_mode 2 (RHS and all sweeps in one cooperative kernel, blocks synchronised by
    sweep counters) and jacobi_mode 3 (two sweeps per launch over row tiles with halos in
    shared memory) reproduce jacobi_mode 1 (one kernel per sweep) bit for bit."""
    if case == "cloth":
        sc, x0, v0 = scene.cloth_on_box(24), None, None
    else:
        sc, x0, v0 = _cube_at_impact(10)
    over = {"residual_tol": 1e-4} if case.endswith("_tol") else {}
    sc.params.ell_lanes = 4
    hs = []
    for m in (1, mode):
        sc.params.jacobi_mode = m
        h = B.Handle(sc, **over)
        if x0 is not None:
            h.set_state(x0, v0)
        hs.append(h)
    gm = hs[1].global_mode()
    assert gm["mode"] == ("persistent" if mode == 2 else "tiled")
    assert hs[0].global_mode()["mode"] == "sweeps"
    for k in range(4):
        st = [h.step(1) for h in hs]
        assert st[0]["iters"] == st[1]["iters"] and st[0]["n_contacts"] == st[1]["n_contacts"]
        assert st[1]["status"] == B.OK
        xa, va = hs[0].get_state()
        xb, vb = hs[1].get_state()
        np.testing.assert_array_equal(xa, xb)
        np.testing.assert_array_equal(va, vb)
    for h in hs:
        h.close()


@pytest.mark.parametrize("mode", [2, 3], ids=["persistent", "tiled"])
def test_persistent_jacobi_entry_bitwise(mode):
    """admm_b200_jacobi (standalone sweeps) in both modes, odd and even sweep counts."""
    sc = scene.cube_on_ground(12)
    sc.params.ell_lanes = 2
    rng = np.random.default_rng(21)
    x = _perturbed(sc, 1e-3, seed=22)
    b = rng.normal(size=(sc.n_dyn, 3))
    out = []
    for m in (1, mode):
        sc.params.jacobi_mode = m
        h = B.Handle(sc)
        res = []
        for sweeps in (2, 3, 4, 7):
            h.write(B.BUF_X, x)
            h.write(B.BUF_B, b)
            h.jacobi(sweeps)
            res.append(h.read(B.BUF_X))
        out.append(res)
        h.close()
    for a, c in zip(*out):
        np.testing.assert_array_equal(a, c)


def _global_state(sc, seed=31):
    """A state after pre-integration and one local step, with random contact-free duals."""
    from oracle import oracle as O
    h = B.Handle(sc)
    o = O.Oracle(h.holder, double=True)
    o.pre_integration()
    o.write(B.BUF_X, _perturbed(sc, 1e-3, seed=seed) + (o.read(B.BUF_X) - sc.verts))
    o.local_step()
    for b in (B.BUF_X, B.BUF_X0, B.BUF_V, B.BUF_P, B.BUF_UC, B.BUF_UE, B.BUF_Z, B.BUF_MXT):
        h.write(b, o.read(b))
    return h, o


@pytest.mark.parametrize("name", ["cloth", "cube"])
def test_pcg_global_step_parity(name):
    """global_solver 1: RHS + pcg_iter Chronopoulos-Gear PCG iterations (diag(A)) against the
    oracle's restatement of the same recurrences in FP64 (1e-5 relative)."""
    sc = scene.cloth_on_box(32) if name == "cloth" else scene.cube_on_ground(12)
    sc.params.global_solver = 1
    sc.params.pcg_iter = 10
    h, o = _global_state(sc)
    h.global_step()
    o.rhs()
    o.pcg(10)
    assert _rel(h.read(B.BUF_B), o.read(B.BUF_B)) <= TOL_STEP
    assert _rel(h.read(B.BUF_X), o.read(B.BUF_X)) <= TOL_STEP


def test_pcg_converges_to_the_solution():
    """Many PCG iterations on the GPU reach the solution of A x = b (the oracle's FP64 Jacobi
    iterated to convergence) to FP32 accuracy; 20 Jacobi sweeps on the same cloth system
    remove only a few per cent of the error."""
    sc = scene.cloth_on_box(16)
    sc.params.global_solver = 1
    sc.params.pcg_iter = 120
    h, o = _global_state(sc)
    x0 = o.read(B.BUF_X)
    o.rhs()
    o.jacobi(40000)
    xs = o.read(B.BUF_X)
    h.global_step()
    e = np.abs(h.read(B.BUF_X) - xs).max() / max(1.0, np.abs(xs).max())
    assert e <= 2e-6, e
    o.write(B.BUF_X, x0)
    o.jacobi(20)
    assert np.abs(o.read(B.BUF_X) - xs).max() / max(1.0, np.abs(xs).max()) > 50 * e


def test_pcg_block_preconditioner_parity():
    """global_solver 2 with per-vertex SPD 3x3 blocks (set on both sides) matches the oracle."""
    sc = scene.cube_on_ground(10)
    sc.params.global_solver = 2
    sc.params.pcg_iter = 8
    h, o = _global_state(sc)
    rng = np.random.default_rng(5)
    L = rng.normal(scale=0.2, size=(sc.n_dyn, 3, 3)) + np.eye(3)
    blk = np.einsum("nij,nkj->nik", L, L) * 1e-3
    h.set_preconditioner(blk)
    o.set_preconditioner(blk)
    h.global_step()
    o.rhs()
    o.pcg(8)
    assert _rel(h.read(B.BUF_X), o.read(B.BUF_X)) <= TOL_STEP


def test_pcg_full_step_parity():
    """Whole substeps with the PCG global step, cloth, against the FP64 oracle: 2e-5 per step
    (the Krylov recurrences carry FP32 rounding further than Jacobi sweeps do)."""
    sc = scene.cloth_on_box(32)
    sc.params.global_solver = 1
    h, o = _setup(sc)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    for k in range(3):
        h.step(1)
        o.step(1)
        err = np.abs(h.get_state()[0] - o.read(B.BUF_X0)).max() / ext
        assert err <= 2 * TOL_STEP * (k + 1), (k, err)


def test_batch_with_per_body_friction_parity():
    """A batch of independent bodies (cubes and ellipsoids, per-body E and friction) in one scene,
    with per-vertex friction coefficients: the first substep free against the FP64 oracle
    (1e-5), then three substeps one at a time from the FP32 oracle's state against it (equal
    contact counts; every vertex but at most 0.1% of them within 1e-4, none beyond 5e-3).  One
    detection per substep.  The outliers are the scene's, not the kernels': the FP32 oracle run
    on the same state in another vertex numbering moves one vertex by 1.3e-3 in one substep
    (a contact on the edge of its active/separating switch over the ADMM iterations) while every
    other vertex stays within 1e-5 (test_oracle_order.py)."""
    sc = scene.batch_bodies(6, seed=3, vmin=300, vmax=3000)
    assert sc.vert_mu is not None and len(np.unique(sc.vert_mu[:sc.n_dyn])) > 1
    # one detection per substep: identical pair sets on both sides from a shared state (with
    # the two bodies at 2 m/s a pair flipped at a later detection moves vertices by millimetres)
    sc.params.dcd_interval = sc.params.admm_max_iter
    # start every body just above the ground, moving down, so that contacts appear at once
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.012
    v0 = np.zeros_like(x0)
    v0[:sc.n_dyn, 1] = -2.0
    h, o = _setup(sc)
    h.set_state(x0, v0)
    for b, a in ((B.BUF_X0, x0), (B.BUF_X, x0), (B.BUF_V, v0)):
        o.write(b, a)
    from oracle import oracle as O
    o32 = O.Oracle(h.holder, double=False)
    for b, a in ((B.BUF_X0, x0), (B.BUF_X, x0), (B.BUF_V, v0)):
        o32.write(b, a)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    sg = h.step(1)
    so = o.step(1)
    o32.step(1)
    err = np.abs(h.get_state()[0] - o.read(B.BUF_X0)).max() / ext
    assert err <= TOL_STEP, (err, sg["n_contacts"], so["n_contacts"])
    seen = sg["n_contacts"]
    for k in range(1, 4):
        h.set_state(o32.read(B.BUF_X0), o32.read(B.BUF_V))
        h.write(B.BUF_UE, o32.read(B.BUF_UE))
        h.write(B.BUF_UC, o32.read(B.BUF_UC))
        sg = h.step(1)
        so = o32.step(1)
        assert sg["n_contacts"] == so["n_contacts"], (k, sg["n_contacts"], so["n_contacts"])
        d = np.abs(h.get_state()[0] - o32.read(B.BUF_X0)).max(axis=1)[:sc.n_dyn] / ext
        n_out = int((d > 1e-4).sum())
        assert n_out <= max(2, sc.n_dyn // 1000) and d.max() <= 5e-3, (k, n_out, d.max())
        seen = min(seen, sg["n_contacts"])
    assert seen > 0


@pytest.mark.parametrize("lanes", [8, 32])
@pytest.mark.parametrize("case", ["cloth_fold", "cube_squeezed", "cloth_flat_on_box", "layers_stack"])
def test_dcd_pairs_bitexact_cpu_semantics(case, lanes):
    """contact_semantics 1 (the CPU backend's ProximalQuery predicates): the device pair set equals
    the oracle's, whose closest points are pinned to the reference's distPT.h / distEE.h."""
    from oracle import oracle as O
    sc, x = _dcd_case(case)
    sc.params.contact_semantics = 1
    sc.params.query_lanes = lanes
    h = B.Handle(sc)
    n = h.detect(x)
    ref_pairs, _ = O.dcd(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, sc.params.thickness,
                         semantics=1, static_begin=sc.n_dyn)
    assert n == len(ref_pairs) and n > 0
    got = h.contacts()
    assert sorted(map(tuple, got["pairs"].tolist())) == sorted(map(tuple, ref_pairs.tolist()))


def test_cpu_semantics_contact_step_parity():
    """The CPU backend's contact predicates through conversion and the contact projection: the
    same pairs as the oracle, converted fields and contact velocities within the tolerances of
    the GPU predicates' test."""
    sc, x = _crumpled_cloth()
    sc.params.contact_semantics = 1
    h, o = _setup(sc)
    x64 = x.astype(np.float64)
    rng = np.random.default_rng(12)
    uc = rng.normal(scale=1e-4, size=(sc.n_dyn, 3))
    for tgt in (h, o):
        tgt.write(B.BUF_X, x64)
        tgt.write(B.BUF_UC, uc)
    n = h.detect()
    assert n == o.detect() and n > 0
    gc, oc = h.contacts(), o.contacts()
    gi = {tuple(p): i for i, p in enumerate(gc["pairs"].tolist())}
    perm = np.array([gi[tuple(p)] for p in oc["pairs"].tolist()])
    assert np.abs(gc["bary"][perm] - oc["bary"]).max() <= 1e-5
    assert np.abs(gc["normal"][perm] - oc["normal"]).max() <= 1e-4
    assert np.abs(gc["gap"][perm] - oc["gap"]).max() <= 1e-6
    h.contact_step()
    o.contact_step()
    pg, po = h.read(B.BUF_P), o.read(B.BUF_P)
    assert _rel(pg[:sc.n_dyn], po[:sc.n_dyn]) <= 1e-4


@pytest.mark.parametrize("case", ["cube_impact", "sheets_small"])
def test_programmatic_launch_does_not_change_bits(case):
    """The same contact substeps with programmatic dependent launch (the default) and with it
    off (ADMM_B200_PDL=0, every kernel starts after its predecessor completes), in child
    processes: identical bits.  The contact kernels load detection data before their
    dependency wait, which is legal only because the kernel launched before each of them
    waits before it triggers."""
    import json
    import os
    import subprocess
    import sys
    code = f"""
import sys, json, numpy as np
sys.path.insert(0, {os.path.dirname(os.path.dirname(os.path.abspath(__file__)))!r})
from parallel_admm_b200 import backend as B, scene
case = {case!r}
if case == "cube_impact":
    sc = scene.cube_on_ground(10, drop=0.0)
    v0 = np.zeros_like(sc.verts); v0[:sc.n_dyn, 1] = -4.0
    x0 = sc.verts.copy(); x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.03
else:
    sc = scene.sheets_on_sphere(256, layers=2, seed=0)
    x0, v0 = sc.verts.copy(), np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -3.0
sc.params.ell_lanes = 4
sc.params.jacobi_mode = 1
h = B.Handle(sc)
h.set_state(x0, v0)
cs = [h.step(1, allow=(B.ERR_CONTACT_OVERFLOW,))["n_contacts"] for _ in range(10)]
x, v = h.get_state()
np.save(sys.argv[1], np.concatenate([x, v]))
print(json.dumps(cs))
"""
    outs = []
    for pdl in ("1", "0"):
        path = f"/tmp/pdl_{case}_{pdl}.npy"
        env = dict(os.environ, ADMM_B200_PDL=pdl)
        r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append((json.loads(r.stdout.strip().splitlines()[-1]), np.load(path)))
    assert outs[0][0] == outs[1][0] and max(outs[0][0]) > 0, (outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_vertex_renumbering_is_invisible_to_the_caller():
    """With ADMM_B200_RENUMBER=1 the library stores the dynamic vertices in Morton order; by
    default it keeps the caller's order.  Through the C ABI both give the same contact pair set and the
    same substeps up to FP32 summation order (every vertex but at most 1% within 1e-4, none
    beyond 5e-3: a contact on the edge of its switch can decide differently, as the oracle
    itself does in another numbering, test_oracle_order.py), and the order is a permutation
    that moves only dynamic vertices."""
    import os
    sc = scene.cube_on_ground(10, drop=0.0)
    sc.params.ell_lanes = 4
    sc.params.dcd_interval = sc.params.admm_max_iter  # one detection per substep: identical pair sets
    v0 = np.zeros_like(sc.verts)
    v0[:sc.n_dyn, 1] = -4.0
    x0 = sc.verts.copy()
    x0[:sc.n_dyn, 1] -= x0[:sc.n_dyn, 1].min() - 0.03
    hi = B.Handle(sc)
    old = os.environ.get("ADMM_B200_RENUMBER")
    os.environ["ADMM_B200_RENUMBER"] = "1"
    try:
        hr = B.Handle(sc)
    finally:
        if old is None:
            del os.environ["ADMM_B200_RENUMBER"]
        else:
            os.environ["ADMM_B200_RENUMBER"] = old
    order = hr.vertex_order()
    assert sorted(order.tolist()) == list(range(sc.n_vert))
    assert np.array_equal(order[sc.n_dyn:], np.arange(sc.n_dyn, sc.n_vert))
    assert not np.array_equal(order[:sc.n_dyn], np.arange(sc.n_dyn))
    assert np.array_equal(hi.vertex_order(), np.arange(sc.n_vert))
    for h in (hr, hi):
        h.set_state(x0, v0)
    xd = x0.copy()
    xd[:sc.n_dyn, 1] -= 0.025
    pr = sorted(map(tuple, (hr.detect(xd), hr.contacts()["pairs"])[1].tolist()))
    pi = sorted(map(tuple, (hi.detect(xd), hi.contacts()["pairs"])[1].tolist()))
    assert pr == pi and len(pr) > 0
    for h in (hr, hi):
        h.set_state(x0, v0)
    ext = np.ptp(x0[:sc.n_dyn], axis=0).max()
    for k in range(3):
        sr = hr.step(1)
        si = hi.step(1)
        assert sr["n_contacts"] == si["n_contacts"]
        d = np.abs(hr.get_state()[0] - hi.get_state()[0]).max(axis=1)[:sc.n_dyn] / ext
        n_out = int((d > 1e-4).sum())
        assert n_out <= max(8, sc.n_dyn // 100) and d.max() <= 5e-3, (k, n_out, d.max())
        hi.set_state(*hr.get_state())
        hi.write(B.BUF_UE, hr.read(B.BUF_UE))
        hi.write(B.BUF_UC, hr.read(B.BUF_UC))
