"""Known-answer and consistency tests of the oracle itself (CPU only)."""
import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene


def _rot(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def test_prox_tet_closed_form(oracle_lib):
    """F = R diag(s) -> z = 1/2 (R + F); an inverted F gets the closest proper rotation."""
    O = oracle_lib
    rng = np.random.default_rng(0)
    for _ in range(100):
        R = _rot(rng)
        F = R @ np.diag(rng.uniform(0.3, 3.0, 3))
        z = O.prox_tet(F.T.reshape(9)).reshape(3, 3).T
        assert np.allclose(z, 0.5 * (R + F), atol=1e-10)
        Fi = F @ np.diag([1, 1, -1])  # inverted element, det < 0
        zi = O.prox_tet(Fi.T.reshape(9)).reshape(3, 3).T
        P = 2 * zi - Fi
        assert abs(np.linalg.det(P) - 1) < 1e-9
        assert np.allclose(P @ P.T, np.eye(3), atol=1e-9)


def test_prox_tri_closed_form(oracle_lib):
    """F = Q diag(s) (3x2, orthonormal Q) -> z = 1/2 (Q + F)."""
    O = oracle_lib
    rng = np.random.default_rng(1)
    for _ in range(100):
        Q = np.linalg.qr(rng.normal(size=(3, 2)))[0]
        W = np.linalg.qr(rng.normal(size=(2, 2)))[0]
        F = Q @ np.diag(rng.uniform(0.3, 3.0, 2)) @ W.T
        P = Q @ W.T
        z = O.prox_tri(np.concatenate([F[:, 0], F[:, 1]]))
        got = np.stack([z[:3], z[3:]], 1)
        assert np.allclose(got, 0.5 * (P + F), atol=1e-10)


def test_dcd_pt_ee_known_answers(oracle_lib):
    O = oracle_lib
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    r = O.dcd_pt(np.array([0.25, 0.25, 0.01], np.float32), *tri)
    assert r[0] == pytest.approx(0.01, rel=1e-6)
    assert r[2:5] == pytest.approx([0.5, 0.25, 0.25], abs=1e-6)   # bary = (1-s-t, s, t)
    assert O.dcd_pt(np.array([2.0, 2.0, 0.01], np.float32), *tri)[0] == -10  # outside region 0
    r = O.dcd_ee(np.array([0, 0, 0], np.float32), np.array([1, 0, 0], np.float32),
                 np.array([0.5, -0.5, 0.02], np.float32), np.array([0.5, 0.5, 0.02], np.float32))
    assert r[0] == pytest.approx(0.02, rel=1e-6) and r[4] == -10
    assert r[2:4] == pytest.approx([0.5, 0.5], abs=1e-6)
    # parallel edges are never accepted (dist_g.cuh parallel branch leaves valid = false)
    assert O.dcd_ee(np.array([0, 0, 0], np.float32), np.array([1, 0, 0], np.float32),
                    np.array([0, 0.001, 0], np.float32), np.array([1, 0.001, 0], np.float32))[0] == -10


def _brute_pairs(x, sv, st, se, thk, O):
    """All pairs by brute force (no grid) with the same filter and predicate."""
    out = set()
    def box(ids):
        p = x[list(ids)]
        return p.min(0), p.max(0)
    def ovl(a, b):
        for k in range(3):
            if np.float32(b[0][k] - a[1][k]) >= thk or np.float32(a[0][k] - b[1][k]) >= thk:
                return False
        return True
    tb = [box(t) for t in st]
    for v in sv:
        q = (x[v], x[v])
        for f, t in enumerate(st):
            if v in t or not ovl(q, tb[f]):
                continue
            r = O.dcd_pt(x[v], x[t[0]], x[t[1]], x[t[2]])
            if 0 <= r[0] < thk:
                out.add((int(v), int(t[0]), int(t[1]), int(t[2])))
    eb = [box(e) for e in se]
    for e in range(len(se)):
        for o in range(e + 1, len(se)):
            if set(se[e]) & set(se[o]) or not ovl(eb[e], eb[o]):
                continue
            r = O.dcd_ee(x[se[e][0]], x[se[e][1]], x[se[o][0]], x[se[o][1]])
            if 0 <= r[0] < thk:
                out.add((int(se[e][0]), int(se[e][1]), int(se[o][0]), int(se[o][1])))
    return out


def test_grid_dcd_equals_brute_force(oracle_lib):
    O = oracle_lib
    sc = scene.cloth_on_box(10, seed=2)
    rng = np.random.default_rng(3)
    x = sc.verts.copy()
    n = sc.n_dyn
    # drape the cloth onto the box top and crumple it
    x[:n, 1] = 0.5 + rng.uniform(0, 2 * sc.params.thickness, n).astype(np.float32)
    x[:n, 0] *= 0.3
    thk = np.float32(sc.params.thickness * 4)
    pairs, _ = O.dcd(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, float(thk))
    got = {tuple(int(v) for v in p) for p in pairs}
    ref = _brute_pairs(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, thk, O)
    assert len(ref) > 20
    assert got == ref


def test_fp32_and_fp64_oracle_agree_on_cloth(oracle_lib):
    O = oracle_lib
    sc = scene.cloth_on_box(12)
    h = B.DescHolder(sc)
    a = O.Oracle(h, double=True)
    b = O.Oracle(h, double=False)
    a.step(3)
    b.step(3)
    xa, xb = a.read(B.BUF_X0), b.read(B.BUF_X0)
    # FP32 rounding alone (stiff pins, k = 1e5): about 1e-5 per step on a 1 m cloth
    assert np.abs(xa - xb).max() < 3e-5


def test_free_fall_is_rigid_and_exact(oracle_lib):
    """Without contact a free-falling body keeps its shape; x follows x0 + h v - g h^2."""
    O = oracle_lib
    sc = scene.cube_on_ground(4)
    h = B.DescHolder(sc)
    o = O.Oracle(h, double=True)
    o.step(3)
    x = o.read(B.BUF_X0)[:sc.n_dyn]
    x0 = sc.verts[:sc.n_dyn].astype(np.float64)
    g, dt = sc.params.g, sc.params.dt
    expect = x0.copy()
    expect[:, 1] -= g * dt * dt * (1 + 2 + 3)
    assert np.abs(x - expect).max() < 1e-9


def test_friction_cone_projection_cases(oracle_lib):
    """Stick, slide and separate: a single contact against a static triangle."""
    O = oracle_lib
    # one dynamic vertex above a static triangle
    from parallel_admm_b200.scene import SolverParams, _Body, assemble
    tri_v = np.array([[-1, 0, -1], [1, 0, -1], [0, 0, 1]], float)
    p = np.array([[0.0, 0.001, 0.0], [0.0, 0.5, 0.0], [0.1, 0.5, 0.0]])
    # a tiny triangle body made of the point and two far vertices (triangle strain only)
    body = _Body(p, np.array([[0, 2, 1]], np.int32), np.zeros((0, 4), np.int32), 1.0, 1e2, 0.0)
    ground = _Body(tri_v, np.array([[0, 2, 1]], np.int32), np.zeros((0, 4), np.int32), 1e12, 0, static=True)
    params = SolverParams(dt=0.01, mu=0.5, thickness=0.005, admm_max_iter=1, gs_max_iter=50)
    sc = assemble("one_contact", [body, ground], [], params)
    h = B.DescHolder(sc)
    for vel, expect in [((0.0, -1.0, 0.0), "stop"), ((0.05, -1.0, 0.0), "stick"), ((5.0, -0.1, 0.0), "slide"),
                        ((0.0, 1.0, 0.0), "free")]:
        o = O.Oracle(h, double=True)
        x = sc.verts.astype(np.float64)
        o.write(B.BUF_X, x)
        o.write(B.BUF_X0, x)
        assert o.detect() >= 1
        xv = x.copy()
        xv[0] += 0.01 * np.array(vel)   # x - x0 = h v
        o.write(B.BUF_X, xv)
        o.contact_step()
        pv = o.read(B.BUF_P)[0]
        if expect == "free":
            assert np.allclose(pv, vel, atol=1e-9)
        else:
            assert pv[1] > vel[1]            # normal velocity pushed up
            if expect in ("stop", "stick"):
                assert abs(pv[0]) < abs(vel[0]) + 1e-12
            if expect == "slide":
                assert pv[0] > 0.0           # keeps sliding, slowed by friction
