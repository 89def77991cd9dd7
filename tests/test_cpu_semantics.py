"""The CPU backend's contact predicates (ProximalQuery, narrow_phase.cpp:192-469) in the oracle:
Eberly's point-triangle and segment-segment closest points (distPT.h / distEE.h) pinned to the
reference's own headers compiled on the host, known answers, and the detection rules checked
against a brute-force loop over all pairs (CPU)."""
import itertools

import numpy as np
import pytest

from oracle import oracle as O
from parallel_admm_b200 import scene


def _cases(n, seed):
    rng = np.random.default_rng(seed)
    for k in range(n):
        sc = 10.0 ** rng.uniform(-3, 1)
        pts = (rng.normal(size=(4, 3)) * sc).astype(np.float32)
        if k % 7 == 0:
            pts[3] = pts[2] + (pts[2] - pts[1]) * np.float32(rng.uniform(-2, 2))  # near-parallel / collinear
        if k % 11 == 0:
            pts[1] = pts[0]                                                      # degenerate edge
        if k % 13 == 0:
            pts[3] = pts[1] + np.float32(1e-7)
        yield pts


@pytest.mark.skipif(O.ref_pin() is None, reason="reference headers not compiled (reference tree absent)")
def test_closest_points_bitexact_vs_reference_headers():
    for pts in _cases(20000, 5):
        a, b = O.gt_pt(*pts), O.gt_pt(*pts, ref=True)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), pts
        c, d = O.gt_ee(*pts), O.gt_ee(*pts, ref=True)
        assert np.array_equal(c.view(np.uint32), d.view(np.uint32)), pts


def test_point_triangle_known_answers():
    T = [np.array(v, np.float32) for v in ((0, 0, 0), (1, 0, 0), (0, 1, 0))]
    # interior: straight above (0.25, 0.25)
    r = O.gt_pt(np.array([0.25, 0.25, 2.0], np.float32), *T)
    assert r[0] == 2.0 and np.allclose(r[2:5], [0.5, 0.25, 0.25]) and np.allclose(r[8:11], [0.25, 0.25, 0])
    # beyond vertex t0, t1, t2 and edges: the distance to the nearest feature
    for p, want in (((-1, -1, 0), np.sqrt(2)), ((3, 0, 0), 2.0), ((0, 3, 0), 2.0), ((0.5, -2, 0), 2.0),
                    ((-2, 0.5, 0), 2.0), ((1, 1, 0), np.sqrt(0.5))):
        r = O.gt_pt(np.array(p, np.float32), *T)
        assert abs(r[0] - want) < 1e-6, (p, r[0])
        assert abs(r[2:5].sum() - 1.0) < 1e-6 and (r[2:5] >= 0).all()


def test_segment_segment_known_answers():
    f = lambda *v: np.array(v, np.float32)
    # crossing at right angles one unit apart: interior parameters
    r = O.gt_ee(f(-1, 0, 0), f(1, 0, 0), f(0, -1, 1), f(0, 1, 1))
    assert r[0] == 1.0 and r[2] == 0.5 and r[3] == 0.5
    # parallel, overlapping: a point of the overlap on segment 0 with t from the projection
    r = O.gt_ee(f(0, 0, 0), f(2, 0, 0), f(1, 1, 0), f(3, 1, 0))
    assert abs(r[0] - 1.0) < 1e-6
    # end point against end point
    r = O.gt_ee(f(0, 0, 0), f(1, 0, 0), f(2, 0, 0), f(3, 0, 0))
    assert r[0] == 1.0 and r[2] == 1.0 and r[3] == 0.0


def _brute_force(x, sc, thickness, static_begin):
    """All pairs by the CPU backend's rules, looping over every pair."""
    out = set()
    for v in sc.surf_verts:
        for t in sc.surf_tris:
            if v in t or (v >= static_begin and t[0] >= static_begin):
                continue
            r = O.gt_pt(x[v], x[t[0]], x[t[1]], x[t[2]])
            if r[0] <= thickness:
                out.add((int(v), int(t[0]), int(t[1]), int(t[2])))
    E = sc.surf_edges
    for i, j in itertools.combinations(range(len(E)), 2):
        a, b = E[i], E[j]
        if len({a[0], a[1], b[0], b[1]}) < 4 or (a[0] >= static_begin and b[0] >= static_begin):
            continue
        r = O.gt_ee(x[a[0]], x[a[1]], x[b[0]], x[b[1]])
        corner = r[2] in (0.0, 1.0) and r[3] in (0.0, 1.0)
        if r[0] < thickness and not corner:
            out.add((int(a[0]), int(a[1]), int(b[0]), int(b[1])))
    return out


def test_cpu_semantics_detection_matches_brute_force():
    sc = scene.cloth_on_box(6)
    x = sc.verts.astype(np.float32).copy()
    n = sc.n_dyn
    # fold the cloth onto itself and onto the box top so that every kind of pair occurs
    u = x[:n, 0] - x[:n, 0].min()
    fold = u > 0.5 * u.max()
    x[:n, 0] = np.where(fold, x[:n, 0].min() + u.max() - u, x[:n, 0])
    x[:n, 1] = np.where(fold, 0.5 + 0.6 * sc.params.thickness, 0.5 + 0.2 * sc.params.thickness)
    rng = np.random.default_rng(2)
    x[:n] += rng.normal(scale=0.3 * sc.params.thickness, size=(n, 3)).astype(np.float32)
    th = sc.params.thickness
    pairs, _ = O.dcd(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, th, semantics=1, static_begin=n)
    got = set(map(tuple, pairs.tolist()))
    assert len(got) == len(pairs)
    assert got == _brute_force(x, sc, th, n)
    # the GPU predicates (interior closest points only) find pairs here too
    gpu, _ = O.dcd(x, sc.surf_verts, sc.surf_tris, sc.surf_edges, th)
    assert len(got) > 0 and len(gpu) > 0
