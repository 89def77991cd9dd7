"""Scene files: the reference's TOML format, its mesh readers and the mesh pipeline (CPU).

The scene files and meshes used here are written by the tests themselves; the reference's own
scene folder, when present, is only parsed (its meshes are not needed for that)."""
import glob
import math
import os
import struct

import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene as S
from parallel_admm_b200 import scene_config as C

REF_SCENES = "/root/reference/resource/scene"

SCENE = """
scene_name = "unit"
out_file = './out'
separate_out = true
show_windows = false
end_frame = 50
GPU = "b200"

[global]
dt = 0.02
sub_step = 2
pin = [0, 5, {static_pin}]
g = 9.8

[solver]
admm_max_iter = 12
DCD_interval = 3
GS_max_iter = 4
Global_Jacobi_iter = 16
admm.warmstart_Ue = true
admm.warmstart_Uc = false
contact.use_CCD = false
contact.enable = true
contact.w_scale = 50
contact.kappa = 1e6
contact.beta = 5e5
contact.mu = 0.35
contact.unique = true
damp.kl = 1e-4
damp.km = 0

[DCD]
narrow.max_collision = 20000
narrow.thickness = 4e-3
broad.radius = 4e-3
broad.strategy = 'rebuild'

[[mesh]]
f.path = 'meshes/cloth.obj'
f.type = 'tri'
f.color = 3
t.scale = 1.5
t.translate = [0.1, 0.6, -0.2]
t.rotate = [30, 45, 10]
k.stretch = 800.0
k.min_limit = 0.95
k.max_limit = 1.05
k.bending = 0.01
k.use_limit = false
density = 0.2

[[mesh]]
f.path = 'meshes/box.obj'
f.type = 'static'
f.color = 1
t.scale = 1
t.translate = [0, 0, 0]
t.rotate = [0, 0, 0]
k.stretch = 1.0
k.min_limit = 1.0
k.max_limit = 1.0
k.bending = 1.0
k.use_limit = false
density = 1.0
animate = ""

[[mesh]]
f.path = 'meshes/cube.msh'
f.type = 'tet'
f.color = 2
t.scale = 0.5
t.translate = [0, 1.2, 0]
t.rotate = [0, 90, 0]
k.stretch = 5e4
k.min_limit = 0.9
k.max_limit = 1.1
k.use_limit = true
density = 1000

[mesh_post]
center_ids = [1]

[[collider]]
type = 'plane'
center = [0, -1, 0]
halfside = 5.0
normal = [0, 1, 0]

[viewer]
scale = 1
color.background = [0.1, 0.1, 0.1]
enable_ground = false
"""


def write_obj(path, V, F, style="plain"):
    with open(path, "w") as f:
        f.write("# test mesh\n")
        for v in V:
            f.write("v " + " ".join(repr(float(c)) for c in v[:3]) + "\n")
        f.write("vt 0 0\n")
        for t in F:
            if style == "slashes":
                f.write("f " + " ".join(f"{i + 1}/1/{i + 1}" for i in t) + "\n")
            elif style == "negative":
                f.write("f " + " ".join(str(i - len(V)) for i in t) + "\n")
            else:
                f.write("f " + " ".join(str(i + 1) for i in t) + "\n")


def write_msh41(path, V, T):
    """Gmsh 4.1 ASCII: two node blocks, a triangle block and a tet block."""
    n, h = len(V), len(V) // 2
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        f.write(f"$Nodes\n2 {n} 1 {n}\n")
        for blk, (a, b) in enumerate(((0, h), (h, n))):
            f.write(f"3 {blk + 1} 0 {b - a}\n")
            for i in range(a, b):
                f.write(f"{i + 1}\n")
            for i in range(a, b):
                f.write(" ".join(repr(float(c)) for c in V[i]) + "\n")
        f.write("$EndNodes\n")
        f.write(f"$Elements\n2 {1 + len(T)} 1 {1 + len(T)}\n")
        f.write("2 1 2 1\n1 1 2 3\n")
        f.write(f"3 1 4 {len(T)}\n")
        for k, t in enumerate(T):
            f.write(f"{k + 2} {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n")
        f.write("$EndElements\n")


def write_msh22(path, V, T, binary):
    with open(path, "wb") as f:
        f.write(b"$MeshFormat\n")
        f.write(b"2.2 1 8\n" if binary else b"2.2 0 8\n")
        if binary:
            f.write(struct.pack("<i", 1) + b"\n")
        f.write(b"$EndMeshFormat\n$Nodes\n")
        f.write(f"{len(V)}\n".encode())
        for i, v in enumerate(V):
            if binary:
                f.write(struct.pack("<i3d", i + 1, *v))
            else:
                f.write((f"{i + 1} " + " ".join(repr(float(c)) for c in v) + "\n").encode())
        f.write(b"\n$EndNodes\n" if binary else b"$EndNodes\n")
        f.write(f"$Elements\n{1 + len(T)}\n".encode())
        if binary:
            f.write(struct.pack("<3i", 2, 1, 2) + struct.pack("<6i", 1, 0, 0, 1, 2, 3))
            f.write(struct.pack("<3i", 4, len(T), 2))
            for k, t in enumerate(T):
                f.write(struct.pack("<7i", k + 2, 0, 0, *(int(i) + 1 for i in t)))
            f.write(b"\n")
        else:
            f.write(b"1 2 2 0 0 1 2 3\n")
            for k, t in enumerate(T):
                f.write(f"{k + 2} 4 2 0 0 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n".encode())
        f.write(b"$EndElements\n")


def _write_scene(root, static_pin, animate=""):
    os.makedirs(os.path.join(root, "meshes"), exist_ok=True)
    os.makedirs(os.path.join(root, "scene"), exist_ok=True)
    cv, cf = S.grid_cloth(6, 0.4)
    write_obj(os.path.join(root, "meshes", "cloth.obj"), cv, cf, "slashes")
    bv, bf = S.box_mesh((-0.5, -0.2, -0.5), (0.5, 0.0, 0.5))
    write_obj(os.path.join(root, "meshes", "box.obj"), bv, bf, "negative")
    tv, tt = S.tet_cube(2, 1.0)
    write_msh41(os.path.join(root, "meshes", "cube.msh"), tv, tt)
    path = os.path.join(root, "scene", "unit.toml")
    with open(path, "w") as f:
        f.write(SCENE.format(static_pin=static_pin).replace('animate = ""', f'animate = "{animate}"'))
    return path, (cv, cf), (bv, bf), (tv, tt)


class AnimatorRef:
    """Restatement of the reference's animator (animator.cpp:81-204) for the tests: the shared
    frame counter (one step per animate_all, one more per rigid track), the clamp at the last
    frame, rigid motion pos[f] + q[f] * rest and point tracks t + R (s * points[f]), velocities
    (new - old) / dt, zero at init and past the end."""

    def __init__(self, tracks, rest, dt):
        self.tracks, self.rest, self.dt = tracks, np.asarray(rest, np.float64), dt
        self.c = -1

    def frames(self, init):
        c = (-1 if init else self.c) + 1
        out = []
        for tr in self.tracks:
            n = len(tr["pos"]) if tr["kind"] == "rigid" else len(tr["points"])
            if tr["kind"] == "rigid":
                c += 1
            if c >= n:
                c = n
                out.append((n - 1, False))
            else:
                out.append((c - 1 if tr["kind"] == "rigid" else c, not init))
        self.c = c
        return out

    @staticmethod
    def rotate(q, v):
        q = np.asarray(q, np.float64)
        u = 2.0 * np.cross(q[:3], v)
        return v + q[3] * u + np.cross(q[:3], u)

    def apply(self, x0, v, init=False):
        for tr, (f, moving) in zip(self.tracks, self.frames(init)):
            a, b = tr["v_begin"], tr["v_end"]
            if tr["kind"] == "rigid":
                new = tr["pos"][f].astype(np.float64) + self.rotate(tr["quat"][f], self.rest[a:b])
            else:
                new = tr["translate"] + (tr["scale"] * tr["points"][f].astype(np.float64)) @ tr["rot"].T
            v[a:b] = (new - x0[a:b]) / self.dt if moving else 0.0
            x0[a:b] = new


def spin_track(n_frames=40, dt=0.01):
    """A rigid track: rotation about y at 2 rad/s and a slow rise."""
    t = np.arange(n_frames) * dt
    ang = 2.0 * t
    quat = np.stack([np.zeros_like(t), np.sin(ang / 2), np.zeros_like(t), np.cos(ang / 2)], 1)
    pos = np.stack([np.zeros_like(t), 0.05 * t, np.zeros_like(t)], 1)
    return pos, quat


def wave_sequence(V, n_frames=30):
    """A point track: the mesh's own vertices with a travelling wave in y."""
    V = np.asarray(V, np.float64)
    return np.stack([V + np.stack([np.zeros(len(V)), 0.01 * np.sin(V[:, 0] * 6 + 0.3 * k),
                                   np.zeros(len(V))], 1) for k in range(n_frames)])


def test_parse_all_keys(tmp_path):
    path, *_ = _write_scene(str(tmp_path), 40)
    c = C.parse_config(path)
    assert c.scene_name == "unit" and c.end_frame == 50 and not c.show_windows
    assert c.selects_b200 and c.use_gpu
    assert c.dt == 0.02 and c.sub_step == 2 and math.isclose(c.substep_dt, 0.01)
    assert c.pin_ids == [0, 5, 40] and c.g == 9.8
    assert (c.admm_max_iter, c.dcd_interval, c.gs_max_iter, c.global_jacobi_iter) == (12, 3, 4, 16)
    assert c.warmstart_ue and not c.warmstart_uc and c.contact_enable and c.unique and not c.use_ccd
    assert (c.w_scale, c.kappa, c.beta, c.mu) == (50.0, 1e6, 5e5, 0.35)
    assert (c.damp_kl, c.damp_km) == (1e-4, 0.0)
    assert (c.max_collision, c.thickness, c.broad_radius, c.broad_strategy) == (20000, 4e-3, 4e-3, "rebuild")
    assert [m.type for m in c.meshes] == ["tri", "static", "tet"]
    tri, sta, tet = c.meshes
    assert tri.rotate == (30.0, 45.0, 10.0) and tri.scale == 1.5 and tri.bending == 0.01 and tri.density == 0.2
    assert tet.use_limit and tet.stretch == 5e4 and tet.density == 1000
    assert sta.animate == ""
    assert c.center_ids == [1]
    assert c.colliders[0].type == "plane" and c.colliders[0].normal == (0.0, 1.0, 0.0)
    assert c.background == (0.1, 0.1, 0.1)


def test_backend_selection_keys():
    base = SCENE.format(static_pin=1)
    assert not C.parse_config(base.replace('GPU = "b200"', "GPU = true")).selects_b200
    assert C.parse_config(base.replace('GPU = "b200"', "GPU = true")).use_gpu
    c = C.parse_config(base.replace('GPU = "b200"', "").replace("[solver]\n", '[solver]\nbackend = "b200"\n'))
    assert c.selects_b200 and not c.use_gpu


@pytest.mark.parametrize("key", ["scene_name = \"unit\"", "dt = 0.02", "narrow.thickness = 4e-3",
                                 "admm.warmstart_Ue = true", "k.bending = 0.01", "color.background"])
def test_missing_required_key_raises(key):
    text = SCENE.format(static_pin=1)
    lines = [l for l in text.split("\n") if not l.strip().startswith(key)]
    with pytest.raises(C.ConfigError):
        C.parse_config("\n".join(lines))


def test_wrong_type_raises():
    text = SCENE.format(static_pin=1).replace("admm_max_iter = 12", "admm_max_iter = 'twelve'")
    with pytest.raises(C.ConfigError):
        C.parse_config(text)


@pytest.mark.parametrize("style", ["plain", "slashes", "negative"])
def test_read_obj(tmp_path, style):
    V, F = S.grid_cloth(4, 1.0)
    p = str(tmp_path / "m.obj")
    write_obj(p, V, F, style)
    V2, F2 = C.read_obj(p)
    assert np.array_equal(F2, F) and np.allclose(V2, V, rtol=0, atol=1e-8)


def test_read_obj_rejects_quads(tmp_path):
    p = str(tmp_path / "q.obj")
    with open(p, "w") as f:
        f.write("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(ValueError):
        C.read_obj(p)


@pytest.mark.parametrize("fmt", ["4.1", "2.2", "2.2b"])
def test_read_msh(tmp_path, fmt):
    V, T = S.tet_cube(3, 1.0)
    V = V + np.array([0.123456789, -1.0, 2.0])
    p = str(tmp_path / "m.msh")
    if fmt == "4.1":
        write_msh41(p, V, T)
    else:
        write_msh22(p, V, T, binary=fmt == "2.2b")
    V2, T2 = C.read_msh(p)
    assert np.array_equal(T2, T)
    assert np.array_equal(V2, V.astype(np.float64))


def test_rotation_order_and_pi():
    R = C.rotation((90, 0, 0))
    a = C.PI_REF / 2
    assert np.allclose(R, [[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    Rx, Ry, Rz = C.rotation((20, 0, 0)), C.rotation((0, 30, 0)), C.rotation((0, 0, 40))
    assert np.allclose(C.rotation((20, 30, 40)), Rz @ Ry @ Rx)


def test_load_scene_matches_direct_assembly(tmp_path):
    path, (cv, cf), (bv, bf), (tv, tt) = _write_scene(str(tmp_path), 65)
    sc = C.load_scene(path)
    c = C.parse_config(path)
    tri, sta, tet = c.meshes
    # load order: tri and tet meshes in file order, then static meshes (mesh ids 0, 1, 2)
    V_cloth = (cv * 1.5) @ C.rotation(tri.rotate).T + np.array(tri.translate)
    V_cube = ((tv - tv.mean(0)) @ C.rotation(tet.rotate).T) * 0.5 + np.array(tet.translate)  # mesh id 1: centred
    p = S.SolverParams(dt=0.01, g=9.8, mu=0.35, kappa=1e6, beta=5e5, thickness=4e-3, admm_max_iter=12,
                       dcd_interval=3, gs_max_iter=4, jacobi_iter=16, max_contacts=20000,
                       enable_contact=True, warmstart_ue=True, warmstart_uc=False, w_scale=50.0)
    bodies = [S._Body(V_cloth, cf, np.zeros((0, 4), np.int32), 0.2, 800.0, 0.01),
              S._Body(V_cube, np.zeros((0, 3), np.int32), tt, 1000.0, 5e4),
              S._Body(bv, bf, np.zeros((0, 4), np.int32), 1e12, 1.0, static=True)]
    ref = S.assemble("unit", bodies, [0, 5, 65], p)
    assert sc.n_dyn == len(cv) + len(tv) and sc.n_vert == sc.n_dyn + len(bv)
    assert np.array_equal(sc.verts, ref.verts)
    for k in ("mass", "tri_inds", "tri_binv", "tri_w", "tet_inds", "tet_binv", "tet_w", "bend_offsets",
              "bend_inds", "bend_coeffs", "bend_w", "pin_inds", "surf_tris", "surf_edges", "surf_verts",
              "contact_w"):
        assert np.array_equal(getattr(sc, k), getattr(ref, k)), k
    assert list(sc.pin_inds) == [0, 5]        # vertex 65 is static: no pin
    assert sc.params.dt == 0.01 and sc.params.jacobi_iter == 16 and sc.params.max_contacts == 20000


def test_heuristic_contact_weights_use_the_system_diagonal():
    """use_heu_wc: the diagonal a_ii behind the weights equals the oracle's global matrix diagonal
    (without damping, sigma = 1, beta = 0 -> w_c,i = a_ii * 10 / h^2)."""
    from oracle import oracle as O
    sc = S.cloth_on_box(8)
    h = sc.params.dt
    o = O.Oracle(B.DescHolder(sc), double=True)
    A = o.system()
    n = sc.n_dyn
    surf = np.zeros(sc.n_vert, bool)
    surf[sc.surf_verts] = True
    a_ref = A.diagonal() - h * h * sc.contact_w[:n].astype(np.float64) * surf[:n]
    w = C.heuristic_contact_weights(sc, h, 0.0, 0.0, 1.0, 0.0)
    a = w[:n].astype(np.float64) * h * h / 10.0
    s = surf[:n]
    assert np.abs(a[s] - a_ref[s]).max() <= 1e-6 * np.abs(a_ref).max()
    # the min/max rule: max(sigma a, min(beta m, a))
    m = sc.mass[:n].astype(np.float64)
    w2 = C.heuristic_contact_weights(sc, h, 0.0, 0.0, 0.001, 25.0).astype(np.float64)
    want = np.maximum(0.001 * a_ref, np.minimum(25.0 * m, a_ref)) * 10.0 / (h * h)
    assert np.allclose(w2[:n][s], want[s], rtol=1e-6, atol=0)
    # mass damping adds h k_M m_i to a_ii
    w3 = C.heuristic_contact_weights(sc, h, 0.0, 0.5, 1.0, 0.0).astype(np.float64)
    assert np.allclose(w3[:n][s] * h * h / 10.0, (a_ref + h * 0.5 * m)[s], rtol=1e-6, atol=0)
    # vertices off the surface keep their weights
    assert np.array_equal(w3[:n][~s], sc.contact_w[:n][~s])


@pytest.mark.skipif(not os.path.isdir(REF_SCENES), reason="reference scene folder absent")
def test_reference_scene_files_parse():
    """Every scene file of the reference parses, except the ones that the reference's own loader
    rejects too (each lacks a key that APPConfig::load_config requires)."""
    ok, rejected = [], []
    for p in sorted(glob.glob(os.path.join(REF_SCENES, "*.toml"))):
        try:
            C.parse_config(p)
            ok.append(os.path.basename(p))
        except C.ConfigError as e:
            rejected.append((os.path.basename(p), str(e)))
    assert len(ok) >= 25, rejected
    for name, why in rejected:
        assert "missing" in why, (name, why)


def test_track_files_and_scene_tracks(tmp_path):
    root = str(tmp_path)
    os.makedirs(os.path.join(root, "track"))
    pos, quat = spin_track()
    np.savez(os.path.join(root, "track", "spin.npz"), pos=pos, quat=quat)
    path, _, (bv, bf), _ = _write_scene(root, 65, animate="track/spin.npz")
    cfg = C.parse_config(path)
    sc = C.load_scene(path)
    tr = C.scene_tracks(cfg, sc)
    assert len(tr) == 1 and tr[0]["kind"] == "rigid" and tr[0]["mesh_id"] == 2
    assert (tr[0]["v_begin"], tr[0]["v_end"]) == (sc.n_dyn, sc.n_vert)
    assert tr[0]["pos"].dtype == np.float32 and np.allclose(tr[0]["quat"], quat)
    # a path with "sequence" holds per-vertex points
    seq = wave_sequence(bv)
    np.savez(os.path.join(root, "track", "box_sequence.npz"), points=seq)
    p2, *_ = _write_scene(root, 65, animate="track/box_sequence.npz")
    tr2 = C.scene_tracks(C.parse_config(p2), C.load_scene(p2))
    assert tr2[0]["kind"] == "points" and tr2[0]["points"].shape == seq.shape
    # too short, wrong shapes
    np.savez(os.path.join(root, "track", "short.npz"), pos=pos[:2], quat=quat[:2])
    with pytest.raises(ValueError):
        C.read_track(os.path.join(root, "track", "short.npz"))
    np.savez(os.path.join(root, "track", "bad_sequence.npz"), points=seq[:, :3])
    p3, *_ = _write_scene(root, 65, animate="track/bad_sequence.npz")
    with pytest.raises(ValueError):
        C.scene_tracks(C.parse_config(p3), C.load_scene(p3))


def test_animator_frame_counter():
    """The reference's counter: a rigid track reads frames 0 (init), 2, 4, ... and holds its
    last frame with zero velocity; a point track reads 0, 1, 2, ...; two rigid tracks advance
    the shared counter three times per substep."""
    rig = {"kind": "rigid", "pos": np.zeros((7, 3)), "quat": np.zeros((7, 4))}
    pts = {"kind": "points", "points": np.zeros((5, 1, 3))}
    a = AnimatorRef([rig], np.zeros((1, 3)), 0.01)
    seq = [a.frames(True)] + [a.frames(False) for _ in range(5)]
    assert [f[0] for f in seq] == [(0, False), (2, True), (4, True), (6, False), (6, False), (6, False)]
    b = AnimatorRef([pts], np.zeros((1, 3)), 0.01)
    seq = [b.frames(True)] + [b.frames(False) for _ in range(6)]
    assert [f[0] for f in seq] == [(0, False), (1, True), (2, True), (3, True), (4, True), (4, False), (4, False)]
    c = AnimatorRef([rig, dict(rig)], np.zeros((1, 3)), 0.01)
    assert c.frames(True) == [(0, False), (1, False)]
    assert c.frames(False) == [(3, True), (4, True)]
