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


def _write_scene(root, static_pin):
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
        f.write(SCENE.format(static_pin=static_pin))
    return path, (cv, cf), (bv, bf), (tv, tt)


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
