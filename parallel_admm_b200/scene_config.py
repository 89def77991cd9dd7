"""Scene files: the reference's TOML scene format, its mesh readers and its mesh pipeline.

A scene file of the reference (``resource/scene/*.toml``) runs through this backend:

    cfg = parse_config("scene.toml")            # APPConfig::load_config
    sc = load_scene("scene.toml", resources)    # meshes -> constraints -> Scene
    h = Handle(sc)                              # the backend, as ADMMSolver would create it

What follows the reference, and where:

* keys, defaults and required entries -- ``src/config/app_config.h:157-358``
  (``APPConfig::load_config``; a missing required key raises :class:`ConfigError`, the
  reference's "CTML_ APPConfig toml file invalid")
* backend selection -- ``src/solver/admm_solver_factory.cpp:14`` picks ADMM_GPU for
  ``GPU = true``; this backend is chosen by ``GPU = "b200"`` or ``[solver] backend = "b200"``
  (:attr:`AppConfig.backend`), so existing scene files keep their meaning
* mesh loading order and transforms -- ``src/config/mesh_from_config.h:18-85``: tri and tet
  meshes in file order, then static meshes; ``centralize`` (``mesh_post.center_ids``, ids in
  load order), then scale, rotate, translate for triangle and static meshes and rotate, scale,
  translate for tet meshes; rotation ``q_z * q_y * q_x`` from degrees with pi = 3.1415926
* mesh files -- OBJ triangles (``igl::readOBJ``, ``mesh_container.h:509``) and Gmsh MSH 2.2
  (ASCII or binary) / 4.1 (ASCII) linear tets (``src/mutils/mesh_io.h:14-77``: every element
  of type 4, node tag - 1 as the vertex index)
* masses, surface sets, constraints, contact weights -- :func:`scene.assemble`
  (``mesh_container.h:232-335,452-472``, ``mesh_to_constraint.h``,
  ``solver_config_applier.cpp:5-53``); static meshes get density 1e12
  (``mesh_from_config.h:71``); pins on static vertices are dropped
  (``mesh_to_constraint.h:36-52``)
* heuristic contact weights (``contact.use_heu_wc``) -- ``admm_impl_gpu.cu:204-218``:
  ``w_c,i = max(sigma a_ii, min(beta m_i, a_ii)) * 10 / h^2`` on surface vertices, a_ii the
  diagonal of ``M + h^2 D^T W^2 D + h (k_L D^T W D + k_M M)``
* time step -- ``global.dt / global.sub_step`` (``app_initializer.cpp:60-61``)

Parsed and kept in :class:`AppConfig` but not used by the substep (as in the reference's GPU
backend): strain limits (``k.use_limit``; the GPU prox ignores them), damping outside the
heuristic weights (``m_Damp_Mat`` is not part of A on the GPU path), ``use_CCD``, ``unique``,
``coloring``, ``use_Jacobi``, broad-phase radius and strategy, plane colliders (used by the
CPU solver's nodal obstacle constraints), viewer and output settings.  Scripted static meshes
(``animate``): :func:`scene_tracks` reads their ``.npz`` tracks (``animator.cpp:9-79``) and
:func:`attach_tracks` hands them to the backend, which moves them on the device.

Vertex transforms are computed in float64 and rounded to float32 once (the reference rounds
after every float32 operation), so positions can differ from the reference's by an ulp.
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct
import tomllib
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import scene as S

PI_REF = 3.1415926  # mesh_from_config.h:25


class ConfigError(ValueError):
    """A scene file that the reference's loader would reject (missing or ill-typed key)."""


# ----------------------------------------------------------------------------
# configuration (APPConfig)
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class MeshSpec:
    path: str
    type: str                       # 'tri' | 'tet' | 'static'
    color: int = 0
    scale: float = 1.0
    translate: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rotate: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # degrees about x, y, z
    density: float = 1.0
    stretch: float = 0.0
    min_limit: float = 0.0
    max_limit: float = 0.0
    bending: float = 0.0
    use_limit: bool = False
    animate: str = ""


@dataclasses.dataclass
class Collider:
    type: str
    center: Tuple[float, float, float]
    halfside: float
    normal: Tuple[float, float, float]


@dataclasses.dataclass
class AppConfig:
    """Mirror of the reference's APPConfig (app_config.h:14-155)."""
    scene_name: str = ""
    out_file: str = ""
    separate_out: bool = False
    show_windows: bool = True
    out_bin: bool = False
    export_obj: bool = False
    end_frame: int = 2000
    use_gpu: bool = False
    backend: str = ""               # "b200" selects this backend
    # [global]
    dt: float = 0.0
    pin_ids: List[int] = dataclasses.field(default_factory=list)
    g: float = 0.0
    sub_step: int = 1
    # [xpbd] (parsed only)
    use_xpbd: bool = False
    xpbd_iter: int = 100
    xpbd_substeps: int = 1
    xpbd_contact_stiffness: float = 10.0
    xpbd_use_gs_contact: bool = True
    # [solver]
    solver_type: str = "admm"
    admm_max_iter: int = 0
    dcd_interval: int = 0
    gs_max_iter: int = 0
    global_jacobi_iter: int = 20
    warmstart_ue: bool = False
    warmstart_uc: bool = False
    dump_a: bool = False
    contact_enable: bool = False
    use_ccd: bool = False
    use_jacobi: bool = False
    w_scale: float = 0.0
    kappa: float = 0.0
    beta: float = 0.0
    mu: float = 0.0
    unique: bool = False
    coloring: bool = False
    use_heu_wc: bool = False
    wc_beta: float = 25.0
    wc_sigma: float = 0.001
    damp_kl: float = 0.0
    damp_km: float = 0.0
    # [DCD]
    max_collision: int = 0
    thickness: float = 0.0
    broad_radius: float = 0.0
    broad_strategy: str = ""
    # meshes and the rest
    meshes: List[MeshSpec] = dataclasses.field(default_factory=list)
    center_ids: List[int] = dataclasses.field(default_factory=list)
    colliders: List[Collider] = dataclasses.field(default_factory=list)
    viewer_scale: float = 1.0
    background: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    enable_ground: bool = False

    @property
    def substep_dt(self) -> float:
        return self.dt / self.sub_step

    @property
    def selects_b200(self) -> bool:
        return self.backend == "b200"


_MISSING = object()


def _get(tbl, dotted: str, default=_MISSING):
    cur = tbl
    for part in dotted.split("."):
        if not isinstance(cur, dict) or part not in cur:
            if default is _MISSING:
                raise ConfigError(f"scene file invalid: missing '{dotted}'")
            return default
        cur = cur[part]
    return cur


def _real(tbl, key, default=_MISSING) -> float:
    v = _get(tbl, key, default)
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        if v is default and default is not _MISSING:
            return v
        raise ConfigError(f"scene file invalid: '{key}' is not a number")
    return float(v)


def _int(tbl, key, default=_MISSING) -> int:
    v = _get(tbl, key, default)
    if isinstance(v, bool) or not isinstance(v, (int, float)) or float(v) != int(v):
        if v is default and default is not _MISSING:
            return v
        raise ConfigError(f"scene file invalid: '{key}' is not an integer")
    return int(v)


def _bool(tbl, key, default=_MISSING) -> bool:
    v = _get(tbl, key, default)
    if not isinstance(v, bool):
        if v is default and default is not _MISSING:
            return v
        raise ConfigError(f"scene file invalid: '{key}' is not a boolean")
    return v


def _str(tbl, key, default=_MISSING) -> str:
    v = _get(tbl, key, default)
    if not isinstance(v, str):
        if v is default and default is not _MISSING:
            return v
        raise ConfigError(f"scene file invalid: '{key}' is not a string")
    return v


def _vec3(tbl, key) -> Tuple[float, float, float]:
    v = _get(tbl, key)
    if not isinstance(v, list) or len(v) < 3:
        raise ConfigError(f"scene file invalid: '{key}' is not a 3-vector")
    return tuple(_real({"x": v[i]}, "x") for i in range(3))


def parse_config(source: str) -> AppConfig:
    """Parse a scene file (path, or the TOML text itself when it contains a newline)."""
    if "\n" in source:
        doc = tomllib.loads(source)
    else:
        with open(source, "rb") as f:
            doc = tomllib.load(f)
    c = AppConfig()
    c.scene_name = _str(doc, "scene_name")
    c.out_file = _str(doc, "out_file")
    c.separate_out = _bool(doc, "separate_out")
    c.show_windows = _bool(doc, "show_windows")
    c.out_bin = _bool(doc, "out_bin", False)
    c.export_obj = _bool(doc, "export_obj", False)
    ef = _int(doc, "end_frame", 0)
    if ef > 0:
        c.end_frame = ef
    gpu = doc.get("GPU")
    if isinstance(gpu, bool):
        c.use_gpu = gpu
    elif isinstance(gpu, str):
        c.use_gpu = True
        c.backend = gpu.lower()
    elif gpu is not None:
        raise ConfigError("scene file invalid: 'GPU' is neither a boolean nor a backend name")

    c.dt = _real(doc, "global.dt")
    c.sub_step = _int(doc, "global.sub_step", 1)
    if c.sub_step < 1:
        raise ConfigError("scene file invalid: 'global.sub_step' < 1")
    pins = _get(doc, "global.pin")
    if not isinstance(pins, list):
        raise ConfigError("scene file invalid: 'global.pin' is not an array")
    c.pin_ids = [_int({"p": p}, "p") for p in pins]
    c.g = _real(doc, "global.g")

    if isinstance(doc.get("xpbd"), dict):
        c.use_xpbd = _bool(doc, "xpbd.enable")
        c.xpbd_iter = _int(doc, "xpbd.iter")
        c.xpbd_substeps = _int(doc, "xpbd.substeps", c.xpbd_substeps)
        c.xpbd_contact_stiffness = _real(doc, "xpbd.contact_stiffness", c.xpbd_contact_stiffness)
        c.xpbd_use_gs_contact = _bool(doc, "xpbd.use_GS_contact", c.xpbd_use_gs_contact)

    c.solver_type = _str(doc, "solver.type", "admm")
    be = _str(doc, "solver.backend", "")
    if be:
        c.backend = be.lower()
    c.admm_max_iter = _int(doc, "solver.admm_max_iter")
    c.dcd_interval = _int(doc, "solver.DCD_interval")
    c.gs_max_iter = _int(doc, "solver.GS_max_iter")
    c.global_jacobi_iter = _int(doc, "solver.Global_Jacobi_iter", c.global_jacobi_iter)
    c.warmstart_ue = _bool(doc, "solver.admm.warmstart_Ue")
    c.warmstart_uc = _bool(doc, "solver.admm.warmstart_Uc")
    c.dump_a = _bool(doc, "solver.admm.dump_A", False)
    c.contact_enable = _bool(doc, "solver.contact.enable")
    c.use_ccd = _bool(doc, "solver.contact.use_CCD")
    c.use_jacobi = _bool(doc, "solver.contact.use_Jacobi", False)
    c.w_scale = _real(doc, "solver.contact.w_scale")
    c.mu = _real(doc, "solver.contact.mu")
    c.kappa = _real(doc, "solver.contact.kappa")
    c.beta = _real(doc, "solver.contact.beta")
    c.unique = _bool(doc, "solver.contact.unique")
    c.coloring = _bool(doc, "solver.contact.coloring", False)
    c.use_heu_wc = _bool(doc, "solver.contact.use_heu_wc", False)
    if c.use_heu_wc:
        c.wc_beta = _real(doc, "solver.contact.wc_beta", c.wc_beta)
        c.wc_sigma = _real(doc, "solver.contact.wc_sigma", c.wc_sigma)
    c.damp_kl = _real(doc, "solver.damp.kl")
    c.damp_km = _real(doc, "solver.damp.km")

    c.max_collision = _int(doc, "DCD.narrow.max_collision")
    c.thickness = _real(doc, "DCD.narrow.thickness")
    c.broad_radius = _real(doc, "DCD.broad.radius")
    c.broad_strategy = _str(doc, "DCD.broad.strategy")

    meshes = _get(doc, "mesh")
    if not isinstance(meshes, list):
        raise ConfigError("scene file invalid: 'mesh' is not an array of tables")
    for m in meshes:
        spec = MeshSpec(path=_str(m, "f.path"), type=_str(m, "f.type"), color=_int(m, "f.color"))
        spec.scale = _real(m, "t.scale")
        spec.translate = _vec3(m, "t.translate")
        spec.rotate = _vec3(m, "t.rotate")
        if spec.type in ("tri", "tet"):
            spec.density = _real(m, "density")
            spec.stretch = _real(m, "k.stretch")
            spec.min_limit = _real(m, "k.min_limit")
            spec.max_limit = _real(m, "k.max_limit")
            if spec.type == "tri":
                spec.bending = _real(m, "k.bending")
            spec.use_limit = _bool(m, "k.use_limit")
        elif spec.type == "static":
            spec.animate = _str(m, "animate")
        c.meshes.append(spec)

    ids = _get(doc, "mesh_post.center_ids", None)
    if isinstance(ids, list):
        c.center_ids = [_int({"i": i}, "i") for i in ids]
    cols = doc.get("collider")
    if isinstance(cols, list):
        for col in cols:
            if not isinstance(col, dict):
                continue
            t = _str(col, "type")
            if t == "plane":
                c.colliders.append(Collider(t, _vec3(col, "center"), _real(col, "halfside"), _vec3(col, "normal")))

    c.viewer_scale = _real(doc, "viewer.scale")
    c.background = _vec3(doc, "viewer.color.background")
    c.enable_ground = _bool(doc, "viewer.enable_ground")
    return c


# ----------------------------------------------------------------------------
# mesh files
# ----------------------------------------------------------------------------

def read_obj(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """Vertices (n x 3 float64) and triangles (m x 3 int32) of an OBJ file.  Face entries may
    carry texture/normal indices (``a/b/c``) and negative (relative) indices; every face must
    be a triangle, as the reference reads faces into an n x 3 matrix."""
    verts: List[Tuple[float, float, float]] = []
    faces: List[Tuple[int, int, int]] = []
    with open(path, "r", encoding="utf-8", errors="replace") as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v":
                if len(parts) < 4:
                    raise ValueError(f"{path}: vertex with fewer than 3 coordinates")
                verts.append((float(parts[1]), float(parts[2]), float(parts[3])))
            elif parts[0] == "f":
                idx = []
                for p in parts[1:]:
                    k = int(p.split("/")[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)
                if len(idx) != 3:
                    raise ValueError(f"{path}: face with {len(idx)} vertices (triangles only)")
                faces.append(tuple(idx))
    V = np.asarray(verts, np.float64).reshape(-1, 3)
    F = np.asarray(faces, np.int64).reshape(-1, 3)
    if len(F) and (F.min() < 0 or F.max() >= len(V)):
        raise ValueError(f"{path}: face index out of range")
    return V, F.astype(np.int32)


def _msh_tets_from_nodes(path, n_nodes, tets_tagged) -> np.ndarray:
    T = np.asarray(tets_tagged, np.int64).reshape(-1, 4) - 1
    if len(T) and (T.min() < 0 or T.max() >= n_nodes):
        raise ValueError(f"{path}: tet node tag out of range")
    return T.astype(np.int32)


def read_msh(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """Nodes (n x 3 float64, in file order) and linear tets (m x 4 int32, node tag - 1) of a
    Gmsh MSH file: version 2.2 (ASCII or binary) or 4.1 (ASCII)."""
    with open(path, "rb") as f:
        data = f.read()
    pos = data.index(b"$MeshFormat")
    line_end = data.index(b"\n", pos)
    hdr_end = data.index(b"\n", line_end + 1)
    version, ftype, dsize = data[line_end + 1:hdr_end].split()[:3]
    version, ftype, dsize = version.decode(), int(ftype), int(dsize)
    if version.startswith("2"):
        return _read_msh2(path, data, binary=ftype == 1, dsize=dsize)
    if version.startswith("4.1") and ftype == 0:
        return _read_msh41_ascii(path, data)
    raise ValueError(f"{path}: unsupported MSH version {version} (file type {ftype})")


def _section(data: bytes, name: str) -> Tuple[int, int]:
    b = data.index(b"$" + name.encode())
    b = data.index(b"\n", b) + 1
    e = data.index(b"$End" + name.encode(), b)
    return b, e


def _read_msh2(path: str, data: bytes, binary: bool, dsize: int) -> Tuple[np.ndarray, np.ndarray]:
    nb, ne = _section(data, "Nodes")
    eb, ee = _section(data, "Elements")
    if not binary:
        nl = data[nb:ne].split(b"\n")
        n = int(nl[0])
        V = np.array([[float(x) for x in nl[1 + i].split()[1:4]] for i in range(n)], np.float64).reshape(-1, 3)
        el = data[eb:ee].split(b"\n")
        m = int(el[0])
        tets = []
        for i in range(m):
            p = [int(x) for x in el[1 + i].split()]
            if p[1] == 4:
                ntag = p[2]
                tets.append(p[3 + ntag:7 + ntag])
        return V, _msh_tets_from_nodes(path, len(V), tets)
    if dsize != 8:
        raise ValueError(f"{path}: binary MSH with {dsize}-byte reals")
    e = data.index(b"\n", nb)
    n = int(data[nb:e])
    rec = np.dtype([("tag", "<i4"), ("xyz", "<f8", 3)])
    V = np.frombuffer(data, rec, n, e + 1)["xyz"].astype(np.float64)
    e = data.index(b"\n", eb)
    m = int(data[eb:e])
    off = e + 1
    tets = []
    seen = 0
    nodes_of = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 10: 9, 11: 10, 15: 1}
    while seen < m:
        etype, nfollow, ntags = struct.unpack_from("<3i", data, off)
        off += 12
        if etype not in nodes_of:
            raise ValueError(f"{path}: unsupported element type {etype}")
        k = 1 + ntags + nodes_of[etype]
        block = np.frombuffer(data, "<i4", nfollow * k, off).reshape(nfollow, k)
        off += 4 * nfollow * k
        if etype == 4:
            tets.append(block[:, 1 + ntags:])
        seen += nfollow
    T = np.concatenate(tets) if tets else np.zeros((0, 4), np.int64)
    return V, _msh_tets_from_nodes(path, len(V), T)


def _read_msh41_ascii(path: str, data: bytes) -> Tuple[np.ndarray, np.ndarray]:
    nb, ne = _section(data, "Nodes")
    tok = data[nb:ne].split()
    nblocks, nnodes = int(tok[0]), int(tok[1])
    k = 4
    coords = []
    for _ in range(nblocks):
        param, cnt = int(tok[k + 2]), int(tok[k + 3])
        k += 4 + cnt  # entity dim, tag, parametric, count, then the node tags
        if param:
            raise ValueError(f"{path}: parametric nodes are not supported")
        coords.append(np.array(tok[k:k + 3 * cnt], np.float64).reshape(cnt, 3))
        k += 3 * cnt
    V = np.concatenate(coords) if coords else np.zeros((0, 3))
    if len(V) != nnodes:
        raise ValueError(f"{path}: node count mismatch")
    eb, ee = _section(data, "Elements")
    tok = data[eb:ee].split()
    nblocks = int(tok[0])
    k = 4
    nodes_of = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 10: 9, 11: 10, 15: 1}
    tets = []
    for _ in range(nblocks):
        dim, etype, cnt = int(tok[k]), int(tok[k + 2]), int(tok[k + 3])
        k += 4
        if etype not in nodes_of:
            raise ValueError(f"{path}: unsupported element type {etype}")
        w = 1 + nodes_of[etype]
        blk = np.array(tok[k:k + w * cnt], np.int64).reshape(cnt, w)
        k += w * cnt
        if dim == 3 and etype == 4:
            tets.append(blk[:, 1:])
    T = np.concatenate(tets) if tets else np.zeros((0, 4), np.int64)
    return V, _msh_tets_from_nodes(path, len(V), T)


# ----------------------------------------------------------------------------
# meshes -> Scene
# ----------------------------------------------------------------------------

def rotation(deg: Sequence[float]) -> np.ndarray:
    """R = R_z R_y R_x for angles in degrees (q_z * q_y * q_x, mesh_from_config.h:26-31)."""
    ax, ay, az = (PI_REF * float(a) / 180.0 for a in deg)
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ ry @ rx


def transform_mesh(V: np.ndarray, spec: MeshSpec, centralize: bool) -> np.ndarray:
    V = np.asarray(V, np.float64)
    if centralize and len(V):
        V = V - V.mean(0)
    R = rotation(spec.rotate)
    if spec.type == "tet":
        V = (V @ R.T) * spec.scale
    else:
        V = (V * spec.scale) @ R.T
    return V + np.asarray(spec.translate, np.float64)


def _d_entries(sc: S.Scene):
    """(row, vertex, coefficient) of D over the elastic rows (triangles, tets, bending)."""
    rows, cols, vals = [], [], []
    r0 = sc.tri_start_row
    for t in range(len(sc.tri_inds)):
        Bi = sc.tri_binv[t].reshape(2, 2).astype(np.float64)
        v = sc.tri_inds[t]
        for r in range(2):
            c1, c2 = Bi[0, r], Bi[1, r]
            rows += [r0 + 2 * t + r] * 3
            cols += [v[0], v[1], v[2]]
            vals += [-(c1 + c2), c1, c2]
    r0 = sc.tet_start_row
    for t in range(len(sc.tet_inds)):
        Bi = sc.tet_binv[t].reshape(3, 3).astype(np.float64)
        v = sc.tet_inds[t]
        for r in range(3):
            c = Bi[:, r]
            rows += [r0 + 3 * t + r] * 4
            cols += [v[0], v[1], v[2], v[3]]
            vals += [-(c[0] + c[1] + c[2]), c[0], c[1], c[2]]
    r0 = sc.bend_start_row
    for b in range(len(sc.bend_w)):
        o0, o1 = sc.bend_offsets[b], sc.bend_offsets[b + 1]
        rows += [r0 + b] * (o1 - o0)
        cols += list(sc.bend_inds[o0:o1])
        vals += list(sc.bend_coeffs[o0:o1].astype(np.float64))
    return np.asarray(rows, np.int64), np.asarray(cols, np.int64), np.asarray(vals, np.float64)


def heuristic_contact_weights(sc: S.Scene, h: float, kl: float, km: float, sigma: float, beta: float) -> np.ndarray:
    """Contact weights of ``use_heu_wc`` (admm_impl_gpu.cu:188-218) for the dynamic surface
    vertices; other vertices keep their weights."""
    n = sc.n_dyn
    m = sc.mass[:n].astype(np.float64)
    rows, cols, vals = _d_entries(sc)
    w_row = np.concatenate([np.repeat(sc.tri_w, 2), np.repeat(sc.tet_w, 3), sc.bend_w]).astype(np.float64)
    keep = cols < n
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    wr = w_row[rows]
    dtwd = np.zeros(n)
    np.add.at(dtwd, cols, wr * wr * vals * vals)       # diag of D^T W^2 D
    dwd = np.zeros(n)
    np.add.at(dwd, cols, wr * vals * vals)             # diag of D^T W D (damping)
    a = m + h * h * dtwd + h * (kl * dwd + km * m)
    # pins (D row e_i, weight w) are part of D^T W^2 D, not of the damping term
    for i, w in zip(sc.pin_inds, sc.pin_w.astype(np.float64)):
        if i < n:
            a[i] += h * h * w * w
    wc = sc.contact_w.astype(np.float64).copy()
    surf = np.zeros(sc.n_vert, bool)
    surf[sc.surf_verts] = True
    s = surf[:n]
    wc_dyn = np.maximum(sigma * a, np.minimum(beta * m, a)) * (1.0 / (h * h)) * 10.0
    wc[:n][s] = wc_dyn[s]
    return wc.astype(np.float32)


def load_scene(path: str, resource_root: Optional[str] = None, cfg: Optional[AppConfig] = None,
               params: Optional[S.SolverParams] = None) -> S.Scene:
    """Scene of a scene file.  Mesh paths are relative to `resource_root` (default: the folder
    above the scene file's folder, the reference's ``resource/`` layout)."""
    cfg = cfg or parse_config(path)
    if resource_root is None:
        resource_root = os.path.dirname(os.path.dirname(os.path.abspath(path)))
    h = cfg.substep_dt
    p = params or S.SolverParams()
    p = dataclasses.replace(
        p, dt=h, g=cfg.g, mu=cfg.mu, kappa=cfg.kappa, beta=cfg.beta, thickness=cfg.thickness,
        admm_max_iter=cfg.admm_max_iter, dcd_interval=cfg.dcd_interval, gs_max_iter=cfg.gs_max_iter,
        jacobi_iter=cfg.global_jacobi_iter, max_contacts=cfg.max_collision, enable_contact=cfg.contact_enable,
        warmstart_ue=cfg.warmstart_ue, warmstart_uc=cfg.warmstart_uc, w_scale=cfg.w_scale)
    order = [m for m in cfg.meshes if m.type in ("tri", "tet")] + [m for m in cfg.meshes if m.type == "static"]
    bodies = []
    meshes = []
    off = 0
    for mesh_id, spec in enumerate(order):
        full = os.path.join(resource_root, spec.path)
        if not os.path.exists(full):
            raise FileNotFoundError(f"mesh file not found: {full}")
        if spec.type == "tet":
            V, T = read_msh(full)
            F = np.zeros((0, 3), np.int32)
        else:
            V, F = read_obj(full)
            T = np.zeros((0, 4), np.int32)
        V = transform_mesh(V, spec, mesh_id in cfg.center_ids)
        static = spec.type == "static"
        bodies.append(S._Body(V, F, T, 1e12 if static else spec.density, spec.stretch,
                              spec.bending if spec.type == "tri" else 0.0, static=static))
        meshes.append({"start": off, "end": off + len(V), "faces": F.astype(np.int64) + off, "type": spec.type})
        off += len(V)
    sc = S.assemble(cfg.scene_name, bodies, list(cfg.pin_ids), p,
                    meta={"config": "scene file", "path": os.path.abspath(path), "meshes": meshes})
    if cfg.contact_enable and cfg.use_heu_wc:
        sc.contact_w = heuristic_contact_weights(sc, h, cfg.damp_kl, cfg.damp_km, cfg.wc_sigma, cfg.wc_beta)
    return sc


# ----------------------------------------------------------------------------
# scripted static meshes (ScriptAnimator)
# ----------------------------------------------------------------------------

def read_track(path: str) -> Dict[str, np.ndarray]:
    """A track file (animator.cpp:9-63): a path containing "sequence" holds per-vertex
    positions ``points`` [frames x vertices x 3]; any other holds a rigid motion ``pos``
    [frames x 3] and ``quat`` [frames x 4] (x, y, z, w).  Values are converted to float32 (the
    reference reinterprets the stored bytes as float32, which garbles float64 files such as its
    own tracks; the values are what the files mean)."""
    with np.load(path) as d:
        if "sequence" in path:
            if "points" not in d.files:
                raise ValueError(f"{path}: no 'points' array")
            pts = np.asarray(d["points"], np.float64)
            if pts.ndim != 3 or pts.shape[2] != 3:
                raise ValueError(f"{path}: 'points' must be frames x vertices x 3")
            return {"kind": "points", "points": pts.astype(np.float32)}
        if "pos" not in d.files or "quat" not in d.files:
            raise ValueError(f"{path}: rigid track needs 'pos' and 'quat'")
        pos = np.asarray(d["pos"], np.float64)
        quat = np.asarray(d["quat"], np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3 or quat.ndim != 2 or quat.shape[1] != 4 or len(pos) != len(quat):
        raise ValueError(f"{path}: 'pos' must be frames x 3 and 'quat' frames x 4")
    if len(pos) < 3:
        raise ValueError(f"{path}: a rigid track needs at least 3 frames")
    return {"kind": "rigid", "pos": pos.astype(np.float32), "quat": quat.astype(np.float32)}


def scene_tracks(cfg: AppConfig, sc: S.Scene, resource_root: Optional[str] = None,
                 scene_path: Optional[str] = None) -> List[dict]:
    """Tracks of the animated static meshes of a loaded scene, in mesh-id order (the order the
    reference's animator applies them), with their vertex ranges and mesh transforms."""
    if resource_root is None:
        base = scene_path or sc.meta.get("path", "")
        resource_root = os.path.dirname(os.path.dirname(os.path.abspath(base)))
    order = [m for m in cfg.meshes if m.type in ("tri", "tet")] + [m for m in cfg.meshes if m.type == "static"]
    meshes = sc.meta.get("meshes")
    if meshes is None or len(meshes) != len(order):
        raise ValueError("scene was not loaded from this scene file")
    out = []
    for mesh_id, spec in enumerate(order):
        if spec.type != "static" or not spec.animate:
            continue
        tr = read_track(os.path.join(resource_root, spec.animate))
        m = meshes[mesh_id]
        tr.update(v_begin=m["start"], v_end=m["end"], mesh_id=mesh_id,
                  rot=rotation(spec.rotate), translate=np.asarray(spec.translate, np.float64), scale=spec.scale)
        if tr["kind"] == "points" and tr["points"].shape[1] != m["end"] - m["start"]:
            raise ValueError(f"{spec.animate}: {tr['points'].shape[1]} points for a mesh of "
                             f"{m['end'] - m['start']} vertices")
        out.append(tr)
    return out


def attach_tracks(handle, tracks: Sequence[dict]) -> None:
    """Attach the tracks to a backend handle (replacing any it had)."""
    handle.clear_tracks()
    for tr in tracks:
        if tr["kind"] == "rigid":
            handle.set_rigid_track(tr["v_begin"], tr["v_end"], tr["pos"], tr["quat"])
        else:
            handle.set_point_track(tr["v_begin"], tr["v_end"], tr["points"], tr["rot"], tr["translate"], tr["scale"])
