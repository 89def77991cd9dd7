"""Synthetic scenes and constraint set-up for the ADMM substep.

This module is the application-layer side of the backend boundary: it turns
meshes into the per-type constraint records the backend consumes, exactly as
the reference's app layer does before it calls ``add_constraints`` /
``set_constraint_dim`` / ``finalize_constraints``:

* triangle strain   -- ``src/constraint/triangle_constraint.h:24-62``
  (``Binv = (basis^T [e12 e13])^-1``, ``area``, ``w = sqrt(k*area)``)
* tetrahedral strain -- ``src/constraint/tetrahedral_constraint.h:22-56``
  (``Binv = [e12 e13 e14]^-1``, ``volume = |det|/6``, ``w = sqrt(k*volume)``)
* Laplacian bending  -- ``src/constraint/bending_constraint.h:24-78,127-171``
  (mean-value (cotangent) ring weights, scaled by ``1/(2*varea)/100``,
  middle coefficient = -sum(ring), rest curvature forced to 0)
* pins               -- ``src/constraint/pin_constraint.h:18-57`` (k = 1e5)
* row bookkeeping    -- ``src/constraint/mesh_to_constraint.h:94-151`` and
  ``src/app/app_initializer.cpp:144-172``: all triangles (2 rows each), then
  all tets (3 rows), then bending (1 row), then pins (1 row).
* lumped mass        -- ``src/mesh/mesh_container.h:452-472``
* surface sets       -- ``src/mesh/mesh_container.h:232-335``
* contact weights    -- ``src/solver/solver_config_applier.cpp:34-47``
  (``w_c = m/h^2 * w_scale`` for dynamic vertices, 1e12 for static ones)

Vertex ring order for bending follows libigl v2.5.0 ``igl::adjacency_list``
called with ``sorted=false`` (``mesh_container.h:236``), whose rings are the
sorted, de-duplicated neighbour indices.

Setup runs once per scene on the host in float64 and is rounded to float32,
the reference's ``ADU::Real``.  None of it is on the per-step hot path.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Tuple

import numpy as np

PI_REF = 3.1415926  # the constant bending_constraint.h:51 uses for varea


@dataclasses.dataclass
class SolverParams:
    """Typed tuning parameters (mirror of ``ADMMSolverConfig``, admm_config.h:13-54)."""
    dt: float = 0.01
    g: float = 9.8
    mu: float = 0.5
    kappa: float = 1e6
    beta: float = 1e5
    thickness: float = 5e-3
    admm_max_iter: int = 25
    dcd_interval: int = 5
    gs_max_iter: int = 10
    jacobi_iter: int = 20
    max_contacts: int = 100000
    enable_contact: bool = True
    warmstart_ue: bool = True
    warmstart_uc: bool = True
    w_scale: float = 200.0
    bvh_refit: bool = True
    ell_lanes: int = 0
    jacobi_mode: int = 0  # 0 autotuned, 1 one kernel per sweep, 2 persistent global step
    broad_phase: int = 0  # 0 default (grid), 1 LBVH, 2 uniform grid
    global_solver: int = 0  # 0 Jacobi (reference), 1 PCG with diag(A), 2 PCG with learned blocks
    pcg_iter: int = 0  # 0 = jacobi_iter // 2
    query_lanes: int = 0  # lanes per grid DCD query: 0 chosen from the query count, or 8, 16, 32
    contact_semantics: int = 0  # contact predicates: 0 the GPU backend's, 1 the CPU backend's
    backend_semantics: int = 0  # solver: 0 the GPU backend's, 1 the CPU backend's (damping, GS contact)
    damp_k_L: float = 1e-4      # Rayleigh damping of the CPU backend (admm_config.h:52-53)
    damp_k_M: float = 0.0


@dataclasses.dataclass
class Scene:
    """Everything the backend needs, in the reference's layouts (row-major N x 3 float32)."""
    name: str
    verts: np.ndarray            # (n, 3) float32, dynamic vertices first
    n_dyn: int                   # static_vert_begin
    mass: np.ndarray             # (n,) float32
    is_fixed: np.ndarray         # (n,) int32, 1 for pinned vertices
    # triangle strain
    tri_inds: np.ndarray         # (nt, 3) int32
    tri_binv: np.ndarray         # (nt, 4) float32, row-major 2x2
    tri_w: np.ndarray            # (nt,) float32
    # tetrahedral strain
    tet_inds: np.ndarray         # (nT, 4) int32
    tet_binv: np.ndarray         # (nT, 9) float32, row-major 3x3
    tet_w: np.ndarray            # (nT,) float32
    # bending (CSR: entry 0 of each segment is the middle vertex)
    bend_offsets: np.ndarray     # (nb+1,) int32
    bend_inds: np.ndarray        # (sum,) int32
    bend_coeffs: np.ndarray      # (sum,) float32
    bend_w: np.ndarray           # (nb,) float32
    # pins
    pin_inds: np.ndarray         # (np,) int32
    pin_pos: np.ndarray          # (np, 3) float32
    pin_w: np.ndarray            # (np,) float32
    # collision geometry
    surf_tris: np.ndarray        # (ns, 3) int32
    surf_edges: np.ndarray       # (ne, 2) int32
    surf_verts: np.ndarray       # (nsv,) int32, sorted
    contact_w: np.ndarray        # (n,) float32
    params: SolverParams
    meta: Dict[str, object] = dataclasses.field(default_factory=dict)
    vert_mu: Optional[np.ndarray] = None  # (n,) float32 per-vertex friction, or None (params.mu)

    # --- row bookkeeping (mesh_to_constraint.h order) ---
    @property
    def tri_start_row(self) -> int:
        return 0

    @property
    def tet_start_row(self) -> int:
        return 2 * len(self.tri_inds)

    @property
    def bend_start_row(self) -> int:
        return self.tet_start_row + 3 * len(self.tet_inds)

    @property
    def pin_start_row(self) -> int:
        return self.bend_start_row + len(self.bend_w)

    @property
    def n_rows(self) -> int:
        return self.pin_start_row + len(self.pin_inds)

    @property
    def n_vert(self) -> int:
        return int(self.verts.shape[0])

    def is_surf(self) -> np.ndarray:
        s = np.zeros(self.n_vert, dtype=np.uint8)
        s[self.surf_verts] = 1
        return s

    def summary(self) -> Dict[str, int]:
        return {
            "n_vert": self.n_vert, "n_dyn": self.n_dyn, "n_tri": len(self.tri_inds),
            "n_tet": len(self.tet_inds), "n_bend": len(self.bend_w), "n_pin": len(self.pin_inds),
            "n_rows": self.n_rows, "n_surf_tri": len(self.surf_tris),
            "n_surf_edge": len(self.surf_edges), "n_surf_vert": len(self.surf_verts),
        }


# ----------------------------------------------------------------------------
# constraint constructors
# ----------------------------------------------------------------------------

def _normalized(v: np.ndarray) -> np.ndarray:
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def triangle_constraints(verts: np.ndarray, faces: np.ndarray, k: float):
    """Binv, area, w for each triangle (triangle_constraint.h:24-62)."""
    v = verts.astype(np.float64)
    e12 = v[faces[:, 1]] - v[faces[:, 0]]
    e13 = v[faces[:, 2]] - v[faces[:, 0]]
    n1 = _normalized(e12)
    n2 = _normalized(e13 - np.sum(e13 * n1, axis=1, keepdims=True) * n1)
    # basis^T * edges (2x2): [[n1.e12, n1.e13], [n2.e12, n2.e13]]
    m = np.empty((len(faces), 2, 2))
    m[:, 0, 0] = np.sum(n1 * e12, 1)
    m[:, 0, 1] = np.sum(n1 * e13, 1)
    m[:, 1, 0] = np.sum(n2 * e12, 1)
    m[:, 1, 1] = np.sum(n2 * e13, 1)
    det = m[:, 0, 0] * m[:, 1, 1] - m[:, 0, 1] * m[:, 1, 0]
    area = det / 2.0
    if np.any(area < 0):
        raise ValueError("TriangleConstraint: inverted initial pose")
    binv = np.linalg.inv(m)
    w = np.sqrt(k * area)
    return binv.reshape(-1, 4).astype(np.float32), area, w.astype(np.float32)


def tet_constraints(verts: np.ndarray, tets: np.ndarray, k):
    """Binv, volume, w for each tet (tetrahedral_constraint.h:22-56)."""
    v = verts.astype(np.float64)
    b0 = np.stack([v[tets[:, 1]] - v[tets[:, 0]],
                   v[tets[:, 2]] - v[tets[:, 0]],
                   v[tets[:, 3]] - v[tets[:, 0]]], axis=2)  # columns e12 e13 e14
    binv = np.linalg.inv(b0)
    vol = np.abs(np.linalg.det(b0) / 6.0)
    w = np.sqrt(np.asarray(k, dtype=np.float64) * vol)
    return binv.reshape(-1, 9).astype(np.float32), vol, w.astype(np.float32)


def adjacency_lists(faces: np.ndarray, n: int) -> List[np.ndarray]:
    """igl::adjacency_list(F, A) with sorted=false: sorted unique neighbours."""
    a = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    a = np.concatenate([a, a[:, ::-1]])
    a = np.unique(a, axis=0)
    starts = np.searchsorted(a[:, 0], np.arange(n + 1))
    return [a[starts[i]:starts[i + 1], 1] for i in range(n)]


def _cot_at(v1, v2, v3):
    a = v1 - v2
    b = v3 - v2
    return np.dot(a, b) / np.linalg.norm(np.cross(a, b))


def _co_linear(v1, v2, v3):
    c = np.cross(v1 - v2, v3 - v2)
    return np.dot(c, c) < 1e-7


def bending_constraints(verts: np.ndarray, faces: np.ndarray, vert_range: Tuple[int, int], k: float):
    """Mean-value Laplacian bending rows (bending_constraint.h:24-78,127-171), vectorised.

    For every vertex with a ring of >= 3 neighbours: radius = mean |ring - mid|,
    varea = pi r^2 / 3, ring weight i = cot at mid towards ring[i+1] + cot towards
    ring[i-1] (each skipped when the three points are co-linear,
    |cross|^2 < 1e-7), scaled by 1/(2 varea)/100; the middle coefficient is the
    sum of the ring weights and the ring weights are negated; w = sqrt(k varea).
    """
    n = verts.shape[0]
    v = verts.astype(np.float64)
    e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    e = np.concatenate([e, e[:, ::-1]])
    e = np.unique(e, axis=0)                       # sorted (vertex, neighbour) pairs
    lo, hi = vert_range
    e = e[(e[:, 0] >= lo) & (e[:, 0] < hi)]
    starts = np.searchsorted(e[:, 0], np.arange(n + 1))
    deg = np.diff(starts)
    mids = np.nonzero(deg >= 3)[0]
    mids = mids[(mids >= lo) & (mids < hi)]
    if len(mids) == 0:
        return (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32), np.zeros(0, np.float32))
    d = deg[mids]
    seg = np.repeat(np.arange(len(mids)), d)
    base = starts[mids]
    pos = np.arange(d.sum()) - np.repeat(np.cumsum(d) - d, d)     # position within the ring
    ring = e[np.repeat(base, d) + pos, 1]
    nxt = e[np.repeat(base, d) + (pos + 1) % np.repeat(d, d), 1]
    prv = e[np.repeat(base, d) + (pos + np.repeat(d, d) - 1) % np.repeat(d, d), 1]
    mid = np.repeat(mids, d)
    pm = v[mid]
    dist = np.linalg.norm(v[ring] - pm, axis=1)
    radius = np.bincount(seg, weights=dist) / d
    varea = PI_REF * radius * radius / 3.0

    def cot_term(a_idx, c_idx):
        a = v[a_idx] - pm
        b = v[c_idx] - pm
        cr = np.cross(a, b)
        c2 = np.sum(cr * cr, axis=1)
        ok = c2 >= 1e-7
        val = np.zeros(len(a))
        val[ok] = np.sum(a * b, axis=1)[ok] / np.sqrt(c2[ok])
        return val
    c = cot_term(ring, nxt) + cot_term(ring, prv)
    c = c / (2.0 * varea[seg]) / 100.0
    middle = np.bincount(seg, weights=c, minlength=len(mids))
    offsets = np.zeros(len(mids) + 1, np.int64)
    offsets[1:] = np.cumsum(d + 1)
    inds = np.empty(offsets[-1], np.int64)
    coeffs = np.empty(offsets[-1], np.float64)
    inds[offsets[:-1]] = mids
    coeffs[offsets[:-1]] = middle
    ring_slot = np.repeat(offsets[:-1] + 1, d) + pos
    inds[ring_slot] = ring
    coeffs[ring_slot] = -c
    ws = np.sqrt(k * varea)
    return (offsets.astype(np.int32), inds.astype(np.int32), coeffs.astype(np.float32), ws.astype(np.float32))


def lumped_mass(n: int, verts: np.ndarray, faces: np.ndarray, face_density: np.ndarray,
                tets: np.ndarray, tet_density: np.ndarray) -> np.ndarray:
    """Area/3 and volume/4 lumping (mesh_container.h:475-494)."""
    v = verts.astype(np.float64)
    mass = np.zeros(n)
    if len(faces):
        area = 0.5 * np.linalg.norm(np.cross(v[faces[:, 1]] - v[faces[:, 0]],
                                             v[faces[:, 2]] - v[faces[:, 0]]), axis=1)
        for j in range(3):
            mass += np.bincount(faces[:, j], weights=area / 3.0 * face_density, minlength=n)
    if len(tets):
        d = np.stack([v[tets[:, 1]] - v[tets[:, 0]], v[tets[:, 2]] - v[tets[:, 0]],
                      v[tets[:, 3]] - v[tets[:, 0]]], axis=2)
        vol = np.abs(np.linalg.det(d)) / 6.0
        for j in range(4):
            mass += np.bincount(tets[:, j], weights=vol / 4.0 * tet_density, minlength=n)
    return mass


def unique_edges(tris: np.ndarray) -> np.ndarray:
    """Undirected edges (i < j) of a triangle list, sorted lexicographically."""
    if len(tris) == 0:
        return np.zeros((0, 2), np.int32)
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0).astype(np.int32)


def boundary_facets(tets: np.ndarray) -> np.ndarray:
    """Faces that belong to exactly one tet, oriented outward (igl::boundary_facets)."""
    faces = np.concatenate([tets[:, [1, 2, 3]], tets[:, [0, 3, 2]],
                            tets[:, [0, 1, 3]], tets[:, [0, 2, 1]]])
    key = np.sort(faces, axis=1).astype(np.int64)
    nv = int(key.max()) + 1 if len(key) else 1
    # one int64 per sorted face (nv^3 < 2^63 for nv < 2 M), so the duplicate count is a 1-D unique
    k1 = (key[:, 0] * nv + key[:, 1]) * nv + key[:, 2]
    _, inv, cnt = np.unique(k1, return_inverse=True, return_counts=True)
    return faces[cnt[inv.ravel()] == 1].astype(np.int32)


# ----------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------

def grid_cloth(nx: int, side: float) -> Tuple[np.ndarray, np.ndarray]:
    """nx x nx vertex grid in the XZ plane centred at the origin."""
    t = np.linspace(-side / 2, side / 2, nx)
    xx, zz = np.meshgrid(t, t, indexing="ij")
    verts = np.stack([xx.ravel(), np.zeros(nx * nx), zz.ravel()], 1)
    idx = np.arange(nx * nx).reshape(nx, nx)
    a = idx[:-1, :-1].ravel()
    b = idx[1:, :-1].ravel()
    c = idx[1:, 1:].ravel()
    d = idx[:-1, 1:].ravel()
    # counter-clockwise seen from +y so that the triangle-constraint area is positive
    tris = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b], 1)])
    return verts, tris.astype(np.int32)


def box_mesh(lo, hi) -> Tuple[np.ndarray, np.ndarray]:
    lo = np.asarray(lo, float)
    hi = np.asarray(hi, float)
    v = np.array([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [hi[0], hi[1], lo[2]], [lo[0], hi[1], lo[2]],
                  [lo[0], lo[1], hi[2]], [hi[0], lo[1], hi[2]], [hi[0], hi[1], hi[2]], [lo[0], hi[1], hi[2]]])
    f = np.array([[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4],
                  [3, 6, 2], [3, 7, 6], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]], np.int32)
    return v, f


def ground_quad(half: float, y: float) -> Tuple[np.ndarray, np.ndarray]:
    v = np.array([[-half, y, -half], [half, y, -half], [half, y, half], [-half, y, half]])
    f = np.array([[0, 2, 1], [0, 3, 2]], np.int32)
    return v, f


def icosphere(radius: float, subdiv: int) -> Tuple[np.ndarray, np.ndarray]:
    p = (1 + 5 ** 0.5) / 2
    v = [[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
         [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
         [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    verts = [np.asarray(x, float) / np.linalg.norm(x) for x in v]
    faces = f
    for _ in range(subdiv):
        cache: Dict[Tuple[int, int], int] = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        faces = nf
    return np.asarray(verts) * radius, np.asarray(faces, np.int32)


def tet_cube(n: int, side: float) -> Tuple[np.ndarray, np.ndarray]:
    """(n+1)^3 lattice, 5 tets per cell with alternating orientation (conforming)."""
    t = np.linspace(0.0, side, n + 1)
    xx, yy, zz = np.meshgrid(t, t, t, indexing="ij")
    verts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    idx = np.arange((n + 1) ** 3).reshape(n + 1, n + 1, n + 1)
    tets = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                c = [idx[i + a, j + b, k + cc] for a in (0, 1) for b in (0, 1) for cc in (0, 1)]
                # c index = a*4 + b*2 + cc
                if (i + j + k) % 2 == 0:
                    cells = [(0, 4, 2, 1), (6, 2, 4, 7), (5, 1, 7, 4), (3, 7, 1, 2), (1, 2, 4, 7)]
                else:
                    cells = [(4, 0, 6, 5), (2, 6, 0, 3), (1, 5, 3, 0), (7, 3, 5, 6), (0, 3, 5, 6)]
                for q in cells:
                    tets.append([c[q[0]], c[q[1]], c[q[2]], c[q[3]]])
    tets = np.asarray(tets, np.int32)
    # orient every tet positively (det > 0)
    v = verts
    d = np.stack([v[tets[:, 1]] - v[tets[:, 0]], v[tets[:, 2]] - v[tets[:, 0]], v[tets[:, 3]] - v[tets[:, 0]]], 2)
    neg = np.linalg.det(d) < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    return verts, tets


def tet_lattice(dims: Tuple[int, int, int], cell: float, keep=None) -> Tuple[np.ndarray, np.ndarray]:
    """Lattice of dims cells (edge `cell`), 5 tets per kept cell with alternating orientation
    (conforming), unused lattice vertices removed.  keep(centres) -> bool mask of cells."""
    nx, ny, nz = dims
    gx, gy, gz = [np.arange(d + 1) * cell for d in dims]
    xx, yy, zz = np.meshgrid(gx, gy, gz, indexing="ij")
    verts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    idx = np.arange((nx + 1) * (ny + 1) * (nz + 1)).reshape(nx + 1, ny + 1, nz + 1)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    if keep is not None:
        m = keep(np.stack([(ii + 0.5) * cell, (jj + 0.5) * cell, (kk + 0.5) * cell], 1))
        ii, jj, kk = ii[m], jj[m], kk[m]
    corner = np.stack([idx[ii + a, jj + b, kk + c] for a in (0, 1) for b in (0, 1) for c in (0, 1)], 1)
    even = ((ii + jj + kk) % 2 == 0)
    pat_e = np.array([(0, 4, 2, 1), (6, 2, 4, 7), (5, 1, 7, 4), (3, 7, 1, 2), (1, 2, 4, 7)])
    pat_o = np.array([(4, 0, 6, 5), (2, 6, 0, 3), (1, 5, 3, 0), (7, 3, 5, 6), (0, 3, 5, 6)])
    tets = np.concatenate([corner[even][:, pat_e].reshape(-1, 4), corner[~even][:, pat_o].reshape(-1, 4)])
    used, inv = np.unique(tets.ravel(), return_inverse=True)
    tets = inv.reshape(-1, 4).astype(np.int32)
    verts = verts[used]
    d = np.stack([verts[tets[:, 1]] - verts[tets[:, 0]], verts[tets[:, 2]] - verts[tets[:, 0]],
                  verts[tets[:, 3]] - verts[tets[:, 0]]], 2)
    neg = np.linalg.det(d) < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    return verts, tets


def _rot_y(theta: float) -> np.ndarray:
    c, s = math.cos(theta), math.sin(theta)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def _rand_rot(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


# ----------------------------------------------------------------------------
# scene assembly
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class _Body:
    verts: np.ndarray
    tris: np.ndarray          # triangle-strain faces (cloth) or empty
    tets: np.ndarray          # tets or empty
    density: float
    k_stretch: float
    k_bend: float = 0.0
    static: bool = False
    mu: Optional[float] = None    # friction of this body's vertices (None: the scene's mu)


def assemble(name: str, bodies: List[_Body], pins: List[int], params: SolverParams,
             meta: Optional[Dict[str, object]] = None) -> Scene:
    """Concatenate dynamic bodies then static bodies and build every constraint record."""
    dyn = [b for b in bodies if not b.static]
    sta = [b for b in bodies if b.static]
    verts, faces, f_dens, tets, t_dens = [], [], [], [], []
    surf_tris = []
    tri_faces, tri_k, tet_all, tet_k = [], [], [], []
    bend_jobs = []
    off = 0
    for b in dyn + sta:
        nv = len(b.verts)
        verts.append(b.verts)
        if len(b.tris):
            faces.append(b.tris + off)
            f_dens.append(np.full(len(b.tris), b.density))
            surf_tris.append(b.tris + off)
            if not b.static:
                tri_faces.append(b.tris + off)
                tri_k.append(np.full(len(b.tris), b.k_stretch))
                bend_jobs.append((b.tris + off, (off, off + nv), b.k_bend))
        if len(b.tets):
            tets.append(b.tets + off)
            t_dens.append(np.full(len(b.tets), b.density))
            tet_all.append(b.tets + off)
            tet_k.append(np.broadcast_to(np.asarray(b.k_stretch, float), (len(b.tets),)))
            surf_tris.append(boundary_facets(b.tets + off))
        off += nv
    n_dyn = int(sum(len(b.verts) for b in dyn))
    V = np.concatenate(verts).astype(np.float64)
    n = len(V)
    F = np.concatenate(faces).astype(np.int32) if faces else np.zeros((0, 3), np.int32)
    T = np.concatenate(tets).astype(np.int32) if tets else np.zeros((0, 4), np.int32)
    mass = lumped_mass(n, V, F, np.concatenate(f_dens) if f_dens else np.zeros(0), T,
                       np.concatenate(t_dens) if t_dens else np.zeros(0))
    # float32 positions are the state; constraints are built from them like the reference
    V32 = V.astype(np.float32)
    if tri_faces:
        TF = np.concatenate(tri_faces)
        tri_binv, _, _ = triangle_constraints(V32, TF, 1.0)
        _, area, _ = triangle_constraints(V32, TF, 1.0)
        tri_w = np.sqrt(np.concatenate(tri_k) * area).astype(np.float32)
    else:
        TF = np.zeros((0, 3), np.int32)
        tri_binv = np.zeros((0, 4), np.float32)
        tri_w = np.zeros(0, np.float32)
    if tet_all:
        TT = np.concatenate(tet_all)
        tet_binv, vol, _ = tet_constraints(V32, TT, 1.0)
        tet_w = np.sqrt(np.concatenate(tet_k) * vol).astype(np.float32)
    else:
        TT = np.zeros((0, 4), np.int32)
        tet_binv = np.zeros((0, 9), np.float32)
        tet_w = np.zeros(0, np.float32)
    bo, bi, bc, bw = [np.zeros(1, np.int32)], [], [], []
    for faces_b, vr, kb in bend_jobs:
        o, i, c, w = bending_constraints(V32, faces_b, vr, kb)
        bo.append(o[1:] + bo[-1][-1] if len(bo[-1]) else o[1:])
        bi.append(i)
        bc.append(c)
        bw.append(w)
    bend_offsets = np.concatenate(bo).astype(np.int32)
    bend_inds = np.concatenate(bi).astype(np.int32) if bi else np.zeros(0, np.int32)
    bend_coeffs = np.concatenate(bc).astype(np.float32) if bc else np.zeros(0, np.float32)
    bend_w = np.concatenate(bw).astype(np.float32) if bw else np.zeros(0, np.float32)
    pins = [p for p in pins if p < n_dyn]
    pin_inds = np.asarray(pins, np.int32)
    pin_pos = V32[pin_inds] if len(pins) else np.zeros((0, 3), np.float32)
    pin_w = np.full(len(pins), math.sqrt(1e5), np.float32)
    is_fixed = np.zeros(n, np.int32)
    is_fixed[pin_inds] = 1
    ST = np.concatenate(surf_tris).astype(np.int32) if surf_tris else np.zeros((0, 3), np.int32)
    # surface_edges = igl::edges(faces) ++ igl::edges(boundary tet facets)  (mesh_container.h:281-291)
    tri_e = unique_edges(F)
    tet_surf = [boundary_facets(t) for t in tet_all]
    tet_e = unique_edges(np.concatenate(tet_surf)) if tet_surf else np.zeros((0, 2), np.int32)
    SE = np.concatenate([tri_e, tet_e]).astype(np.int32)
    SV = np.unique(ST.ravel()).astype(np.int32)
    cw = np.full(n, 1e12, np.float64)
    cw[:n_dyn] = mass[:n_dyn] / (params.dt * params.dt) * params.w_scale
    vert_mu = None
    if any(b.mu is not None for b in bodies):
        vert_mu = np.concatenate([np.full(len(b.verts), params.mu if b.mu is None else b.mu)
                                  for b in dyn + sta]).astype(np.float32)
    sc = Scene(name=name, verts=V32, n_dyn=n_dyn, mass=mass.astype(np.float32), is_fixed=is_fixed,
               tri_inds=TF.astype(np.int32), tri_binv=tri_binv, tri_w=tri_w,
               tet_inds=TT.astype(np.int32), tet_binv=tet_binv, tet_w=tet_w,
               bend_offsets=bend_offsets, bend_inds=bend_inds, bend_coeffs=bend_coeffs, bend_w=bend_w,
               pin_inds=pin_inds, pin_pos=pin_pos.astype(np.float32), pin_w=pin_w,
               surf_tris=ST, surf_edges=SE, surf_verts=SV, contact_w=cw.astype(np.float32),
               params=params, meta=dict(meta or {}), vert_mu=vert_mu)
    return sc


# ----------------------------------------------------------------------------
# the synthetic configurations
# ----------------------------------------------------------------------------

def cloth_on_box(nx: int = 32, seed: int = 0, side: float = 1.0) -> Scene:
    """Square cloth (nx x nx vertices, side 1 m, 0.1 kg/m^2) 0.5 m above a fixed unit box.

    Triangle strain k = E/(1+nu) with E = 1e5, nu = 0.3 (k = 2*mu, so that the reference
    energy 1/2 k A |F-R|^2 equals the ARAP energy mu A |F-R|^2); bending k = 1e-3; two
    corners pinned; seed-jittered vertices (U(+-1e-4 m)); mu = 0.3; h = 1/200; 20 ADMM
    iterations per step.
    """
    rng = np.random.default_rng(seed)
    v, f = grid_cloth(nx, side)
    v = v + np.array([0.0, 1.0, 0.0])
    v = v + rng.uniform(-1e-4, 1e-4, size=v.shape)
    bv, bf = box_mesh([-0.5, 0.0, -0.5], [0.5, 1.0 - 0.5, 0.5])
    E, nu = 1e5, 0.3
    params = SolverParams(dt=1.0 / 200, g=9.8, mu=0.3, thickness=5e-3, admm_max_iter=20,
                          dcd_interval=5, gs_max_iter=10, jacobi_iter=20, max_contacts=200000)
    bodies = [_Body(v, f, np.zeros((0, 4), np.int32), 0.1, E / (1 + nu), 1e-3),
              _Body(bv, bf, np.zeros((0, 4), np.int32), 1e12, 0.0, static=True)]
    return assemble(f"cloth{nx}x{nx}", bodies, [0, nx - 1], params,
                    meta={"config": "cloth on box", "seed": seed, "nx": nx})


def cube_on_ground(n: int = 20, seed: int = 0, side: float = 0.5, drop: float = 1.0,
                   E: Optional[float] = None, rotate: bool = False) -> Scene:
    """Tetrahedralised cube (n^3 cells, 5 tets/cell, edge `side`) dropped `drop` m onto a ground quad.

    E log-uniform in [1e4, 1e6] per seed (unless given), nu = 0.4, k = E/(1+nu),
    density 1000 kg/m^3, mu = 0.5, h = 1/100, 30 ADMM iterations per step.
    """
    rng = np.random.default_rng(seed)
    if E is None:
        E = float(10 ** rng.uniform(4, 6))
    nu = 0.4
    v, t = tet_cube(n, side)
    v = v - side / 2
    if rotate:
        v = v @ _rand_rot(rng).T
    v = v + np.array([0.0, drop + side, 0.0])
    gv, gf = ground_quad(4.0 * side + 1.0, 0.0)
    cell = side / n
    params = SolverParams(dt=1.0 / 100, g=9.8, mu=0.5, thickness=0.6 * cell, admm_max_iter=30,
                          dcd_interval=5, gs_max_iter=10, jacobi_iter=20,
                          max_contacts=max(200000, 40 * (n + 1) ** 2))
    bodies = [_Body(v, np.zeros((0, 3), np.int32), t, 1000.0, E / (1 + nu)),
              _Body(gv, gf, np.zeros((0, 4), np.int32), 1e12, 0.0, static=True)]
    return assemble(f"cube{n}", bodies, [], params,
                    meta={"config": "tet cube on ground", "seed": seed, "E": E, "n": n})


def sheets_on_sphere(nx: int = 512, layers: int = 4, seed: int = 0, side: float = 1.0,
                     gap: float = 0.02, radius: float = 0.3, subdiv: int = 4) -> Scene:
    """`layers` cloth sheets of nx x nx vertices, `gap` m apart, random in-plane rotations, over a sphere."""
    rng = np.random.default_rng(seed)
    bodies = []
    E, nu = 1e5, 0.3
    for l in range(layers):
        v, f = grid_cloth(nx, side)
        v = v @ _rot_y(rng.uniform(0, 2 * math.pi)).T
        v = v + np.array([0.0, radius + 0.05 + l * gap, 0.0])
        bodies.append(_Body(v, f, np.zeros((0, 4), np.int32), 0.1, E / (1 + nu), 1e-3))
    sv, sf = icosphere(radius, subdiv)
    bodies.append(_Body(sv, sf, np.zeros((0, 4), np.int32), 1e12, 0.0, static=True))
    params = SolverParams(dt=1.0 / 300, g=9.8, mu=0.4, thickness=1e-3, admm_max_iter=40,
                          dcd_interval=5, gs_max_iter=10, jacobi_iter=20, max_contacts=4_000_000)
    return assemble(f"sheets{layers}x{nx}", bodies, [], params,
                    meta={"config": "sheets on sphere", "seed": seed, "nx": nx, "layers": layers})


def batch_bodies(n_bodies: int = 256, seed: int = 0, vmin: int = 500, vmax: int = 20000,
                 only: Optional[List[int]] = None) -> Scene:
    """`n_bodies` independent tet soft bodies of uneven size: cubes and voxelised ellipsoids with
    log-uniform vertex counts in [vmin, vmax], E log-uniform in [1e4, 1e6], friction U(0.2, 0.6)
    per body, each released at rest with its lowest point 6-20 mm above the ground (contact
    thickness 12 mm), so the ground contacts start in the first frames and last through the
    run.  The bodies sit on a square layout with gaps wider than any body, over one ground quad
    (for bodies that never meet, the same as a ground each); h = 1/100, 30 ADMM iterations.
    The engine treats the batch as one scene: one block-diagonal segmented matrix, one
    collision grid.  `only` keeps the listed bodies (same sizes, materials and placements as
    in the full batch), e.g. a size-stratified sample for a CPU baseline.
    """
    rng = np.random.default_rng(seed)
    cell = 0.02
    bodies = []
    nside = int(math.ceil(math.sqrt(n_bodies)))
    pitch = 0.0
    specs = []
    for b in range(n_bodies):
        target = math.exp(rng.uniform(math.log(vmin), math.log(vmax)))
        ellipsoid = bool(rng.random() < 0.5)
        if ellipsoid:
            r = rng.uniform(0.6, 1.4, size=3)
            r = r / np.cbrt(r.prod())
            # voxelised ellipsoid keeps ~pi/6 of the box's cells
            n = max(3, int(round((target / (math.pi / 6 * r.prod())) ** (1 / 3))) - 1)
            dims = tuple(max(2, int(round(n * ri))) for ri in r)
        else:
            n = max(2, int(round(target ** (1 / 3))) - 1)
            dims = (n, n, n)
        specs.append((ellipsoid, dims))
        pitch = max(pitch, max(dims) * cell)
    pitch = pitch * 1.5 + 0.1
    keep_set = None if only is None else set(int(k) for k in only)
    body_ids = []
    all_counts = []
    for b, (ellipsoid, dims) in enumerate(specs):
        if ellipsoid:
            half = np.array(dims) * cell / 2

            def keep(c, half=half):
                q = (c - half) / half
                return (q * q).sum(1) <= 1.0
            v, t = tet_lattice(dims, cell, keep)
        else:
            v, t = tet_lattice(dims, cell)
        v = v - v.mean(0)
        v = v @ _rand_rot(rng).T
        gx, gz = (b % nside - (nside - 1) / 2) * pitch, (b // nside - (nside - 1) / 2) * pitch
        v = v + np.array([gx, -v[:, 1].min() + rng.uniform(0.006, 0.02), gz])
        E = float(10 ** rng.uniform(4, 6))
        mu = float(rng.uniform(0.2, 0.6))
        all_counts.append((len(v), len(t)))
        if keep_set is not None and b not in keep_set:
            continue
        bodies.append(_Body(v, np.zeros((0, 3), np.int32), t, 1000.0, E / (1 + 0.4), mu=mu))
        body_ids.append(b)
    gv, gf = ground_quad(nside * pitch / 2 + 1.0, 0.0)
    bodies.append(_Body(gv, gf, np.zeros((0, 4), np.int32), 1e12, 0.0, static=True))
    params = SolverParams(dt=1.0 / 100, g=9.8, mu=0.4, thickness=0.6 * cell, admm_max_iter=30,
                          dcd_interval=5, gs_max_iter=10, jacobi_iter=20, max_contacts=2_000_000)
    return assemble(f"batch{n_bodies}", bodies, [], params,
                    meta={"config": "batched soft bodies", "seed": seed, "bodies": n_bodies,
                          "only": None if only is None else sorted(keep_set), "body_ids": body_ids,
                          "body_verts": [len(b.verts) for b in bodies if not b.static],
                          "all_body_counts": all_counts})


CONFIGS = {
    "cloth": cloth_on_box,
    "cube": cube_on_ground,
    "sheets": sheets_on_sphere,
    "batch": batch_bodies,
}
