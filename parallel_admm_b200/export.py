"""Headless runs of a scene file: frame export, step metrics and run-to-run comparison.

What the reference's application does around the solver, for this backend:

* :func:`run_scene` -- the headless main loop (``src/main.cpp:29-93``): frames 0..end_frame,
  ``sub_step`` solver steps per frame, the frame exported after its steps when ``export_obj``
  is set, ``step_metrics.csv`` written into ``out_file`` at the end (``main.cpp:161-166``)
* :func:`export_frame` -- ``src/mesh/export_frame.h:14-54``: one OBJ (or binary PLY with
  ``out_bin``) of all vertices and surface triangles per frame, or one file per mesh with
  ``separate_out``.  The reference builds the names ``<scene>\\_<frame>`` and
  ``<scene>\\_<mesh>\\_<frame>`` on Windows, where the backslash is a folder separator; the
  files land at ``<out>/<scene>/_<frame:05>.obj`` and ``<out>/<scene>/_<mesh:03>/_<frame:05>.obj``,
  which is where the reference's comparison tool looks for them
* :func:`write_step_metrics_csv` -- ``src/solver/solver.h:27-45`` (header
  ``frame,step_ms,n_contacts``; frame = the solver's step count after the step, step_ms its
  host wall time, n_contacts the contacts of its last detection)
* :func:`compare_runs` -- the comparison half of ``tools/compare_solvers.py:125-198``: per
  common frame the mean and max vertex distance between two runs, with both runs' contacts
  and step times, written as ``frames.csv``
"""
from __future__ import annotations

import csv
import dataclasses
import glob
import os
import re
import struct
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


@dataclasses.dataclass
class StepMetrics:
    frame: int
    step_ms: float
    n_contacts: int


def write_obj(path: str, V: np.ndarray, F: np.ndarray) -> None:
    """Vertices and 1-based triangles; 9 significant digits keep float32 positions exact."""
    V = np.asarray(V, np.float64).reshape(-1, 3)
    F = np.asarray(F, np.int64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("".join(f"v {a:.9g} {b:.9g} {c:.9g}\n" for a, b, c in V))
        f.write("".join(f"f {a + 1} {b + 1} {c + 1}\n" for a, b, c in F))


def write_ply(path: str, V: np.ndarray, F: np.ndarray) -> None:
    """Binary little-endian PLY: float32 vertices, uchar-counted int32 triangle lists."""
    V = np.ascontiguousarray(V, "<f4").reshape(-1, 3)
    F = np.asarray(F, "<i4").reshape(-1, 3)
    hdr = ("ply\nformat binary_little_endian 1.0\n"
           f"element vertex {len(V)}\nproperty float x\nproperty float y\nproperty float z\n"
           f"element face {len(F)}\nproperty list uchar int vertex_indices\nend_header\n")
    faces = np.zeros(len(F), dtype=[("n", "u1"), ("v", "<i4", 3)])
    faces["n"] = 3
    faces["v"] = F
    with open(path, "wb") as f:
        f.write(hdr.encode())
        f.write(V.tobytes())
        f.write(faces.tobytes())


def read_obj_vertices(path: str) -> np.ndarray:
    out = []
    with open(path) as f:
        for line in f:
            if line.startswith("v "):
                p = line.split()
                out.append((float(p[1]), float(p[2]), float(p[3])))
    return np.asarray(out, np.float64).reshape(-1, 3)


def export_frame(out_path: str, scene_name: str, step_idx: int, verts: np.ndarray, surface_tris: np.ndarray,
                 meshes: Optional[Sequence[dict]] = None, use_bin: bool = False, separate_out: bool = False) -> List[str]:
    """Write one frame; returns the files written.  `meshes` (load order): dicts with the
    vertex range [start, end) and the mesh's triangle-strain or static faces (global indices;
    tet meshes have none), as ``MeshData::getFaceInds`` gives them."""
    ext = ".ply" if use_bin else ".obj"
    write = write_ply if use_bin else write_obj
    base = os.path.join(out_path, scene_name)
    written = []
    if separate_out and meshes:
        for mesh_id, m in enumerate(meshes):
            d = os.path.join(base, f"_{mesh_id:03d}")
            os.makedirs(d, exist_ok=True)
            p = os.path.join(d, f"_{step_idx:05d}{ext}")
            write(p, verts[m["start"]:m["end"]], np.asarray(m["faces"], np.int64) - m["start"])
            written.append(p)
    else:
        os.makedirs(base, exist_ok=True)
        p = os.path.join(base, f"_{step_idx:05d}{ext}")
        write(p, verts, surface_tris)
        written.append(p)
    return written


def write_step_metrics_csv(path: str, metrics: Sequence[StepMetrics]) -> None:
    with open(path, "w", newline="") as f:
        f.write("frame,step_ms,n_contacts\n")
        for m in metrics:
            f.write(f"{m.frame},{m.step_ms:g},{m.n_contacts}\n")


def read_step_metrics_csv(path: str) -> Dict[int, Tuple[float, int]]:
    out = {}
    if not os.path.exists(path):
        return out
    with open(path, newline="") as f:
        for row in csv.DictReader(f):
            out[int(row["frame"])] = (float(row["step_ms"]), int(row["n_contacts"]))
    return out


class Runner:
    """The headless application loop over a stepping engine with ``step(1) -> stats`` and
    ``get_state() -> (x, v)`` (the backend's Handle; tests also drive other engines through
    it)."""

    def __init__(self, engine, cfg, scene, out_path: Optional[str] = None):
        self.engine = engine
        self.cfg = cfg
        self.scene = scene
        self.out_path = out_path if out_path is not None else cfg.out_file
        self.metrics: List[StepMetrics] = []
        self.step_cnt = 0
        self.save_res = True
        try:
            os.makedirs(self.out_path, exist_ok=True)
        except OSError:
            self.save_res = False

    def step_frame(self, frame: int) -> None:
        for _ in range(self.cfg.sub_step):
            t0 = time.perf_counter()
            st = self.engine.step(1)
            ms = (time.perf_counter() - t0) * 1e3
            self.step_cnt += 1
            self.metrics.append(StepMetrics(self.step_cnt, ms, int(st.get("n_contacts", 0) if st else 0)))
        if self.cfg.export_obj and self.save_res:
            x, _ = self.engine.get_state()
            export_frame(self.out_path, self.cfg.scene_name, frame, x, self.scene.surf_tris,
                         self.scene.meta.get("meshes"), self.cfg.out_bin, self.cfg.separate_out)

    def run(self, frames: Optional[int] = None) -> List[StepMetrics]:
        end = self.cfg.end_frame if frames is None else frames
        for frame in range(end + 1):
            self.step_frame(frame)
        if self.save_res and self.metrics:
            write_step_metrics_csv(os.path.join(self.out_path, "step_metrics.csv"), self.metrics)
        return self.metrics


def run_scene(path: str, resource_root: Optional[str] = None, frames: Optional[int] = None,
              out_path: Optional[str] = None, export_obj: Optional[bool] = None):
    """Load a scene file and run it headless on this backend (the CUDA library must be built).
    Returns (metrics, handle)."""
    from . import backend as B
    from . import scene_config as C
    cfg = C.parse_config(path)
    if export_obj is not None:
        cfg.export_obj = export_obj
    sc = C.load_scene(path, resource_root, cfg)
    h = B.Handle(sc)
    tracks = C.scene_tracks(cfg, sc, resource_root, path)
    if tracks:
        C.attach_tracks(h, tracks)
    r = Runner(h, cfg, sc, out_path)
    return r.run(frames), h


def load_frames(run_dir: str, scene_name: str) -> Dict[int, np.ndarray]:
    """frame -> vertex positions of the single-file OBJ exports of a run."""
    out = {}
    for p in sorted(glob.glob(os.path.join(run_dir, scene_name, "_*.obj"))):
        m = re.search(r"_(\d{5})\.obj$", p)
        if m:
            out[int(m.group(1))] = read_obj_vertices(p)
    return out


def compare_runs(dir_a: str, dir_b: str, scene_name: str, out_csv: Optional[str] = None) -> List[tuple]:
    """Per common frame: (frame, mean vertex distance, max vertex distance, contacts a,
    contacts b, step ms a, step ms b).  Metrics are matched by frame number as the
    reference's tool does (solver step count against export frame index)."""
    fa, fb = load_frames(dir_a, scene_name), load_frames(dir_b, scene_name)
    ma = read_step_metrics_csv(os.path.join(dir_a, "step_metrics.csv"))
    mb = read_step_metrics_csv(os.path.join(dir_b, "step_metrics.csv"))
    rows = []
    for f in sorted(set(fa) & set(fb)):
        a, b = fa[f], fb[f]
        n = min(len(a), len(b))
        d = np.linalg.norm(a[:n] - b[:n], axis=1) if n else np.zeros(1)
        xa, xb = ma.get(f, ("", "")), mb.get(f, ("", ""))
        rows.append((f, float(d.mean()), float(d.max()), xa[1], xb[1], xa[0], xb[0]))
    if out_csv:
        with open(out_csv, "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(["frame", "mean_vertex_diff", "max_vertex_diff", "contacts_a", "contacts_b",
                        "step_ms_a", "step_ms_b"])
            w.writerows(rows)
    return rows
