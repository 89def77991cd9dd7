"""Headless runs: frame export, step metrics and run comparison (CPU, with a stand-in engine)."""
import os

import numpy as np
import pytest

from parallel_admm_b200 import export as X
from parallel_admm_b200 import scene_config as C
from test_scene_config import SCENE, _write_scene


class DriftEngine:
    """Moves every vertex by +1 in y per step and reports step-count contacts."""

    def __init__(self, sc):
        self.x = sc.verts.astype(np.float32).copy()
        self.n = 0

    def step(self, k):
        self.x[:, 1] += 1.0
        self.n += 1
        return {"n_contacts": self.n * 10}

    def get_state(self):
        return self.x.copy(), np.zeros_like(self.x)


def test_obj_and_ply_writers(tmp_path):
    V = np.array([[0.1, 2.5, -3.25], [1e-7, 3.4028235e38, 0.0], [1, 2, 3]], np.float32)
    F = np.array([[0, 1, 2]])
    p = str(tmp_path / "a.obj")
    X.write_obj(p, V, F)
    assert np.array_equal(X.read_obj_vertices(p).astype(np.float32), V)
    assert open(p).read().strip().endswith("f 1 2 3")
    q = str(tmp_path / "a.ply")
    X.write_ply(q, V, F)
    data = open(q, "rb").read()
    head, body = data.split(b"end_header\n")
    assert b"element vertex 3" in head and b"element face 1" in head
    assert len(body) == 3 * 12 + 1 + 12
    assert np.array_equal(np.frombuffer(body[:36], "<f4").reshape(3, 3), V)


def test_export_frame_names(tmp_path):
    V = np.zeros((6, 3), np.float32)
    F = np.array([[0, 1, 2], [3, 4, 5]])
    single = X.export_frame(str(tmp_path), "sc", 7, V, F)
    assert single == [os.path.join(str(tmp_path), "sc", "_00007.obj")]
    meshes = [{"start": 0, "end": 3, "faces": np.array([[0, 1, 2]])},
              {"start": 3, "end": 6, "faces": np.zeros((0, 3), np.int64)}]
    sep = X.export_frame(str(tmp_path), "sc", 12, V, F, meshes, use_bin=True, separate_out=True)
    assert sep == [os.path.join(str(tmp_path), "sc", "_000", "_00012.ply"),
                   os.path.join(str(tmp_path), "sc", "_001", "_00012.ply")]


def test_runner_frames_metrics_and_compare(tmp_path):
    path, *_ = _write_scene(str(tmp_path / "res"), 65)
    cfg = C.parse_config(path)
    cfg.export_obj = True
    cfg.separate_out = False
    sc = C.load_scene(path, cfg=cfg)
    outs = []
    for name in ("a", "b"):
        out = str(tmp_path / name)
        r = X.Runner(DriftEngine(sc), cfg, sc, out)
        m = r.run(frames=4)
        outs.append(out)
        # frames 0..4, sub_step = 2 solver steps each
        assert [x.frame for x in m] == list(range(1, 11))
        assert [x.n_contacts for x in m] == [10 * k for k in range(1, 11)]
        lines = open(os.path.join(out, "step_metrics.csv")).read().splitlines()
        assert lines[0] == "frame,step_ms,n_contacts" and len(lines) == 11
        files = sorted(os.listdir(os.path.join(out, "unit")))
        assert files == [f"_{k:05d}.obj" for k in range(5)]
        x4 = X.read_obj_vertices(os.path.join(out, "unit", "_00004.obj"))
        assert np.allclose(x4[:, 1], sc.verts[:, 1].astype(np.float64) + 10.0, atol=1e-4)
    rows = X.compare_runs(outs[0], outs[1], "unit", str(tmp_path / "frames.csv"))
    assert [r[0] for r in rows] == list(range(5))
    assert all(r[1] == 0.0 and r[2] == 0.0 for r in rows)
    assert open(str(tmp_path / "frames.csv")).readline().startswith("frame,mean_vertex_diff")


def test_runner_separate_meshes(tmp_path):
    path, *_ = _write_scene(str(tmp_path / "res"), 65)
    cfg = C.parse_config(path)
    cfg.export_obj = True
    cfg.separate_out = True
    sc = C.load_scene(path, cfg=cfg)
    out = str(tmp_path / "sep")
    X.Runner(DriftEngine(sc), cfg, sc, out).run(frames=1)
    # load order: cloth (tri), cube (tet, no faces), box (static)
    meshes = sc.meta["meshes"]
    assert [m["type"] for m in meshes] == ["tri", "tet", "static"]
    for k, m in enumerate(meshes):
        p = os.path.join(out, "unit", f"_{k:03d}", "_00001.obj")
        assert X.read_obj_vertices(p).shape == (m["end"] - m["start"], 3)
        nf = sum(1 for l in open(p) if l.startswith("f "))
        assert nf == len(m["faces"])
