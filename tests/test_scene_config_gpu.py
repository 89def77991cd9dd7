"""A scene file through the CUDA backend: the TOML scene written by the CPU loader tests (a
rotated cloth, a centred tet cube and a static box), stepped on the GPU against the oracle."""
import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene_config as C
from test_scene_config import _write_scene

pytestmark = pytest.mark.gpu

TOL_LONG = 1e-3  # positions after 20 substeps, relative to the extent of the dynamic bodies


def test_scene_file_steps_match_oracle(tmp_path):
    from oracle import oracle as O
    path, *_ = _write_scene(str(tmp_path), 65)
    sc = C.load_scene(path)
    assert C.parse_config(path).selects_b200
    h = B.Handle(sc)
    o = O.Oracle(h.holder, double=True)
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    for k in range(20):
        h.step(1)
        o.step(1)
    xg, _ = h.get_state()
    err = np.abs(xg - o.read(B.BUF_X0)).max() / ext
    assert err <= TOL_LONG, err
    assert np.isfinite(xg).all()


class _OracleEngine:
    def __init__(self, o):
        self.o = o

    def step(self, k):
        return {"n_contacts": self.o.step(k)["n_contacts"]}

    def get_state(self):
        return self.o.read(B.BUF_X0), self.o.read(B.BUF_V)


def test_headless_run_against_oracle_run(tmp_path):
    """The headless application loop on the GPU and on the oracle: frame exports and step
    metrics of both runs, compared frame by frame as the reference's comparison tool does."""
    from oracle import oracle as O
    from parallel_admm_b200 import export as X
    path, *_ = _write_scene(str(tmp_path / "res"), 65)
    cfg = C.parse_config(path)
    cfg.export_obj = True
    cfg.separate_out = False
    sc = C.load_scene(path, cfg=cfg)
    h = B.Handle(sc)
    X.Runner(h, cfg, sc, str(tmp_path / "gpu")).run(frames=6)
    o = O.Oracle(B.DescHolder(sc), double=True)
    X.Runner(_OracleEngine(o), cfg, sc, str(tmp_path / "oracle")).run(frames=6)
    rows = X.compare_runs(str(tmp_path / "gpu"), str(tmp_path / "oracle"), cfg.scene_name)
    assert [r[0] for r in rows] == list(range(7))
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    assert max(r[2] for r in rows) <= TOL_LONG * ext
    assert all(r[3] == r[4] for r in rows)  # same contact counts per step


@pytest.mark.parametrize("kind", ["rigid", "points"])
def test_scripted_static_mesh_matches_oracle(tmp_path, kind):
    """A static box moved by a track: the device animator against the oracle driven by the
    restated animator (static rows of x0 and v written before every oracle substep)."""
    import os
    from oracle import oracle as O
    from test_scene_config import AnimatorRef, spin_track, wave_sequence
    root = str(tmp_path)
    os.makedirs(os.path.join(root, "track"))
    if kind == "rigid":
        pos, quat = spin_track(n_frames=30)
        np.savez(os.path.join(root, "track", "spin.npz"), pos=pos, quat=quat)
        anim = "track/spin.npz"
    else:
        from parallel_admm_b200 import scene as S
        bv, _ = S.box_mesh((-0.5, -0.2, -0.5), (0.5, 0.0, 0.5))
        np.savez(os.path.join(root, "track", "box_sequence.npz"), points=wave_sequence(bv, 12))
        anim = "track/box_sequence.npz"
    path, *_ = _write_scene(root, 65, animate=anim)
    cfg = C.parse_config(path)
    sc = C.load_scene(path, cfg=cfg)
    tracks = C.scene_tracks(cfg, sc)
    h = B.Handle(sc)
    C.attach_tracks(h, tracks)
    o = O.Oracle(B.DescHolder(sc), double=True)
    ref = AnimatorRef(tracks, sc.verts, sc.params.dt)
    x0, v = o.read(B.BUF_X0), o.read(B.BUF_V)
    ref.apply(x0, v, init=True)
    o.write(B.BUF_X0, x0)
    o.write(B.BUF_V, v)
    xg, vg = h.get_state()
    assert np.abs(xg - x0).max() <= 1e-6 * max(1.0, np.abs(x0).max())
    assert np.abs(vg[sc.n_dyn:]).max() == 0.0
    ext = np.ptp(sc.verts[:sc.n_dyn], axis=0).max()
    for k in range(16):  # past the end of the point track: held with zero velocity
        x0, v = o.read(B.BUF_X0), o.read(B.BUF_V)
        ref.apply(x0, v)
        o.write(B.BUF_X0, x0)
        o.write(B.BUF_V, v)
        o.step(1)
        h.step(1)
        xg, vg = h.get_state()
        xo = o.read(B.BUF_X0)
        assert np.abs(xg[sc.n_dyn:] - xo[sc.n_dyn:]).max() <= 1e-5 * max(1.0, np.abs(xo).max()), k
        assert np.abs(xg - xo).max() / ext <= TOL_LONG, k
    # velocities of the static rows as the animator set them for the last substep
    assert np.allclose(vg[sc.n_dyn:], v[sc.n_dyn:], rtol=1e-4, atol=1e-4)
    # reset places the meshes at their first frame again
    h.reset()
    x0r = sc.verts.astype(np.float64).copy()
    vr = np.zeros_like(x0r)
    AnimatorRef(tracks, sc.verts, sc.params.dt).apply(x0r, vr, init=True)
    xg, _ = h.get_state()
    assert np.abs(xg[sc.n_dyn:] - x0r[sc.n_dyn:]).max() <= 1e-6 * max(1.0, np.abs(x0r).max())
