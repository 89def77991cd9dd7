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
