"""The C++ IADMMBackend adapter (include/admm_b200_backend.hpp).

CPU: it compiles against the reference-type mirror and links the library.
GPU: driven with the reference's call order, it reproduces the C-ABI path bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def _build(tmp_path):
    exe = str(tmp_path / "drive_backend")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(CPP, "mirror"), "-I", os.path.join(ROOT, "include"),
           os.path.join(CPP, "drive_backend.cpp"), "-o", exe, "-L", os.path.join(ROOT, "parallel_admm_b200"),
           "-ladmm_b200", "-Wl,-rpath," + os.path.join(ROOT, "parallel_admm_b200")]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def _write_scene(sc, path, nsteps):
    p = sc.params
    ints = np.array([sc.n_vert, sc.n_dyn, sc.n_rows, sc.tri_start_row, sc.tet_start_row, sc.bend_start_row,
                     sc.pin_start_row, p.admm_max_iter, p.dcd_interval, p.gs_max_iter, p.jacobi_iter,
                     p.max_contacts, int(p.enable_contact), nsteps, p.ell_lanes], np.int32)
    flts = np.array([p.dt, p.g, p.mu, p.kappa, p.beta, p.thickness], np.float32)
    arrays = [ints, flts, sc.verts.astype(np.float32), sc.mass.astype(np.float32),
              sc.tri_inds.astype(np.int32), sc.tri_binv.astype(np.float32), sc.tri_w.astype(np.float32),
              sc.tet_inds.astype(np.int32), sc.tet_binv.astype(np.float32), sc.tet_w.astype(np.float32),
              sc.bend_offsets.astype(np.int32), sc.bend_inds.astype(np.int32), sc.bend_coeffs.astype(np.float32),
              sc.bend_w.astype(np.float32), sc.pin_inds.astype(np.int32), sc.pin_pos.astype(np.float32),
              sc.pin_w.astype(np.float32), sc.surf_tris.astype(np.int32), sc.surf_edges.astype(np.int32),
              sc.surf_verts.astype(np.int32), sc.contact_w.astype(np.float32)]
    with open(path, "wb") as f:
        for a in arrays:
            a = np.ascontiguousarray(a)
            f.write(np.int64(a.size).tobytes())
            f.write(a.tobytes())


def test_adapter_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cloth", "cube"])
def test_adapter_matches_c_abi_path(tmp_path, name):
    sc = scene.cloth_on_box(16) if name == "cloth" else scene.cube_on_ground(6, drop=0.02)
    sc.params.ell_lanes = 4  # both processes sum in the same order (no per-process autotuning)
    exe = _build(tmp_path)
    nsteps = 4
    _write_scene(sc, tmp_path / "scene.bin", nsteps)
    out = tmp_path / "x.bin"
    r = subprocess.run([exe, str(tmp_path / "scene.bin"), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    x_cpp = np.fromfile(out, np.float32).reshape(sc.n_vert, 3)
    h = B.Handle(sc)
    h.step(nsteps)
    x_py, _ = h.get_state()
    assert np.array_equal(x_cpp, x_py)


@pytest.mark.gpu
def test_collision_detector_view_matches_the_c_abi(tmp_path):
    """ADU::BVHB200, the ICollisionDetector view of the backend's handle, through the
    reference's contract: the contact count, max_slots() rows of points and normals (zero past
    the count) and the peak equal the C ABI's contacts on the same positions."""
    sc = scene.batch_bodies(4, seed=1, vmin=300, vmax=900)  # bodies within the contact band of the ground
    sc.params.ell_lanes = 4
    exe = _build(tmp_path)
    nsteps = 1
    _write_scene(sc, tmp_path / "scene.bin", nsteps)
    r = subprocess.run([exe, str(tmp_path / "scene.bin"), str(tmp_path / "x.bin"), str(tmp_path / "c.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = open(tmp_path / "c.bin", "rb").read()
    count, slots, peak = np.frombuffer(raw[:24], np.int64)
    body = np.frombuffer(raw[24:], np.float32).reshape(2, slots, 3)
    x_cpp = np.fromfile(tmp_path / "x.bin", np.float32).reshape(sc.n_vert, 3)
    h = B.Handle(sc)
    n = h.detect(x_cpp, allow=(B.ERR_CONTACT_OVERFLOW,))
    c = h.contacts()
    assert count == n > 0 and slots == h.max_slots() and peak >= count
    np.testing.assert_array_equal(body[0, :n], c["point"])
    np.testing.assert_array_equal(body[1, :n], c["normal"])
    assert not body[:, n:].any()
