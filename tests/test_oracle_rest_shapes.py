"""The oracle computes the rest-shape records (Binv, area or volume, hence w = sqrt(k A)) and
the lumped masses itself from the mesh (triangle_constraint.h:41-58,
tetrahedral_constraint.h:41-51, mesh_container.h:452-472) and they agree with the records
of the scene builder, which feed both the oracle and the GPU (no GPU)."""
import ctypes

import numpy as np

from oracle import oracle as O
from parallel_admm_b200 import scene

_d = ctypes.POINTER(ctypes.c_double)
_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int32)


def _lib():
    L = O.lib()
    L.orc_tri_rest.argtypes = [_f, _i, ctypes.c_int, _d, _d]
    L.orc_tet_rest.argtypes = [_f, _i, ctypes.c_int, _d, _d]
    L.orc_lumped_mass.argtypes = [ctypes.c_int, _f, _i, ctypes.c_int, _d, _i, ctypes.c_int, _d, _d]
    return L


def _p(a, t):
    return a.ctypes.data_as(t)


def test_triangle_rest_shapes_and_weights():
    sc = scene.cloth_on_box(16, seed=3)
    L = _lib()
    v = np.ascontiguousarray(sc.verts, np.float32)
    t = np.ascontiguousarray(sc.tri_inds, np.int32)
    binv = np.zeros((len(t), 4))
    area = np.zeros(len(t))
    L.orc_tri_rest(_p(v, _f), _p(t, _i), len(t), _p(binv, _d), _p(area, _d))
    np.testing.assert_allclose(sc.tri_binv, binv, rtol=2e-5, atol=2e-5 * np.abs(binv).max())
    k = 1e5 / 1.3  # E / (1 + nu) of the cloth
    np.testing.assert_allclose(sc.tri_w, np.sqrt(k * area), rtol=1e-5)


def test_tet_rest_shapes_weights_and_masses():
    for sc, dens in ((scene.cube_on_ground(6, seed=1), 1000.0), (scene.batch_bodies(3, seed=2, vmin=300, vmax=800), 1000.0)):
        L = _lib()
        v = np.ascontiguousarray(sc.verts, np.float32)
        t = np.ascontiguousarray(sc.tet_inds, np.int32)
        binv = np.zeros((len(t), 9))
        vol = np.zeros(len(t))
        L.orc_tet_rest(_p(v, _f), _p(t, _i), len(t), _p(binv, _d), _p(vol, _d))
        np.testing.assert_allclose(sc.tet_binv, binv, rtol=2e-5, atol=2e-5 * np.abs(binv).max())
        # w^2 / volume is the stiffness k of the tet's body
        k = sc.tet_w.astype(np.float64) ** 2 / vol
        assert np.all(k > 1e4 / 1.4 * 0.999) and np.all(k < 1e6 / 1.4 * 1.001)
        mass = np.zeros(sc.n_vert)
        td = np.full(len(t), dens)
        L.orc_lumped_mass(sc.n_vert, _p(v, _f), None, 0, None, _p(t, _i), len(t), _p(td, _d), _p(mass, _d))
        np.testing.assert_allclose(sc.mass[:sc.n_dyn], mass[:sc.n_dyn], rtol=1e-5)
