"""Scene set-up: sizes of the synthetic configurations and the constraint records."""
import numpy as np
import pytest

from parallel_admm_b200 import scene


def test_cloth_config_sizes():
    sc = scene.cloth_on_box(32)
    s = sc.summary()
    assert s["n_dyn"] == 1024 and s["n_vert"] == 1032          # + the 8 box vertices
    assert s["n_tri"] == 1922                                     # 31*31*2
    assert s["n_bend"] == 1022                                    # ring >= 3 (two corners have 2)
    assert s["n_pin"] == 2 and s["n_rows"] == 2 * 1922 + 1022 + 2
    assert abs(sc.mass[:sc.n_dyn].sum() - 0.1) < 1e-6            # 1 m^2 at 0.1 kg/m^2


def test_cube_config_sizes():
    sc = scene.cube_on_ground(20)
    s = sc.summary()
    assert s["n_dyn"] == 9261 and s["n_tet"] == 40000 and s["n_rows"] == 120000
    assert s["n_surf_tri"] == 6 * 20 * 20 * 2 + 2                 # + ground quad
    assert abs(sc.mass[:sc.n_dyn].sum() - 125.0) < 1e-3          # 0.5^3 m^3 at 1000 kg/m^3
    assert np.all(sc.tet_w > 0)


def test_rest_deformation_gradient_is_identity():
    """D x_rest = F = I for every tet and the 2x2 identity frame for every triangle."""
    for sc in (scene.cube_on_ground(4), scene.cloth_on_box(8)):
        x = sc.verts.astype(np.float64)
        for c in range(len(sc.tet_inds)):
            i = sc.tet_inds[c]
            E = np.stack([x[i[1]] - x[i[0]], x[i[2]] - x[i[0]], x[i[3]] - x[i[0]]], 1)
            F = E @ sc.tet_binv[c].reshape(3, 3)
            assert np.allclose(F, np.eye(3), atol=1e-5)
        for c in range(len(sc.tri_inds)):
            i = sc.tri_inds[c]
            E = np.stack([x[i[1]] - x[i[0]], x[i[2]] - x[i[0]]], 1)
            F = E @ sc.tri_binv[c].reshape(2, 2)
            assert np.allclose(F.T @ F, np.eye(2), atol=1e-5)


def test_bending_rows_annihilate_constants():
    sc = scene.cloth_on_box(8)
    for c in range(len(sc.bend_w)):
        a, b = sc.bend_offsets[c], sc.bend_offsets[c + 1]
        assert abs(sc.bend_coeffs[a:b].sum()) < 1e-3 * np.abs(sc.bend_coeffs[a:b]).max()


def test_surface_sets_and_contact_weights():
    sc = scene.cube_on_ground(6)
    assert set(np.unique(sc.surf_tris)) == set(sc.surf_verts.tolist())
    e = {tuple(sorted(x)) for x in sc.surf_edges.tolist()}
    assert len(e) == len(sc.surf_edges)
    assert np.all(sc.contact_w[sc.n_dyn:] == np.float32(1e12))
    dt = sc.params.dt
    assert np.allclose(sc.contact_w[:sc.n_dyn], sc.mass[:sc.n_dyn] / dt / dt * sc.params.w_scale, rtol=1e-6)


def test_tet_cube_is_conforming():
    """Every interior face is shared by exactly two tets (boundary_facets count)."""
    n = 5
    v, t = scene.tet_cube(n, 1.0)
    f = scene.boundary_facets(t)
    assert len(f) == 6 * n * n * 2
    vol = 0.0
    for tt in t:
        E = np.stack([v[tt[1]] - v[tt[0]], v[tt[2]] - v[tt[0]], v[tt[3]] - v[tt[0]]], 1)
        d = np.linalg.det(E)
        assert d > 0
        vol += d / 6
    assert abs(vol - 1.0) < 1e-9
