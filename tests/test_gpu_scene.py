"""Scene files on the GPU: saving geometry, BVH and moments and loading them back gives the same
arrays (a new revision), moments refit from the loaded BVH equal to the saved ones bit for bit, and
queries equal to those on the original objects; damaged files are refused."""
from __future__ import annotations

import numpy as np
import pytest

import smallgwn_b200 as g
from smallgwn_b200 import api, meshes
from test_gpu_build import build, upload

pytestmark = pytest.mark.gpu


def host_geometry(geo):
    v = geo.accessor()
    out = {}
    for k, n, dt in (("vertex_x", v.vertex_count, np.float32), ("vertex_y", v.vertex_count, np.float32),
                     ("vertex_z", v.vertex_count, np.float32), ("tri_i0", v.triangle_count, np.uint32),
                     ("tri_i1", v.triangle_count, np.uint32), ("tri_i2", v.triangle_count, np.uint32)):
        out[k] = np.frombuffer(api._copy_to_host(getattr(v, k), int(n) * 4), dt)
    return out


@pytest.mark.parametrize("name", ["soup", "sphere", "single"])
def test_save_load_round_trip(cuda, tmp_path, name):
    mesh = {"soup": lambda: meshes.soup_mesh(60, seed=4), "sphere": lambda: meshes.to_soa(*meshes.uv_sphere(64, 32, seed=9)),
            "single": lambda: {"x": np.array([0, 1, 0], np.float32), "y": np.array([0, 0, 1], np.float32),
                               "z": np.zeros(3, np.float32), "i0": np.array([0], np.uint32),
                               "i1": np.array([1], np.uint32), "i2": np.array([2], np.uint32)}}[name]()
    geo = upload(mesh)
    bvh = build(geo, g.gwn_bvh_build_method.k_hploc)
    moms = []
    for order in (0, 1, 2):
        m = g.gwn_bvh4_moment_object(order)
        assert g.gwn_refit_bvh_moment(order, bvh, m).is_ok()
        moms.append(m)
    path = tmp_path / "scene.gwnb"
    assert api.save_scene(path, geo, bvh, moms).is_ok()
    st, geo2, bvh2, moms2 = api.load_scene(path)
    assert st.is_ok(), st.message
    assert sorted(moms2) == [0, 1, 2]
    a, b = api.bvh_host_arrays(bvh), api.bvh_host_arrays(bvh2)
    for k in ("nodes", "primitive_indices", "triangles", "root_reference", "root_bounds", "internal_stack_bound",
              "packed_stack_bound"):
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]))
    assert b["revision"] != a["revision"] and b["revision"] != 0
    for k, v in host_geometry(geo).items():
        np.testing.assert_array_equal(v, host_geometry(geo2)[k])
    for order in (0, 1, 2):
        np.testing.assert_array_equal(api.moment_host_array(moms[order]), api.moment_host_array(moms2[order]))
        assert moms2[order].is_valid_for(bvh2)
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, 5000, seed=5)]
    o1, o2 = cuda.empty_like(q[0]), cuda.empty_like(q[0])
    for order in (1, 2):
        assert g.gwn_compute_winding_number_taylor_batch(order, bvh, moms[order], *q, o1, accuracy_scale=2.0).is_ok()
        assert g.gwn_compute_winding_number_taylor_batch(order, bvh2, moms2[order], *q, o2, accuracy_scale=2.0).is_ok()
        cuda.cuda.synchronize()
        assert cuda.equal(o1, o2)


def test_damaged_and_partial_files(cuda, tmp_path):
    mesh = meshes.soup_mesh(30, seed=5)
    geo = upload(mesh)
    bvh = build(geo)
    m1 = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, m1).is_ok()
    path = tmp_path / "s.gwnb"
    # geometry and BVH only
    assert api.save_scene(path, geo, bvh).is_ok()
    st, geo2, bvh2, moms = api.load_scene(path)
    assert st.is_ok() and moms == {} and bvh2.has_data()
    # one flipped byte in the body
    assert api.save_scene(path, geo, bvh, [m1]).is_ok()
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0x40
    path.write_bytes(bytes(raw))
    st, *_ = api.load_scene(path)
    assert st.error == api.gwn_error.invalid_argument and "checksum" in st.message
    # truncated
    assert api.save_scene(path, geo, bvh, [m1]).is_ok()
    path.write_bytes(path.read_bytes()[:-100])
    st, *_ = api.load_scene(path)
    assert st.error == api.gwn_error.invalid_argument
    # stale moments and duplicate orders are refused when saving
    stale = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, stale).is_ok()
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    assert api.save_scene(path, geo, bvh, [stale]).error == api.gwn_error.invalid_argument
    assert g.gwn_refit_bvh_moment(1, bvh, m1).is_ok()
    m1b = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, m1b).is_ok()
    assert "same order" in api.save_scene(path, geo, bvh, [m1, m1b]).message


@pytest.mark.parametrize("order", ["C", "F"])
def test_matrix_upload_equals_soa_upload(cuda, order):
    """N x 3 / M x 3 matrices (double positions, int32 or integer-valued float indices, either
    memory order) upload to the same device arrays as the SoA upload."""
    mesh = meshes.soup_mesh(40, seed=8)
    V = np.asarray(np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=1).astype(np.float64), order=order)
    F = np.stack([mesh["i0"], mesh["i1"], mesh["i2"]], axis=1)
    ref = host_geometry(upload(mesh))
    for Fm in (np.asarray(F.astype(np.int32), order=order), F.astype(np.float64)):
        geo = g.gwn_geometry_object()
        assert g.gwn_upload_geometry_from_eigen(geo, V, Fm).is_ok()
        got = host_geometry(geo)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k])
