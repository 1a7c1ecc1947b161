"""The oracle's distance and ray queries (CPU): smallgwn's known answers
(tests/unit_gwn_query_distance_ray.cu, restated in spatial_cases.py), overflow behaviour, and the
canonical traversal against brute force over every triangle on seeded meshes."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from smallgwn_b200 import meshes
from spatial_cases import CASES, INVALID, layered


def check_ray(hit, expect):
    status, t, prim, t_tol, uv = expect
    assert hit["status"] == status
    assert hit["primitive_id"] == prim
    if t_tol == 0.0:
        assert abs(float(hit["t"]) - t) <= 4 * np.spacing(np.float32(abs(t) or 1.0))
    else:
        assert abs(float(hit["t"]) - t) <= t_tol
    if uv is not None:
        assert abs(float(hit["u"]) - uv[0]) <= uv[2] and abs(float(hit["v"]) - uv[1]) <= uv[2]
    if status == 0:
        assert hit["u"] == 0 and hit["v"] == 0 and hit["nx"] == 0 and hit["ny"] == 0 and hit["nz"] == 0
    else:
        assert np.isfinite([hit["u"], hit["v"]]).all()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_known_answers(case):
    name, make, method, cap, rays, dists = case
    mesh = make()
    b = oracle.build_bvh(mesh, method)
    if cap < 64:
        assert b["internal_stack_bound"] <= cap
    for args, expect in rays:
        ox, oy, oz, dx, dy, dz, t0, t1 = args
        h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], [ox], [oy], [oz],
                                 [dx], [dy], [dz], t_min=t0, t_max=t1, stack_capacity=cap)[0]
        check_ray(h, expect)
    for (qx, qy, qz, band), expect in dists:
        d = oracle.unsigned_distance(b["nodes"], b["triangles"], b["root_reference"], [qx], [qy], [qz],
                                     culling_band=band, stack_capacity=cap)[0]
        assert abs(float(d) - expect) <= 1e-6 * max(1.0, expect), (qx, qy, qz, band, d)


def test_leaf_root_hit_record():
    """gwn_query_distance_ray.cu:223-249: t = 1, weights 1/4, normal (0, 0, 1) for the unit triangle."""
    b = oracle.build_bvh(layered(1), "lbvh")
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], [0.25], [0.25], [1],
                             [0], [0], [-1])[0]
    assert (h["t"], h["nx"], h["ny"], h["nz"]) == (1.0, 0.0, 0.0, 1.0)


def test_subnormal_weights_keep_positive_normal():
    from spatial_cases import tiny_triangle
    b = oracle.build_bvh(tiny_triangle(1e-20), "lbvh")
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], [0.25e-20],
                             [0.25e-20], [1], [0], [0], [-1], t_max=2)[0]
    assert h["status"] == 1 and h["nz"] > 0


def test_overflow_reports_nan_and_status():
    """gwn_query_distance_ray.cu:690-705: capacity 1 below the bound of 32 layers."""
    b = oracle.build_bvh(layered(32), "hploc")
    assert b["internal_stack_bound"] > 1
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], [0.25], [0.25], [40],
                             [0], [0], [-1], t_max=100, stack_capacity=1)[0]
    assert h["status"] == 2
    d = oracle.unsigned_distance(b["nodes"], b["triangles"], b["root_reference"], [0.25], [0.25], [15.5],
                                 stack_capacity=1)[0]
    assert np.isnan(d)


@pytest.mark.parametrize("method", ["lbvh", "hploc"])
def test_traversal_equals_brute_force(method):
    """The pruned near-first traversal returns the minimum over every triangle (distance) and the
    nearest hit with the lower-id tie rule (ray), bit for bit."""
    mesh = meshes.to_soa(*meshes.uv_sphere(48, 24, seed=2))
    b = oracle.build_bvh(mesh, method)
    rng = np.random.default_rng(7)
    q = rng.uniform(-1.6, 1.6, (3, 3000)).astype(np.float32)
    d = oracle.unsigned_distance(b["nodes"], b["triangles"], b["root_reference"], *q)
    np.testing.assert_array_equal(d, oracle.distance_brute(b["triangles"], *q))
    for band in (0.05, 0.3):
        d = oracle.unsigned_distance(b["nodes"], b["triangles"], b["root_reference"], *q, culling_band=band)
        np.testing.assert_array_equal(d, oracle.distance_brute(b["triangles"], *q, culling_band=band))
    dirs = rng.normal(size=(3, 3000)).astype(np.float32)
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], *q, *dirs)
    hb = oracle.ray_brute(b["triangles"], b["sorted_ids"], *q, *dirs)
    assert (h["status"] == 1).mean() > 0.2
    np.testing.assert_array_equal(h, hb)
    # a bounded interval
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], *q, *dirs,
                             t_min=0.1, t_max=0.9)
    hb = oracle.ray_brute(b["triangles"], b["sorted_ids"], *q, *dirs, t_min=0.1, t_max=0.9)
    np.testing.assert_array_equal(h, hb)


def test_distance_matches_fp64_closest_point():
    mesh = meshes.to_soa(*meshes.uv_sphere(48, 24, seed=2))
    b = oracle.build_bvh(mesh, "hploc")
    rng = np.random.default_rng(8)
    q = rng.uniform(-1.6, 1.6, (3, 2000)).astype(np.float32)
    d = oracle.unsigned_distance(b["nodes"], b["triangles"], b["root_reference"], *q)
    ref = oracle.mesh_distance(mesh, *q)
    assert np.abs(d - ref).max() < 2e-6


def test_miss_record_layout():
    b = oracle.build_bvh(layered(3), "lbvh")
    h = oracle.ray_first_hit(b["nodes"], b["triangles"], b["sorted_ids"], b["root_reference"], [5], [5], [5], [1],
                             [0], [0])[0]
    assert h["status"] == 0 and h["t"] == -1.0 and h["primitive_id"] == INVALID
    assert bytes(h["pad"]) == b"\0\0\0"
