"""GPU parity of the unsigned-distance and ray first-hit batches.

Against the oracle (the canonical traversal of detail/gwn_query_distance_impl.cuh:40-160 and
detail/gwn_query_ray_impl.cuh:376-560 restated in C with the same fixed pattern of fused
multiply-adds) on the tree the GPU built: distances, hit records and traversal statistics bit for bit, in input order and in
Hilbert order (distances under every walk of a Hilbert-ordered batch). Against smallgwn's known answers (tests/unit_gwn_query_distance_ray.cu, restated in
spatial_cases.py), against FP64 closest points, and against smallgwn's own kernels (oracle/_ref,
compiled with FMA contraction, so within a few ulps; equal-t hits may name either triangle there).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import api, meshes
from spatial_cases import CASES
from test_gpu_build import WORKLOADS, build, upload
from test_oracle_spatial import check_ray

pytestmark = pytest.mark.gpu

METHODS = {"lbvh": g.gwn_bvh_build_method.k_lbvh, "hploc": g.gwn_bvh_build_method.k_hploc}


def dev(cuda, *arrs):
    return [cuda.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in arrs]


def gpu_distance(cuda, bvh, q, band=float("inf"), **kw):
    d = dev(cuda, *q)
    out = cuda.empty_like(d[0])
    st = g.gwn_compute_unsigned_distance_batch(bvh, *d, out, culling_band=band, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out.cpu().numpy()


def gpu_ray(cuda, bvh, o, d, t_min=0.0, t_max=float("inf"), offset_words=0, **kw):
    r = dev(cuda, *o, *d)
    n = r[0].numel()
    buf = cuda.full((n * api.RAY_HIT_WORDS + offset_words,), -7, dtype=cuda.int32, device="cuda")
    out = buf[offset_words:]
    st = g.gwn_compute_ray_first_hit_batch(bvh, *r, out, t_min=t_min, t_max=t_max, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return api.ray_hit_records(out)


def host_tree(bvh):
    h = api.bvh_host_arrays(bvh)
    return h["nodes"], h["triangles"], h["primitive_indices"], h["root_reference"]


def as_oracle_hits(recs):
    out = np.zeros(recs.size, oracle.HIT_DTYPE)
    out.view(np.uint8)[:] = np.ascontiguousarray(recs).view(np.uint8)
    return out


def query_mix(mesh, n, seed):
    rng = np.random.default_rng(seed)
    lo = np.array([mesh[k].min() for k in "xyz"], np.float32)
    hi = np.array([mesh[k].max() for k in "xyz"], np.float32)
    c, e = (lo + hi) / 2, (hi - lo) / 2 * 1.3 + 1e-3
    box = (c[:, None] + e[:, None] * rng.uniform(-1, 1, (3, n // 2))).astype(np.float32)
    # points near the surface: vertices pushed by a small random offset
    vid = rng.integers(0, mesh["x"].size, n - n // 2)
    near = np.stack([mesh[k][vid] for k in "xyz"]) + rng.normal(0, 1e-3, (3, n - n // 2))
    return np.concatenate([box, near.astype(np.float32)], axis=1)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_known_answers(cuda, case):
    name, make, method, cap, rays, dists = case
    geo = upload(make())
    bvh = build(geo, METHODS[method])
    cfg = g.gwn_query_batch_config(block_size=256, stack_capacity=cap)
    for args, expect in rays:
        ox, oy, oz, dx, dy, dz, t0, t1 = args
        h = gpu_ray(cuda, bvh, [[ox], [oy], [oz]], [[dx], [dy], [dz]], t0, t1, config=cfg)[0]
        h = as_oracle_hits(np.array([h]))[0]
        check_ray(h, expect)
    for (qx, qy, qz, band), expect in dists:
        d = gpu_distance(cuda, bvh, [[qx], [qy], [qz]], band, config=cfg)[0]
        assert abs(float(d) - expect) <= 1e-6 * max(1.0, expect), (name, qx, qy, qz, band, d)


@pytest.mark.parametrize("method", list(METHODS))
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_distance_bit_exact_with_oracle(cuda, name, method):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    bvh = build(geo, METHODS[method])
    nodes, tris, prims, root = host_tree(bvh)
    q = query_mix(mesh, 4000, seed=11)
    for band in (float("inf"), 0.02, -1.0):
        ref, st = oracle.unsigned_distance(nodes, tris, root, *q, culling_band=band, stats=True)
        np.testing.assert_array_equal(gpu_distance(cuda, bvh, q, band), ref)
        # Hilbert order: the warp-cooperative walk, the per-thread walk and the timed choice
        for walk in ("warp", "thread", "timed", "timed", "timed"):
            np.testing.assert_array_equal(gpu_distance(cuda, bvh, q, band, sort_queries=True, traversal=walk), ref)
    # traversal statistics (unbounded band) equal the oracle's counts
    ref, st = oracle.unsigned_distance(nodes, tris, root, *q, stats=True)
    dq = dev(cuda, *q)
    sn = cuda.empty(q.shape[1], dtype=cuda.int32, device="cuda")
    stri = cuda.empty_like(sn)
    assert api.spatial_traversal_stats(bvh, *dq, sn, stri).is_ok()
    np.testing.assert_array_equal(sn.cpu().numpy().view(np.uint32), st[:, 0])
    np.testing.assert_array_equal(stri.cpu().numpy().view(np.uint32), st[:, 1])


@pytest.mark.parametrize("method", list(METHODS))
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_ray_bit_exact_with_oracle(cuda, name, method):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    bvh = build(geo, METHODS[method])
    nodes, tris, prims, root = host_tree(bvh)
    o = query_mix(mesh, 4000, seed=12)
    d = np.random.default_rng(13).normal(size=o.shape).astype(np.float32)
    d[:, :50] = 0.0  # zero directions miss
    d[0, 50:100] = 0.0  # axis-parallel slabs
    for t_min, t_max in ((0.0, float("inf")), (-0.5, 0.25)):
        ref, st = oracle.ray_first_hit(nodes, tris, prims, root, *o, *d, t_min=t_min, t_max=t_max, stats=True)
        got = as_oracle_hits(gpu_ray(cuda, bvh, o, d, t_min, t_max))
        assert (ref["status"] == 1).any()
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_array_equal(as_oracle_hits(gpu_ray(cuda, bvh, o, d, t_min, t_max, sort_queries=True)), ref)
    # 4-byte-aligned (not 16-byte-aligned) output storage takes the scalar store path
    np.testing.assert_array_equal(as_oracle_hits(gpu_ray(cuda, bvh, o, d, offset_words=1)),
                                  oracle.ray_first_hit(nodes, tris, prims, root, *o, *d))
    ref, st = oracle.ray_first_hit(nodes, tris, prims, root, *o, *d, stats=True)
    dq = dev(cuda, *o, *d)
    sn = cuda.empty(o.shape[1], dtype=cuda.int32, device="cuda")
    stri = cuda.empty_like(sn)
    assert api.spatial_traversal_stats(bvh, *dq[:3], sn, stri, *dq[3:]).is_ok()
    np.testing.assert_array_equal(sn.cpu().numpy().view(np.uint32), st[:, 0])
    np.testing.assert_array_equal(stri.cpu().numpy().view(np.uint32), st[:, 1])


def test_distance_matches_fp64_closest_point(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(64, 32, seed=9))
    bvh = build(upload(mesh), METHODS["hploc"])
    q = query_mix(mesh, 3000, seed=14)
    d = gpu_distance(cuda, bvh, q)
    ref = oracle.mesh_distance(mesh, *q)
    assert np.abs(d - ref).max() < 2e-6


def test_ray_hits_lie_on_the_mesh(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(64, 32, seed=9))
    bvh = build(upload(mesh), METHODS["hploc"])
    rng = np.random.default_rng(15)
    o = rng.uniform(-0.3, 0.3, (3, 3000)).astype(np.float32)  # inside the closed surface: every ray hits
    d = rng.normal(size=o.shape).astype(np.float32)
    h = gpu_ray(cuda, bvh, o, d)
    assert (h["status"] == 1).all()
    p = o.astype(np.float64) + h["t"].astype(np.float64) * d.astype(np.float64)
    assert oracle.mesh_distance(mesh, *p).max() < 1e-5
    # the reported triangle is the one hit: the hit point lies in its plane
    v0, v1, v2 = (np.stack([mesh[k][mesh[i][h["primitive_id"]]] for k in "xyz"], 1).astype(np.float64)
                  for i in ("i0", "i1", "i2"))
    n = np.cross(v1 - v0, v2 - v0)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    assert np.abs(np.einsum("ij,ij->i", p.T - v0, n)).max() < 1e-5


def test_large_mesh_properties(cuda):
    """1,046,528-triangle displaced sphere, 1M queries: bit-exact with the oracle on a subset,
    Hilbert order identical to input order, distances never negative."""
    mesh = meshes.sphere_mesh()
    bvh = build(upload(mesh), METHODS["hploc"])
    q = np.stack(meshes.mixed_queries(mesh, 1_000_000, seed=2))
    d0 = gpu_distance(cuda, bvh, q)
    d1 = gpu_distance(cuda, bvh, q, sort_queries=True)
    np.testing.assert_array_equal(d0, d1)
    assert (d0 >= 0).all() and np.isfinite(d0).all()
    nodes, tris, prims, root = host_tree(bvh)
    sub = q[:, ::500]
    np.testing.assert_array_equal(d0[::500], oracle.unsigned_distance(nodes, tris, root, *sub))
    dirs = np.random.default_rng(16).normal(size=q.shape).astype(np.float32)
    h0 = gpu_ray(cuda, bvh, q, dirs)
    h1 = gpu_ray(cuda, bvh, q, dirs, sort_queries=True)
    np.testing.assert_array_equal(h0, h1)
    np.testing.assert_array_equal(as_oracle_hits(h0[::500]),
                                  oracle.ray_first_hit(nodes, tris, prims, root, *sub, *dirs[:, ::500]))


needs_ref = pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's kernels (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40"])
def test_against_smallgwn_kernels(cuda, name):
    mesh = WORKLOADS[name]()
    bvh = build(upload(mesh), METHODS["hploc"])
    ref = oracle.Reference(mesh)
    ref.build(method=0, radius=8)
    q = query_mix(mesh, 4000, seed=17)
    ours = gpu_distance(cuda, bvh, q)
    theirs = ref.distance(*q)
    assert np.abs(ours - theirs).max() <= 1e-6 * max(1.0, float(np.abs(theirs).max()))
    d = np.random.default_rng(18).normal(size=q.shape).astype(np.float32)
    h = gpu_ray(cuda, bvh, q, d)
    r = ref.ray(*q, *d)
    same_status = h["status"] == r["status"]
    assert same_status.mean() >= 0.999
    both = same_status & (h["status"] == 1)
    assert np.abs(h["t"][both] - r["t"][both]).max() <= 1e-5 * max(1.0, float(np.abs(r["t"][both]).max()))
    # a different primitive id only where another triangle is hit at (nearly) the same t
    assert (h["primitive_id"][both] == r["primitive_id"][both]).mean() >= 0.999
    ref.close()
