"""The oracle against known answers and against smallgwn's own outputs (golden vectors).

CPU only. Known answers restate smallgwn's tests: closed meshes wind once inside and zero outside,
FP32 exact within 2e-6 of FP64 (tests/unit_gwn_query_winding.cu:193-215), full-descent Taylor equal
to exact within 1e-6 (tests/unit_gwn_bvh_moment.cu:42-114), far-field order progression
(tests/unit_gwn_query_winding.cu:146-189), exact stack bounds (tests/integration_gwn_builder.cu:35-119)
and H-PLOC on equal bounds (:301-343). Golden files come from tests/golden/make_golden.py.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import asym_octahedron, cube, equal_bounds, golden_files, octahedron, open_cube, single_triangle
from smallgwn_b200 import meshes

VALID = 1 << 47
OFF = (1 << 47) - 1


def host_stack_bounds(nodes: np.ndarray, root_ref: int, nprims: int) -> tuple[int, int, int]:
    """Recompute (internal, packed) stack bounds and count reachable nodes by depth-first walk."""
    nd = nodes.reshape(-1, 4)
    if (root_ref >> 48) != 0:
        return 0, 0, 0
    visited = np.zeros(nd.shape[0], bool)

    def walk(i):
        assert not visited[i], "node reachable twice"
        visited[i] = True
        valid = internal = 0
        mi = mp = 0
        for s in range(4):
            r = int(nd[i, s]["reference"])
            if not (r >> 47) & 1:
                continue
            valid += 1
            if (r >> 48) == 0:
                internal += 1
                ci, cp = walk(r & OFF)
                mi, mp = max(mi, ci), max(mp, cp)
            else:
                assert (r & OFF) + (r >> 48) <= nprims
        assert valid > 0
        return (internal - 1 + mi if internal else 0), valid - 1 + mp

    ib, pb = walk(root_ref & OFF)
    return ib, pb, int(visited.sum())


@pytest.mark.parametrize("mesh_fn", [octahedron, cube])
def test_closed_meshes_wind_once(mesh_fn):
    m = mesh_fn()
    qx = np.array([0.0, 0.1, 4.0, -3.0], np.float32)
    qy = np.array([0.0, -0.2, 3.0, 0.5], np.float32)
    qz = np.array([0.0, 0.05, 2.0, 0.0], np.float32)
    w = oracle.exact_winding(m, qx, qy, qz)
    np.testing.assert_allclose(w, [1, 1, 0, 0], atol=1e-6)


def test_open_cube_is_fractional():
    w = oracle.exact_winding(open_cube(), np.array([0.0], np.float32), np.array([0.0], np.float32),
                             np.array([0.0], np.float32))
    assert 0.7 < w[0] < 0.9  # five of six faces seen from the centre: 5/6


def test_exact_fp32_matches_fp64_asymmetric_octahedron():
    m = asym_octahedron()
    qx = np.array([0, 4, -2, 0.2, 1.5], np.float32)
    qy = np.array([0, 3, 1, -1.4, 0.2], np.float32)
    qz = np.array([0, 2, -3, 2.2, -1.8], np.float32)
    w32 = oracle.exact_winding(m, qx, qy, qz)
    w64 = oracle.exact_winding(m, qx, qy, qz, fp64=True)
    np.testing.assert_allclose(w32, w64, atol=2e-6)


def test_vertex_hit_contributes_zero():
    m = single_triangle()
    w = oracle.exact_winding(m, np.array([0.0], np.float32), np.array([0.0], np.float32), np.array([0.0], np.float32))
    assert w[0] == 0.0


def test_morton_corners_and_stability():
    # point triangles at opposite scene corners plus an exact duplicate of the first
    m = {"x": np.array([0, 1], np.float32), "y": np.array([0, 1], np.float32), "z": np.array([0, 1], np.float32),
         "i0": np.array([0, 1, 0], np.uint32), "i1": np.array([0, 1, 0], np.uint32), "i2": np.array([0, 1, 0], np.uint32)}
    for bits, full in ((32, (1 << 30) - 1), (64, (1 << 63) - 1)):
        aabbs, codes, scene = oracle.morton(m, bits)
        assert codes[0] == codes[2] == 0
        assert codes[1] == full
        sc, ids = oracle.sort_pairs(codes)
        assert list(ids) == [0, 2, 1]  # equal codes keep ascending ids
        np.testing.assert_array_equal(scene[:3], [0, 0, 0])
        np.testing.assert_array_equal(scene[3:6], [1, 1, 1])


def _naive_split_tree(codes: np.ndarray, bits: int) -> set:
    """Leaf sets of the radix tree built by recursive highest-differing-bit splits (with the
    index extension for equal codes) -- an independent statement of the LBVH topology."""
    n = codes.size
    keys = [(int(c) << 32) | i for i, c in enumerate(codes)] if True else None
    out = set()

    def rec(lo, hi):
        if hi - lo < 1:
            return
        out.add(frozenset(range(lo, hi + 1)))
        a, b = keys[lo], keys[hi]
        top = (a ^ b).bit_length() - 1
        split = lo
        for i in range(lo, hi):
            if (keys[i + 1] >> top) & 1 != (a >> top) & 1:
                split = i
                break
        rec(lo, split)
        rec(split + 1, hi)

    rec(0, n - 1)
    return out


@pytest.mark.parametrize("bits", [32, 64])
def test_karras_matches_naive_radix_tree(bits):
    m = meshes.to_soa(*meshes.uv_sphere(24, 12, seed=3))
    aabbs, codes, _ = oracle.morton(m, bits)
    sc, ids = oracle.sort_pairs(codes)
    nodes, ip, lp = oracle.karras(sc, bits)
    assert oracle.binary_leaf_sets(nodes, 0) == _naive_split_tree(sc, bits)
    # parent links are consistent with child references
    for i, (li, lk, ri, rk) in enumerate(nodes):
        for slot, (ci, ck) in enumerate(((li, lk), (ri, rk))):
            par = ip[ci] if ck == 1 else lp[ci]
            assert par == (i << 1) | slot


@pytest.mark.parametrize("method", ["lbvh", "hploc"])
def test_collapse_stack_bounds_and_reachability(method):
    m = meshes.to_soa(*meshes.uv_sphere(40, 21, seed=4))
    aabbs, codes, _ = oracle.morton(m, 64)
    sc, ids = oracle.sort_pairs(codes)
    saabb = aabbs[ids]
    if method == "lbvh":
        bn, _, _ = oracle.karras(sc, 64)
        root = 0
        bb = oracle.binary_bounds(bn, saabb, root)
    else:
        bn, bb, root = oracle.hploc(sc, 64, saabb, 8)
    nodes, ib, pb = oracle.collapse(bn, bb, saabb, root)
    hib, hpb, reach = host_stack_bounds(nodes, VALID, ids.size)
    assert (ib, pb) == (hib, hpb)
    assert reach == len(nodes)
    leaves = sorted(int(r & OFF) for r in nodes["reference"].ravel() if (r >> 47) & 1 and (r >> 48) != 0)
    assert leaves == list(range(ids.size))


@pytest.mark.parametrize("count", [15, 16, 17, 31, 32, 33, 63, 64, 65, 129, 513])
@pytest.mark.parametrize("radius", [1, 4, 8])
def test_hploc_equal_bounds_converges(count, radius):
    m = equal_bounds(count)
    aabbs, codes, _ = oracle.morton(m, 64)
    sc, ids = oracle.sort_pairs(codes)
    bn, bb, root = oracle.hploc(sc, 64, aabbs[ids], radius)
    assert root == count - 2
    sets = oracle.binary_leaf_sets(bn, root)
    assert frozenset(range(count)) in sets and len(sets) == count - 1
    nodes, ib, pb = oracle.collapse(bn, bb, aabbs[ids], root)
    tris = oracle.triangles(m, ids)
    q = [np.array([0.2, 0.7, -0.3], np.float32), np.array([0.2, 0.1, 0.3], np.float32),
         np.array([1, -2, 0.5], np.float32)]
    mom = oracle.moments(2, nodes, tris)
    wt = oracle.taylor(2, nodes, mom, tris, VALID, *q, beta=1e6)
    we = oracle.exact_winding(m, *q)
    assert np.all(np.abs(wt - we) <= 2e-5 + 2e-5 * np.abs(we)), (wt, we)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_full_descent_taylor_equals_exact(order):
    m = octahedron()
    b = oracle.build_lbvh(m)
    q = [np.array([0.13, 3.25], np.float32), np.array([-0.21, -2.5], np.float32), np.array([0.17, 4.75], np.float32)]
    mom = oracle.moments(order, b["nodes"], b["triangles"])
    wt = oracle.taylor(order, b["nodes"], mom, b["triangles"], b["root_reference"], *q, beta=1e6)
    we = oracle.exact_records(b["triangles"], *q)
    np.testing.assert_allclose(wt, we, atol=1e-6)


@pytest.mark.parametrize("method", ["lbvh", "hploc"])
def test_far_field_order_progression(method):
    m = asym_octahedron()
    aabbs, codes, _ = oracle.morton(m, 64)
    sc, ids = oracle.sort_pairs(codes)
    saabb = aabbs[ids]
    if method == "lbvh":
        bn, _, _ = oracle.karras(sc, 64)
        bb, root = oracle.binary_bounds(bn, saabb, 0), 0
    else:
        bn, bb, root = oracle.hploc(sc, 64, saabb, 8)
    nodes, _, _ = oracle.collapse(bn, bb, saabb, root)
    tris = oracle.triangles(m, ids)
    q = [np.array(v, np.float32) for v in ([2.9, -2.7, 0.4, -0.6, 3.2, -2.8, 1.8, -2.1],
                                          [0.4, -0.8, 3.1, -2.9, 2.2, 1.7, -2.6, 2.4],
                                          [1.1, -0.5, 0.8, -1.2, -2.3, 2.5, 2.8, -2.5])]
    ref = oracle.exact_winding(m, *q)
    errs = []
    for order in (0, 1, 2):
        mom = oracle.moments(order, nodes, tris)
        w = oracle.taylor(order, nodes, mom, tris, VALID, *q, beta=0.0)
        errs.append(float(np.mean(np.abs(w - ref))))
    assert errs[1] < errs[0] and errs[2] < errs[1] and errs[2] < 2e-3


@pytest.mark.parametrize("order", [0, 1])
def test_frozen_fp64_taylor_is_the_float_traversal_in_fp64(order):
    """The adjoint's checker: the FP64 Taylor sum with the float traversal's decisions equals the
    float traversal up to FP32 rounding (the float near field loses up to ~1e-4 at a query by an
    edge's line), and with every slot descended equals the FP64 exact sum."""
    m = meshes.soup_mesh(24, seed=7)
    b = oracle.build_lbvh(m)
    mom = oracle.moments(order, b["nodes"], b["triangles"])
    q = meshes.mixed_queries(m, 400, seed=9)
    V = np.stack([m["x"], m["y"], m["z"]], -1).astype(np.float64)
    q64 = [v.astype(np.float64) for v in q]
    w32 = oracle.taylor(order, b["nodes"], mom, b["triangles"], b["root_reference"], *q, beta=2.0)
    w64 = oracle.taylor_frozen_f64(order, b["nodes"], mom, b["root_reference"], V, m, b["sorted_ids"], q, q64,
                                   beta=2.0)
    d = np.abs(w64 - w32)
    assert np.quantile(d, 0.99) < 2e-6 and d.max() < 5e-4, (np.quantile(d, 0.99), d.max())
    full = oracle.taylor_frozen_f64(order, b["nodes"], mom, b["root_reference"], V, m, b["sorted_ids"], q, q64,
                                    beta=1e6)
    np.testing.assert_allclose(full, oracle.exact_winding(m, *q64, fp64=True), atol=1e-12)


def test_mesh_distance_known_answers():
    """Unit right triangle in z = 0: above the interior, beside the edge v0 v1, beside the
    hypotenuse, beyond vertex v0, beyond vertex v1."""
    m = single_triangle()
    q = [np.array([0.25, 0.5, 2.0, -1.0, 2.0]), np.array([0.25, -1.0, 2.0, -1.0, -1.0]),
         np.array([0.5, 0.0, 0.0, 0.0, 0.0])]
    d = oracle.mesh_distance(m, *q)
    np.testing.assert_allclose(d, [0.5, 1.0, np.sqrt(4.5), np.sqrt(2.0), np.sqrt(2.0)], atol=1e-15)


def test_leaf_root_build_record():
    b = oracle.build_lbvh(single_triangle())
    assert b["root_reference"] == VALID | (1 << 48)
    np.testing.assert_array_equal(b["triangles"][0], [0, 0, 0, 1, 0, 0, 0, 1, 0])


# ---- pinned to smallgwn's own kernels -----------------------------------------------------------

GOLDEN = golden_files()


@pytest.mark.skipif(not GOLDEN, reason="no golden vectors recorded yet")
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    g = dict(np.load(path))
    mesh = {k: g[k] for k in ("x", "y", "z", "i0", "i1", "i2")}
    q = (g["qx"], g["qy"], g["qz"])
    for bits in (32, 64):
        aabbs, codes, _ = oracle.morton(mesh, bits)
        sc, ids = oracle.sort_pairs(codes)
        np.testing.assert_array_equal(sc, g[f"codes{bits}"])
        np.testing.assert_array_equal(ids, g[f"ids{bits}"])
        np.testing.assert_array_equal(aabbs[ids], g[f"aabbs{bits}"])
        if sc.size > 1:
            bn, _, _ = oracle.karras(sc, bits)
            np.testing.assert_array_equal(bn, g[f"lbvh{bits}_nodes"])
            np.testing.assert_array_equal(oracle.binary_bounds(bn, aabbs[ids], 0), g[f"lbvh{bits}_bounds"])
            hn, hb, hroot = oracle.hploc(sc, bits, aabbs[ids], 8)
            sets = sorted(sorted(s) for s in oracle.binary_leaf_sets(hn, hroot))
            flat = np.array([x for s in sets for x in [len(s)] + s], np.uint32)
            np.testing.assert_array_equal(flat, g[f"hploc{bits}_leafsets"])
    b = oracle.build_lbvh(mesh, 64)
    meta = g["lbvh_meta"]
    assert int(meta[1]) == b["internal_stack_bound"] and int(meta[2]) == b["packed_stack_bound"]
    assert oracle.canonical_wide(b["nodes"], b["root_reference"]) == oracle.canonical_wide(g["lbvh_nodes"], int(meta[0]))
    np.testing.assert_array_equal(b["triangles"], g["lbvh_tris"])
    # FP32 tolerance of smallgwn's builder tests: 2e-5 + 2e-5 |w| (tests/integration_gwn_builder.cu:228-233)
    np.testing.assert_allclose(oracle.exact_winding(mesh, *q), g["exact"], atol=1e-5, rtol=2e-5)
    np.testing.assert_allclose(oracle.exact_winding(mesh, *q, fp64=True), g["exact_f64"], atol=1e-12, rtol=1e-12)
    # moments and Taylor on the reference's own tree
    for order in (0, 1, 2):
        mom = oracle.moments(order, g["lbvh_nodes"], g["lbvh_tris"])
        ref_mom = g[f"moment{order}"]
        scale = np.abs(ref_mom).max(axis=(0, 2), keepdims=True) + 1e-12
        assert np.max(np.abs(mom - ref_mom) / scale) < 1e-4
        w2 = oracle.taylor(order, g["lbvh_nodes"], ref_mom, g["lbvh_tris"], int(meta[0]), *q, beta=2.0)
        np.testing.assert_allclose(w2, g[f"taylor{order}_b2"], atol=1e-5, rtol=2e-5)
        w6 = oracle.taylor(order, g["lbvh_nodes"], ref_mom, g["lbvh_tris"], int(meta[0]), *q, beta=1e6)
        np.testing.assert_allclose(w6, g[f"taylor{order}_b1e6"], atol=1e-5, rtol=2e-5)


# ---- the oracle against smallgwn's own CPU reference code (oracle/_ref/libgwnrefcpu.so) -------------

REF_CPU = oracle.ref_cpu_lib() is not None


@pytest.mark.skipif(not REF_CPU, reason="smallgwn's CPU reference code (oracle/_ref/libgwnrefcpu.so) not built")
@pytest.mark.parametrize("name", ["small", "soup", "octahedron"])
def test_oracle_exact_is_the_reference_cpu_exact_bit_for_bit(name):
    """The oracle's FP32 exact brute force restates tests/reference_cpu.cuh:22-114; compiled from
    the reference's own source (Eigen / oneTBB stand-ins), that code gives the same bits."""
    from conftest import octahedron
    from smallgwn_b200 import meshes

    mesh = {"small": meshes.small_mesh, "soup": lambda: meshes.soup_mesh(24, seed=11), "octahedron": octahedron}[name]()
    q = meshes.small_queries(3000) if name != "soup" else meshes.mixed_queries(mesh, 3000, seed=7)
    np.testing.assert_array_equal(oracle.reference_cpu_exact(mesh, *q), oracle.exact_winding(mesh, *q))


@pytest.mark.skipif(not REF_CPU, reason="smallgwn's CPU reference code (oracle/_ref/libgwnrefcpu.so) not built")
def test_reference_hdk_taylor_within_the_reference_tolerances_of_the_oracle_traversal():
    """smallgwn's CPU Taylor path (the vendored SideFX HDK tree, tests/reference_hdk.cuh) against the
    oracle's restatement of smallgwn's GPU traversal on the same mesh at accuracy scale 2, within the
    tolerances smallgwn holds its GPU Taylor batch to against HDK (tests/e2e_gwn.cu:103-106):
    5e-2, 3e-2, 2e-2 for orders 0, 1, 2."""
    from smallgwn_b200 import meshes

    mesh = meshes.to_soa(*meshes.uv_sphere(64, 32, seed=9))
    q = meshes.mixed_queries(mesh, 4000, seed=3)
    b = oracle.build_bvh(mesh, "hploc", radius=8)
    for order, eps in ((0, 5e-2), (1, 3e-2), (2, 2e-2)):
        hdk = oracle.ReferenceHDK(mesh, order)
        try:
            got = hdk.query(*q, beta=2.0)
        finally:
            hdk.close()
        mom = oracle.moments(order, b["nodes"], b["triangles"])
        ref = oracle.taylor(order, b["nodes"], mom, b["triangles"], b["root_reference"], *q, beta=2.0)
        assert np.max(np.abs(got - ref)) <= eps, (order, np.max(np.abs(got - ref)))
