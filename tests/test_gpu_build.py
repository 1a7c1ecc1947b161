"""GPU parity of the build: Morton codes, sorted permutation, LBVH topology and the BVH4 are
bit-identical to the oracle (and to smallgwn's own kernels when oracle/_ref is built); H-PLOC
trees match up to internal-node numbering; triangle records, stack bounds, refit bounds.

Known answers restate smallgwn's tests: leaf-root record (tests/unit_gwn_bvh.cu:93-139),
two-triangle records (:141-218), refit bounds (-7,-4,-6)-(11,9,3) and preserved primitive order
(:220-287), strong guarantee on rejected options (:289-358), refit with a changed triangle count
(:412-465), exact stack bounds and reachability (tests/integration_gwn_builder.cu:35-119).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from conftest import asym_octahedron, equal_bounds, octahedron, single_triangle
from smallgwn_b200 import _lib, api, meshes
from test_oracle import host_stack_bounds

pytestmark = pytest.mark.gpu

VALID = 1 << 47


def upload(mesh, stream=None):
    geo = g.gwn_geometry_object()
    st = g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"], stream)
    assert st.is_ok(), st.message
    return geo


def build(geo, method=g.gwn_bvh_build_method.k_lbvh, radius=8, bits=64):
    bvh = g.gwn_bvh4_object()
    st = g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=method, hploc_search_radius=radius),
                         morton_bits=bits)
    assert st.is_ok(), st.message
    return bvh


def device_preprocess(cuda, geo, bits):
    n = geo.triangle_count()
    codes = cuda.empty(n, dtype=cuda.int64 if bits == 64 else cuda.int32, device="cuda")
    ids = cuda.empty(n, dtype=cuda.int32, device="cuda")
    aabbs = cuda.empty((n, 6), dtype=cuda.float32, device="cuda")
    rc = _lib.load().gwnb_build_preprocess_f32(C.byref(geo.accessor()), bits, codes.data_ptr(), ids.data_ptr(),
                                               aabbs.data_ptr(), None)
    assert rc == 0, _lib.last_error()
    c = codes.cpu().numpy().view(np.uint64 if bits == 64 else np.uint32).astype(np.uint64)
    return c, ids.cpu().numpy().view(np.uint32), aabbs.cpu().numpy()


WORKLOADS = {
    "icosphere4": lambda: meshes.small_mesh(),
    "uv64x32": lambda: meshes.to_soa(*meshes.uv_sphere(64, 32, seed=9)),
    "soup40": lambda: meshes.soup_mesh(40, seed=13),
    "equal_513": lambda: equal_bounds(513),
    "octahedron": octahedron,
}


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_morton_and_permutation_bit_exact(cuda, name, bits):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    codes, ids, aabbs = device_preprocess(cuda, geo, bits)
    o_aabb, o_codes, _ = oracle.morton(mesh, bits)
    o_sorted, o_ids = oracle.sort_pairs(o_codes)
    np.testing.assert_array_equal(codes, o_sorted)
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(aabbs, o_aabb[o_ids])


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_lbvh_topology_and_bvh4_bit_exact(cuda, name, bits):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    # binary LBVH through the stage entry point
    codes, ids, aabbs = device_preprocess(cuda, geo, bits)
    n = codes.size
    dc = cuda.from_numpy(codes.astype(np.uint64 if bits == 64 else np.uint32).view(
        np.int64 if bits == 64 else np.int32)).cuda()
    da = cuda.from_numpy(aabbs).cuda()
    bn = cuda.empty((n - 1, 4), dtype=cuda.int32, device="cuda")
    bp = cuda.empty(n - 1, dtype=cuda.int32, device="cuda")
    bb = cuda.empty((n - 1, 6), dtype=cuda.float32, device="cuda")
    rc = _lib.load().gwnb_build_binary_lbvh(dc.data_ptr(), bits, n, da.data_ptr(), bn.data_ptr(), bp.data_ptr(),
                                            bb.data_ptr(), None)
    assert rc == 0, _lib.last_error()
    o_nodes, _, _ = oracle.karras(codes, bits)
    np.testing.assert_array_equal(bn.cpu().numpy().view(np.uint32), o_nodes)
    np.testing.assert_array_equal(bb.cpu().numpy(), oracle.binary_bounds(o_nodes, aabbs, 0))
    # full build: canonical breadth-first BVH4 identical to the oracle's
    bvh = build(geo, bits=bits)
    h = api.bvh_host_arrays(bvh)
    ob = oracle.build_lbvh(mesh, bits)
    np.testing.assert_array_equal(h["primitive_indices"], ob["sorted_ids"])
    np.testing.assert_array_equal(h["nodes"]["reference"], ob["nodes"]["reference"])
    np.testing.assert_array_equal(h["nodes"]["bounds"], ob["nodes"]["bounds"])
    np.testing.assert_array_equal(h["triangles"], ob["triangles"])
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (ob["internal_stack_bound"], ob["packed_stack_bound"])
    ib, pb, reach = host_stack_bounds(h["nodes"], h["root_reference"], n)
    assert (ib, pb, reach) == (h["internal_stack_bound"], h["packed_stack_bound"], len(h["nodes"]))


@pytest.mark.parametrize("radius", [1, 4, 8])
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40"])
def test_hploc_tree_matches_oracle_up_to_numbering(cuda, name, radius):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    codes, ids, aabbs = device_preprocess(cuda, geo, 64)
    n = codes.size
    dc = cuda.from_numpy(codes.view(np.int64)).cuda()
    da = cuda.from_numpy(aabbs).cuda()
    bn = cuda.empty((n - 1, 4), dtype=cuda.int32, device="cuda")
    bp = cuda.empty(n - 1, dtype=cuda.int32, device="cuda")
    bb = cuda.empty((n - 1, 6), dtype=cuda.float32, device="cuda")
    root = C.c_uint32()
    rc = _lib.load().gwnb_build_binary_hploc(dc.data_ptr(), 64, n, da.data_ptr(), radius, bn.data_ptr(),
                                             bp.data_ptr(), bb.data_ptr(), C.byref(root), None)
    assert rc == 0, _lib.last_error()
    assert root.value == n - 2
    o_nodes, o_bounds, o_root = oracle.hploc(codes, 64, aabbs, radius)
    assert oracle.binary_leaf_sets(bn.cpu().numpy().view(np.uint32), root.value) == \
        oracle.binary_leaf_sets(o_nodes, o_root)


@pytest.mark.parametrize("count", [15, 16, 17, 31, 32, 33, 63, 64, 65, 129, 513])
def test_hploc_equal_bounds_builds(cuda, count):
    geo = upload(equal_bounds(count))
    for radius in (1, 4, 8):
        bvh = build(geo, g.gwn_bvh_build_method.k_hploc, radius)
        h = api.bvh_host_arrays(bvh)
        ib, pb, reach = host_stack_bounds(h["nodes"], h["root_reference"], count)
        assert (ib, pb, reach) == (h["internal_stack_bound"], h["packed_stack_bound"], len(h["nodes"]))
        assert sorted(h["primitive_indices"].tolist()) == list(range(count))


def test_leaf_root_build_record(cuda):
    bvh = build(upload(single_triangle()), g.gwn_bvh_build_method.k_hploc)
    h = api.bvh_host_arrays(bvh)
    assert h["root_reference"] == VALID | (1 << 48) and len(h["nodes"]) == 0
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (0, 0)
    np.testing.assert_array_equal(h["root_bounds"], [0, 0, 0, 1, 1, 0])
    np.testing.assert_array_equal(h["triangles"][0], [0, 0, 0, 1, 0, 0, 0, 1, 0])


def two_triangles():
    return {"x": np.array([0, 1, 0, 4, 6, 4], np.float32), "y": np.array([0, 0, 2, 0, 0, 3], np.float32),
            "z": np.array([1, 1, 1, -2, -2, -2], np.float32), "i0": np.array([0, 3], np.uint32),
            "i1": np.array([1, 4], np.uint32), "i2": np.array([2, 5], np.uint32)}


def test_two_triangle_records_and_refit(cuda):
    m = two_triangles()
    geo = upload(m)
    bvh = build(geo)
    h = api.bvh_host_arrays(bvh)
    assert len(h["nodes"]) == 1
    kids = [r for r in h["nodes"][0]["reference"] if (r >> 47) & 1]
    assert len(kids) == 2 and all((r >> 48) == 1 for r in kids)
    order_before = h["primitive_indices"].copy()
    x = np.array([-7, -2, -7, 8, 11, 8], np.float32)
    y = np.array([5, 5, 9, -4, -4, 2], np.float32)
    z = np.array([3, 3, 3, -6, -6, -6], np.float32)
    assert g.gwn_update_geometry(geo, x, y, z).is_ok()
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    h = api.bvh_host_arrays(bvh)
    np.testing.assert_array_equal(h["primitive_indices"], order_before)
    np.testing.assert_array_equal(h["root_bounds"], [-7, -4, -6, 11, 9, 3])
    for s, pid in enumerate(h["primitive_indices"]):
        a, b, c = m["i0"][pid], m["i1"][pid], m["i2"][pid]
        np.testing.assert_array_equal(h["triangles"][s], [x[a], y[a], z[a], x[b] - x[a], y[b] - y[a], z[b] - z[a],
                                                         x[c] - x[a], y[c] - y[a], z[c] - z[a]])


@pytest.mark.parametrize("method", [g.gwn_bvh_build_method.k_lbvh, g.gwn_bvh_build_method.k_hploc])
def test_refit_equals_fresh_build_bounds(cuda, method):
    base = meshes.to_soa(*meshes.uv_sphere(48, 24, seed=21))
    moved = meshes.to_soa(*meshes.uv_sphere(48, 24, seed=22))
    geo = upload(base)
    bvh = build(geo, method)
    assert g.gwn_update_geometry(geo, moved["x"], moved["y"], moved["z"]).is_ok()
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    h = api.bvh_host_arrays(bvh)
    # bottom-up recomputation of every child bound from the moved triangle records
    nodes = h["nodes"]
    tri = h["triangles"]
    v0 = tri[:, 0:3]
    v1 = v0 + tri[:, 3:6]
    v2 = v0 + tri[:, 6:9]
    P = np.stack([moved["x"], moved["y"], moved["z"]], -1)
    ids = h["primitive_indices"]
    np.testing.assert_array_equal(v0, P[moved["i0"][ids]])
    lo = np.minimum(np.minimum(P[moved["i0"][ids]], P[moved["i1"][ids]]), P[moved["i2"][ids]])
    hi = np.maximum(np.maximum(P[moved["i0"][ids]], P[moved["i1"][ids]]), P[moved["i2"][ids]])
    box = {}

    def node_box(i):
        if i in box:
            return box[i]
        l, u = np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)
        for s in range(4):
            r = int(nodes[i, s]["reference"])
            if not (r >> 47) & 1:
                continue
            if (r >> 48) == 0:
                cl, cu = node_box(r & (VALID - 1))
            else:
                off = r & (VALID - 1)
                cl, cu = lo[off], hi[off]
            np.testing.assert_array_equal(nodes[i, s]["bounds"], np.concatenate([cl, cu]))
            l, u = np.minimum(l, cl), np.maximum(u, cu)
        box[i] = (l, u)
        return box[i]

    l, u = node_box(0)
    np.testing.assert_array_equal(h["root_bounds"], np.concatenate([l, u]))
    del v1, v2


def test_rejected_options_preserve_bvh_and_stream(cuda):
    s_a = cuda.cuda.Stream()
    s_b = cuda.cuda.Stream()
    geo = upload(single_triangle(), s_a)
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(), s_a).is_ok()
    before = (bvh.accessor().nodes, bvh.accessor().primitive_indices, bvh.accessor().triangles,
              bvh.accessor().root.reference)
    for opts in (g.gwn_bvh_build_options(method=0xff), g.gwn_bvh_build_options(method=0, hploc_search_radius=0),
                 g.gwn_bvh_build_options(method=0, hploc_search_radius=9)):
        st = g.gwn_build_bvh(geo, bvh, opts, s_b)
        assert st.error == g.gwn_error.invalid_argument
        assert bvh.stream() is s_a
        assert (bvh.accessor().nodes, bvh.accessor().primitive_indices, bvh.accessor().triangles,
                bvh.accessor().root.reference) == before
    s_a.synchronize()


def test_refit_rejects_topology_change(cuda):
    geo1 = upload(single_triangle())
    bvh = build(geo1)
    before = api.bvh_host_arrays(bvh)
    geo2 = upload({"x": np.array([0, 1, 0, 1], np.float32), "y": np.array([0, 0, 1, 1], np.float32),
                   "z": np.zeros(4, np.float32), "i0": np.array([0, 1], np.uint32),
                   "i1": np.array([1, 3], np.uint32), "i2": np.array([2, 2], np.uint32)})
    st = g.gwn_refit_bvh(geo2, bvh)
    assert st.error == g.gwn_error.invalid_argument
    after = api.bvh_host_arrays(bvh)
    np.testing.assert_array_equal(after["triangles"], before["triangles"])
    assert after["root_reference"] == before["root_reference"] and after["revision"] == before["revision"]


def test_failed_refit_leaves_bvh_unqueryable_then_rebuildable(cuda):
    m = asym_octahedron()
    geo = upload(m)
    bvh = build(geo)
    mom = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
    # corrupt one device index (host-side fault injection into device geometry)
    bad = np.array([m["x"].size], np.uint32)
    cudart = api._cudart()
    dst = geo.accessor().tri_i0 + 4 * (m["i0"].size - 1)
    assert cudart.cudaMemcpy(C.c_void_p(dst), C.c_void_p(bad.ctypes.data), 4, 1) == 0
    st = g.gwn_refit_bvh(geo, bvh)
    assert st.error == g.gwn_error.internal_error
    assert not bvh.has_data() and not mom.is_valid_for(bvh)
    good = np.array([m["i0"][-1]], np.uint32)
    assert cudart.cudaMemcpy(C.c_void_p(dst), C.c_void_p(good.ctypes.data), 4, 1) == 0
    bvh.clear()
    assert g.gwn_build_bvh(geo, bvh).is_ok() and bvh.has_data()


def test_build_rejects_invalid_upload_indices(cuda):
    m = single_triangle()
    geo = g.gwn_geometry_object()
    st = g.gwn_upload_geometry(geo, m["x"], m["y"], m["z"], [0], [1], [7])
    assert st.error == g.gwn_error.invalid_argument and not geo.has_data()


def test_empty_geometry_build_clears_bvh(cuda):
    geo = upload(single_triangle())
    bvh = build(geo)
    empty = g.gwn_geometry_object()
    assert g.gwn_build_bvh(empty, bvh).is_ok()
    assert not bvh.has_data()


@pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's own kernels (oracle/_ref) not built")
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40", "equal_513"])
def test_build_matches_reference_kernels(cuda, name):
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    R = oracle.Reference(mesh)
    for bits in (32, 64):
        codes, ids, aabbs = device_preprocess(cuda, geo, bits)
        rc, rids, raabbs = R.preprocess(bits)
        np.testing.assert_array_equal(codes, rc)
        np.testing.assert_array_equal(ids, rids)
        np.testing.assert_array_equal(aabbs, raabbs)
        rn, rb, _ = oracle.ref_binary(1, bits, rc, raabbs)
        on, _, _ = oracle.karras(codes, bits)
        np.testing.assert_array_equal(on, rn)
    R.build(1, 8, 64)
    rb = R.bvh()
    bvh = build(geo)
    h = api.bvh_host_arrays(bvh)
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (rb["internal_stack_bound"], rb["packed_stack_bound"])
    assert oracle.canonical_wide(h["nodes"], h["root_reference"]) == oracle.canonical_wide(rb["nodes"], rb["root_reference"])
    np.testing.assert_array_equal(h["primitive_indices"], rb["primitive_indices"])
    np.testing.assert_array_equal(h["triangles"], rb["triangles"])
    R.close()


def deep_mesh(n: int = 420) -> dict:
    """Small triangles at x = 1.1^k: H-PLOC merges them into a caterpillar whose BVH4 has 40 levels,
    deeper than the levels a build enqueues before its single read-back."""
    xs = (1.1 ** np.arange(n)).astype(np.float32)
    return {"x": np.concatenate([xs, xs + xs * np.float32(1e-3), xs]).astype(np.float32),
            "y": np.concatenate([np.zeros(n), np.zeros(n), xs * np.float32(1e-3)]).astype(np.float32),
            "z": np.zeros(3 * n, np.float32), "i0": np.arange(n, dtype=np.uint32),
            "i1": np.arange(n, 2 * n, dtype=np.uint32), "i2": np.arange(2 * n, 3 * n, dtype=np.uint32)}


def test_build_deeper_than_first_collapse_batch(cuda):
    mesh = deep_mesh()
    h = api.bvh_host_arrays(build(upload(mesh), g.gwn_bvh_build_method.k_hploc))
    ob = oracle.build_bvh(mesh, "hploc", radius=8)
    assert oracle.canonical_wide(h["nodes"], h["root_reference"]) == oracle.canonical_wide(ob["nodes"], (1 << 47))
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (ob["internal_stack_bound"],
                                                                   ob["packed_stack_bound"])
    ib, pb, reach = host_stack_bounds(h["nodes"], h["root_reference"], mesh["i0"].size)
    assert (ib, pb, reach) == (h["internal_stack_bound"], h["packed_stack_bound"], len(h["nodes"]))
    # the refit state derived on that path is complete: a refit reproduces the bounds
    before = api.bvh_host_arrays(build(upload(mesh), g.gwn_bvh_build_method.k_hploc))
    geo = upload(mesh)
    bvh = build(geo, g.gwn_bvh_build_method.k_hploc)
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    np.testing.assert_array_equal(api.bvh_host_arrays(bvh)["nodes"]["bounds"], before["nodes"]["bounds"])
