"""Bit-exact build parity at the benchmark's mesh sizes.

The small-mesh build tests (test_gpu_build.py) cover one or two sort tiles of the onesweep radix
sort. Here the meshes are the workloads' own: the 1,046,528-triangle displaced sphere (1024 x 512,
seed 2; 256 tiles of the decoupled look-back) and the 8,381,024-triangle one (2896 x 1448, seed 5;
2,047 tiles). Against the oracle's C restatement, bit for bit:
- Morton codes (30- and 63-bit, detail/gwn_bvh_build_common.cuh:31-214), the stable sorted
  permutation and the sorted triangle boxes (:290-367);
- Karras LBVH topology and internal bounds (detail/gwn_bvh_build_binary.cuh:29-192);
- the LBVH BVH4: nodes, primitive order, triangle records and both stack bounds;
- H-PLOC (radius 8): the family of leaf sets under every binary node equals the oracle's (the
  internal numbering is scheduling-dependent; fingerprints per node, oracle.binary_leaf_set_hashes).
Against smallgwn's own kernels (oracle/_ref) on the 1M-triangle sphere: the same codes,
permutation and boxes, Karras topology, and the LBVH BVH4 up to node numbering.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import _lib, api, meshes
from test_gpu_build import build, device_preprocess, upload

pytestmark = pytest.mark.gpu

MESHES = {
    "sphere1m": lambda: meshes.sphere_mesh(),
    "sphere8m": lambda: meshes.sphere_mesh(2896, 1448, seed=5),
}
_cache: dict = {}


def mesh_of(name):
    if name not in _cache:
        _cache.clear()  # one large mesh on the host at a time
        _cache[name] = MESHES[name]()
    return _cache[name]


def device_binary(cuda, codes, aabbs, bits, hploc_radius=None):
    n = codes.size
    dc = cuda.from_numpy(codes.astype(np.uint64 if bits == 64 else np.uint32).view(
        np.int64 if bits == 64 else np.int32)).cuda()
    da = cuda.from_numpy(np.ascontiguousarray(aabbs)).cuda()
    bn = cuda.empty((n - 1, 4), dtype=cuda.int32, device="cuda")
    bp = cuda.empty(n - 1, dtype=cuda.int32, device="cuda")
    bb = cuda.empty((n - 1, 6), dtype=cuda.float32, device="cuda")
    lib = _lib.load()
    if hploc_radius is None:
        rc = lib.gwnb_build_binary_lbvh(dc.data_ptr(), bits, n, da.data_ptr(), bn.data_ptr(), bp.data_ptr(),
                                        bb.data_ptr(), None)
        root = 0
    else:
        r = C.c_uint32()
        rc = lib.gwnb_build_binary_hploc(dc.data_ptr(), bits, n, da.data_ptr(), hploc_radius, bn.data_ptr(),
                                         bp.data_ptr(), bb.data_ptr(), C.byref(r), None)
        root = r.value
    assert rc == 0, _lib.last_error()
    return bn.cpu().numpy().view(np.uint32), bb.cpu().numpy(), root


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("name", list(MESHES))
def test_morton_sort_karras_bit_exact_at_size(cuda, name, bits):
    mesh = mesh_of(name)
    geo = upload(mesh)
    codes, ids, aabbs = device_preprocess(cuda, geo, bits)
    o_aabb, o_codes, _ = oracle.morton(mesh, bits)
    o_sorted, o_ids = oracle.sort_pairs(o_codes)
    np.testing.assert_array_equal(codes, o_sorted)
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(aabbs, o_aabb[o_ids])
    bn, bb, _ = device_binary(cuda, codes, aabbs, bits)
    o_nodes, _, _ = oracle.karras(o_sorted, bits)
    np.testing.assert_array_equal(bn, o_nodes)
    np.testing.assert_array_equal(bb, oracle.binary_bounds(o_nodes, o_aabb[o_ids], 0))


@pytest.mark.parametrize("name", list(MESHES))
def test_lbvh_bvh4_bit_exact_at_size(cuda, name):
    mesh = mesh_of(name)
    bvh = build(upload(mesh), bits=64)
    h = api.bvh_host_arrays(bvh)
    ob = oracle.build_lbvh(mesh, 64)
    np.testing.assert_array_equal(h["primitive_indices"], ob["sorted_ids"])
    np.testing.assert_array_equal(h["nodes"]["reference"], ob["nodes"]["reference"])
    np.testing.assert_array_equal(h["nodes"]["bounds"], ob["nodes"]["bounds"])
    np.testing.assert_array_equal(h["triangles"], ob["triangles"])
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (ob["internal_stack_bound"],
                                                                   ob["packed_stack_bound"])


@pytest.mark.parametrize("name", list(MESHES))
def test_hploc_leaf_sets_equal_oracle_at_size(cuda, name):
    mesh = mesh_of(name)
    geo = upload(mesh)
    codes, _, aabbs = device_preprocess(cuda, geo, 64)
    bn, _, root = device_binary(cuda, codes, aabbs, 64, hploc_radius=8)
    assert root == codes.size - 2
    o_nodes, _, o_root = oracle.hploc(codes, 64, aabbs, 8)
    np.testing.assert_array_equal(oracle.binary_leaf_set_hashes(bn, root),
                                  oracle.binary_leaf_set_hashes(o_nodes, o_root))
    # the full H-PLOC build (collapse included) holds every primitive exactly once
    h = api.bvh_host_arrays(build(geo, g.gwn_bvh_build_method.k_hploc, 8))
    np.testing.assert_array_equal(np.sort(h["primitive_indices"]), np.arange(codes.size, dtype=np.uint32))


@pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's own kernels (oracle/_ref) not built")
def test_build_matches_reference_kernels_at_size(cuda):
    mesh = mesh_of("sphere1m")
    geo = upload(mesh)
    R = oracle.Reference(mesh)
    try:
        for bits in (32, 64):
            codes, ids, aabbs = device_preprocess(cuda, geo, bits)
            rc, rids, raabbs = R.preprocess(bits)
            np.testing.assert_array_equal(codes, rc)
            np.testing.assert_array_equal(ids, rids)
            np.testing.assert_array_equal(aabbs, raabbs)
            rn, _, _ = oracle.ref_binary(1, bits, rc, raabbs)
            bn, _, _ = device_binary(cuda, codes, aabbs, bits)
            np.testing.assert_array_equal(bn, rn)
        R.build(1, 8, 64)
        rb = R.bvh()
        h = api.bvh_host_arrays(build(geo))
        assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (rb["internal_stack_bound"],
                                                                       rb["packed_stack_bound"])
        oracle.match_wide_nodes(h["nodes"], h["root_reference"], rb["nodes"], rb["root_reference"])
        np.testing.assert_array_equal(h["primitive_indices"], rb["primitive_indices"])
        np.testing.assert_array_equal(h["triangles"], rb["triangles"])
    finally:
        R.close()
