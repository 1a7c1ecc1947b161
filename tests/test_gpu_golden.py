"""The GPU path against the golden vectors recorded from smallgwn's own kernels (tests/golden/,
written by tests/golden/make_golden.py on a B200): six fixture meshes (asymmetric octahedron, cube,
icosphere level 2, displaced 32 x 16 sphere, open soup, 129 coincident triangles) with 64 queries
each, uniform in 1.6x the mesh's half extent.

Bit for bit: sorted Morton codes (30/63-bit), the sorted permutation and boxes, the Karras binary
topology and bounds, H-PLOC leaf sets, and the LBVH BVH4 up to node numbering with its primitive
order, triangle records and stack bounds. Within tolerance: exact and Taylor (beta = 2, 1e6)
winding numbers within 1e-5 + 2e-5 |w| of smallgwn's, every disagreement explained in FP64
(tests/taylor_decisions.py); full descent with the compensated near field within 1e-6 of smallgwn's
FP64 exact winding number (its own check is 1e-6, tests/unit_gwn_bvh_moment.cu:42-114).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from conftest import golden_files
from smallgwn_b200 import api
from test_gpu_build import build, device_preprocess, upload
from test_gpu_build_fullsize import device_binary
from test_gpu_query import assert_agree_or_explained, moments_of, run_exact, run_taylor

pytestmark = pytest.mark.gpu

GOLDEN = golden_files()


@pytest.mark.skipif(not GOLDEN, reason="no golden vectors recorded")
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_gpu_matches_reference_golden(cuda, path):
    gd = dict(np.load(path))
    mesh = {k: gd[k] for k in ("x", "y", "z", "i0", "i1", "i2")}
    q = (gd["qx"], gd["qy"], gd["qz"])
    geo = upload(mesh)
    for bits in (32, 64):
        codes, ids, aabbs = device_preprocess(cuda, geo, bits)
        np.testing.assert_array_equal(codes, gd[f"codes{bits}"])
        np.testing.assert_array_equal(ids, gd[f"ids{bits}"])
        np.testing.assert_array_equal(aabbs, gd[f"aabbs{bits}"])
        if codes.size > 1:
            bn, bb, _ = device_binary(cuda, codes, aabbs, bits)
            np.testing.assert_array_equal(bn, gd[f"lbvh{bits}_nodes"])
            np.testing.assert_array_equal(bb, gd[f"lbvh{bits}_bounds"])
            hn, _, hroot = device_binary(cuda, codes, aabbs, bits, hploc_radius=8)
            sets = sorted(sorted(s) for s in oracle.binary_leaf_sets(hn, hroot))
            flat = np.array([x for s in sets for x in [len(s)] + s], np.uint32)
            np.testing.assert_array_equal(flat, gd[f"hploc{bits}_leafsets"])
    bvh = build(geo)
    h = api.bvh_host_arrays(bvh)
    meta = gd["lbvh_meta"]
    assert (h["internal_stack_bound"], h["packed_stack_bound"]) == (int(meta[1]), int(meta[2]))
    pairing = oracle.match_wide_nodes(h["nodes"], h["root_reference"], gd["lbvh_nodes"], int(meta[0]))
    np.testing.assert_array_equal(h["primitive_indices"], gd["lbvh_prims"])
    np.testing.assert_array_equal(h["triangles"], gd["lbvh_tris"])

    mh0 = api.moment_host_array(moments_of(bvh, 0))
    exact = run_exact(cuda, bvh, q)
    assert_agree_or_explained(exact, gd["exact"], q, h, mh0, mh0, None, 1e6, allow=("conditioning",), rel=0.0)
    # 1e-6; on the 129 stacked copies of one triangle every term carries the same FP32 rounding, 129
    # times over, so there the bound is relative, 2e-6 |w|
    w64 = np.abs(gd["exact_f64"])
    tol = (2e-6 * np.maximum(1.0, w64) if path.stem.startswith("equal") else np.full_like(w64, 1e-6)) + \
        np.spacing(w64.astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(exact - gd["exact_f64"]) <= tol)
    for order in (0, 1, 2):
        mom = moments_of(bvh, order)
        mh = api.moment_host_array(mom)
        ref_m = gd[f"moment{order}"]
        scale = np.abs(ref_m).max(axis=(0, 2), keepdims=True) + 1e-12
        assert np.max(np.abs(mh - ref_m[pairing]) / scale) < 1e-4
        assert_agree_or_explained(run_taylor(cuda, order, bvh, mom, q, 2.0), gd[f"taylor{order}_b2"], q, h, mh, ref_m,
                                  pairing, 2.0, allow=("decision", "conditioning", "moments"))
        assert_agree_or_explained(run_taylor(cuda, order, bvh, mom, q, 1e6), gd[f"taylor{order}_b1e6"], q, h, mh, mh,
                                  None, 1e6, allow=("conditioning",), rel=0.0)
        full = run_taylor(cuda, order, bvh, mom, q, 1e6, precision=g.near_precision.compensated)
        assert np.all(np.abs(full - gd["exact_f64"]) <= tol)
