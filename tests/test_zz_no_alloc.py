"""The Taylor batch that allocates no device memory matches the allocating one.

gwnb_winding_taylor_batch_noalloc_f32 exists for callers that cannot let a library allocate device
memory during a query: engines that hand the library a fixed memory budget and account for every
byte themselves, real-time loops where an allocation would stall a frame, and replayed work that
forbids new allocations. It keeps its query-ordering scratch in one file-scope device array of
GWNB_NOALLOC_MAX_QUERIES queries instead of allocating per call.

The test calls it through the C ABI twice in a row (the second call runs on scratch left over from
the first) on a batch of exactly GWNB_NOALLOC_MAX_QUERIES queries, so every scratch region and the
sort's last tile are full, and compares both results with gwnb_winding_taylor_batch_f32 on the same
inputs. It checks the property the entry point exists for: across both calls the library's device
memory pool neither grows nor hands out memory (gwnb_memory_stats, after the allocating batch's
scratch is trimmed back). It builds everything it needs, so it passes in a fresh process as well as
after the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import smallgwn_b200 as g
from smallgwn_b200 import _lib, api, meshes

pytestmark = pytest.mark.gpu

MAX_QUERIES = 262144  # GWNB_NOALLOC_MAX_QUERIES in include/gwnb.h


def test_no_alloc_taylor_batch_matches_allocating_batch():
    import torch

    torch.cuda.set_device(0)
    mesh = meshes.to_soa(*meshes.uv_sphere(128, 64, seed=5))
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=g.gwn_bvh_build_method.k_hploc)).is_ok()
    mom = g.gwn_bvh4_moment_object(2)
    assert g.gwn_refit_bvh_moment(2, bvh, mom).is_ok()

    n = MAX_QUERIES
    q = [torch.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, n, seed=23)]
    expected = torch.empty(n, device="cuda")
    assert g.gwn_compute_winding_number_taylor_batch(2, bvh, mom, *q, expected, accuracy_scale=3.0).is_ok()
    torch.cuda.synchronize()
    want = expected.cpu().numpy()

    lib = _lib.load()
    opt = _lib.taylor_options(256, 64, 1, _lib.GWNB_NEAR_PLAIN, 1e-3, 0)
    outs = [torch.full((n,), float("nan"), device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    assert api.memory_trim(0).is_ok()
    pool_before = api.memory_stats()
    for out in outs:
        rc = lib.gwnb_winding_taylor_batch_noalloc_f32(
            C.byref(bvh.accessor()), C.byref(mom.accessor()), q[0].data_ptr(), q[1].data_ptr(), q[2].data_ptr(),
            out.data_ptr(), n, 3.0, C.byref(opt), None)
        assert rc == _lib.GWNB_OK, _lib.last_error()
        torch.cuda.synchronize()
        assert api.memory_stats() == pool_before
    for out in outs:
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, want, atol=1e-6, rtol=1e-6)

    # batches above the fixed scratch capacity are refused before any work is queued
    rc = lib.gwnb_winding_taylor_batch_noalloc_f32(
        C.byref(bvh.accessor()), C.byref(mom.accessor()), q[0].data_ptr(), q[1].data_ptr(), q[2].data_ptr(),
        expected.data_ptr(), MAX_QUERIES + 1, 3.0, C.byref(opt), None)
    assert rc == _lib.GWNB_INVALID_ARGUMENT
    assert "maximum" in _lib.last_error()
    # the timed walk choice keeps CUDA events, which this entry point does not create
    timed = _lib.taylor_options(256, 64, 1, _lib.GWNB_NEAR_PLAIN, 1e-3, _lib.GWNB_WALK_TIMED)
    rc = lib.gwnb_winding_taylor_batch_noalloc_f32(
        C.byref(bvh.accessor()), C.byref(mom.accessor()), q[0].data_ptr(), q[1].data_ptr(), q[2].data_ptr(),
        expected.data_ptr(), n, 3.0, C.byref(timed), None)
    assert rc == _lib.GWNB_INVALID_ARGUMENT and "Unknown traversal" in _lib.last_error()
