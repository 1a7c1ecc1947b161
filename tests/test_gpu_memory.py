"""The library's device memory pool: freed scratch stays mapped across host synchronizations (so
repeated builds do not map memory again), gwnb_memory_trim hands it back, and work after a trim is
unaffected."""
from __future__ import annotations

import numpy as np
import pytest

import smallgwn_b200 as g
from smallgwn_b200 import api, meshes
from test_gpu_build import upload

pytestmark = pytest.mark.gpu


def test_pool_retains_and_trims(cuda):
    mesh = meshes.sphere_mesh()  # 1M triangles: the build's scratch spans several pool chunks
    geo = upload(mesh)
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=0, hploc_search_radius=8)).is_ok()
    cuda.cuda.synchronize()
    reserved, used = api.memory_stats()
    # the build's scratch (codes, sorted boxes, binary nodes, collapse lists) was freed but is kept
    assert reserved - used > (64 << 20) and used > 0
    first = api.bvh_host_arrays(bvh)
    # building again reuses the retained memory and gives the same tree
    bvh2 = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh2, g.gwn_bvh_build_options(method=0, hploc_search_radius=8)).is_ok()
    again = api.bvh_host_arrays(bvh2)
    np.testing.assert_array_equal(first["nodes"], again["nodes"])
    np.testing.assert_array_equal(first["primitive_indices"], again["primitive_indices"])
    # freed objects leave whole pool chunks unused; a trim hands them back to the driver
    bvh2.clear()
    bvh.clear()
    geo.clear()
    cuda.cuda.synchronize()
    reserved3, used3 = api.memory_stats()
    assert used3 < used and reserved3 >= reserved
    assert api.memory_trim(0).is_ok()
    reserved4, used4 = api.memory_stats()
    assert used4 == used3 and reserved4 < reserved3
    # and work after a trim is unaffected
    geo = upload(meshes.soup_mesh(30, seed=2))
    assert g.gwn_build_bvh(geo, bvh).is_ok()


def test_launch_counter_counts_library_kernels(cuda):
    """gwnb_launch_count moves by exactly the kernels a call issues: one traversal for a Taylor
    batch in input order; query codes, the radix sort (histogram and four 8-bit passes over the
    30-bit codes), the gather of the queries into that order and the traversal for an ordered
    batch; nothing for a rejected call."""
    mesh = meshes.soup_mesh(40, seed=6)
    geo = upload(mesh)
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    mom = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, 5000, seed=1)]
    out = cuda.empty_like(q[0])
    c0 = api.launch_count()
    assert g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, *q, out, sort_queries=False).is_ok()
    c1 = api.launch_count()
    assert g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, *q, out, sort_queries=True).is_ok()
    c2 = api.launch_count()
    stale = g.gwn_bvh4_moment_object(1)
    assert not g.gwn_compute_winding_number_taylor_batch(1, bvh, stale, *q, out).is_ok()
    c3 = api.launch_count()
    assert (c1 - c0, c2 - c1, c3 - c2) == (1, 8, 0)
