"""The C ABI library loads, exports every symbol include/gwnb.h declares, and rejects invalid
arguments before touching the GPU (CPU only: no kernel is launched here).

Argument checks restate smallgwn's contract tests: invalid build method and H-PLOC radius 0 / 9
(tests/unit_gwn_bvh.cu:289-358), empty BVH / stale moment / negative or NaN accuracy scale and span
mismatches (tests/unit_gwn_query_winding.cu:245-313).
"""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from smallgwn_b200 import _lib, api

HEADER = Path(__file__).resolve().parents[1] / "include" / "gwnb.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"GWNB_API[^;(]*?\b(gwnb_\w+)\s*\(", text))


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.library_path())], capture_output=True, text=True)
    exported = set(re.findall(r" T (gwnb_\w+)", out.stdout))
    assert names <= exported
    assert set(_lib.SIGNATURES) == names


def test_library_reports_version():
    assert b"sm_100a" in _lib.load().gwnb_version()


def test_structure_sizes_match_the_reference_layout():
    assert C.sizeof(_lib.child_f32) == 32
    assert C.sizeof(_lib.node4_f32) == 128
    assert C.sizeof(_lib.triangle_f32) == 36
    for order, fields in ((0, 7), (1, 13), (2, 23)):
        assert _lib.load().gwnb_moment_node_bytes(order) == fields * 16


def test_build_rejects_bad_options_without_gpu():
    lib = _lib.load()
    g = _lib.geometry_f32()
    out = _lib.bvh4_f32()
    assert lib.gwnb_bvh4_build_f32(C.byref(g), 7, 8, 64, C.byref(out), None) == _lib.GWNB_INVALID_ARGUMENT
    assert "method" in _lib.last_error()
    for radius in (0, 9):
        assert lib.gwnb_bvh4_build_f32(C.byref(g), 0, radius, 64, C.byref(out), None) == _lib.GWNB_INVALID_ARGUMENT
        assert "radius" in _lib.last_error()
    assert lib.gwnb_bvh4_build_f32(C.byref(g), 1, 8, 16, C.byref(out), None) == _lib.GWNB_INVALID_ARGUMENT


def test_python_mirror_rejects_bad_options_and_keeps_object():
    geo = api.gwn_geometry_object()
    bvh = api.gwn_bvh4_object()
    st = api.gwn_build_bvh(geo, bvh, api.gwn_bvh_build_options(method=0, hploc_search_radius=9))
    assert st.error == api.gwn_error.invalid_argument and not bvh.has_data()
    st = api.gwn_upload_geometry(geo, [0, 1], [0, 1, 2], [0, 1], [0], [1], [2])
    assert st.error == api.gwn_error.invalid_argument and not geo.has_data()


def test_queries_reject_invalid_state_without_gpu():
    lib = _lib.load()
    empty = _lib.bvh4_f32()
    mom = _lib.moment4_f32()
    assert lib.gwnb_winding_exact_batch_f32(C.byref(empty), None, None, None, None, 0, 256, None) == \
        _lib.GWNB_INVALID_ARGUMENT
    assert "no queryable data" in _lib.last_error()
    assert lib.gwnb_winding_taylor_batch_f32(C.byref(empty), C.byref(mom), None, None, None, None, 0, 2.0, None,
                                             None) == _lib.GWNB_INVALID_ARGUMENT
    # a syntactically valid leaf-root view (host pointers never dereferenced) with a stale moment
    fake = _lib.bvh4_f32()
    fake.primitive_count = 1
    fake.primitive_indices = 8
    fake.triangles = 8
    fake.revision = 5
    fake.root.reference = (1 << 47) | (1 << 48)
    stale = _lib.moment4_f32(order=0, bvh_revision=4)
    assert lib.gwnb_winding_taylor_batch_f32(C.byref(fake), C.byref(stale), None, None, None, None, 0, 2.0, None,
                                             None) == _lib.GWNB_INVALID_ARGUMENT
    assert "not aligned" in _lib.last_error()
    fresh = _lib.moment4_f32(order=0, bvh_revision=5)
    for beta in (-1.0, float("nan")):
        assert lib.gwnb_winding_taylor_batch_f32(C.byref(fake), C.byref(fresh), None, None, None, None, 0, beta,
                                                 None, None) == _lib.GWNB_INVALID_ARGUMENT
        assert "accuracy scale" in _lib.last_error()
    # non-empty batch with null storage
    assert lib.gwnb_winding_exact_batch_f32(C.byref(fake), None, None, None, None, 3, 256, None) == \
        _lib.GWNB_INVALID_ARGUMENT
    assert "non-null storage" in _lib.last_error()
    # an unknown traversal value
    bad_walk = _lib.taylor_options(256, 64, 1, 0, 1.0 / 16.0, 7)
    assert lib.gwnb_winding_taylor_batch_f32(C.byref(fake), C.byref(fresh), None, None, None, None, 0, 2.0,
                                             C.byref(bad_walk), None) == _lib.GWNB_INVALID_ARGUMENT
    assert "Unknown traversal" in _lib.last_error()
    beyond = _lib.taylor_options(256, 64, 1, 0, 1.0 / 16.0, _lib.GWNB_WALK_TIMED + 1)
    assert lib.gwnb_winding_taylor_batch_f32(C.byref(fake), C.byref(fresh), None, None, None, None, 0, 2.0,
                                             C.byref(beyond), None) == _lib.GWNB_INVALID_ARGUMENT
    assert "Unknown traversal" in _lib.last_error()


def test_stack_capacity_below_bound_is_rejected():
    lib = _lib.load()
    fake = _lib.bvh4_f32()
    fake.nodes = 8
    fake.node_count = 3
    fake.primitive_count = 9
    fake.primitive_indices = 8
    fake.triangles = 8
    fake.revision = 5
    fake.internal_stack_bound = 2
    fake.root.reference = 1 << 47
    mom = _lib.moment4_f32(order=1, bvh_revision=5, node_count=3, nodes=8, aux=8)
    opt = _lib.taylor_options(256, 1, 1, 0, 1e-3)
    rc = lib.gwnb_winding_taylor_batch_f32(C.byref(fake), C.byref(mom), None, None, None, None, 0, 2.0,
                                           C.byref(opt), None)
    assert rc == _lib.GWNB_INVALID_ARGUMENT
    assert "Traversal stack capacity" in _lib.last_error()


def test_adjoint_pair_validation():
    """The Taylor forward / backward pair refuses bad calls on the host, before any device work."""
    lib = _lib.load()
    fake = _lib.bvh4_f32()
    fake.nodes = 8
    fake.node_count = 3
    fake.primitive_count = 9
    fake.primitive_indices = 8
    fake.triangles = 8
    fake.revision = 5
    fake.internal_stack_bound = 2
    fake.root.reference = 1 << 47
    mom1 = _lib.moment4_f32(order=1, bvh_revision=5, node_count=3, nodes=8, aux=8)
    mom2 = _lib.moment4_f32(order=2, bvh_revision=5, node_count=3, nodes=8, aux=8)
    saved = _lib.taylor_saved_f32()
    # no saved state
    assert lib.gwnb_winding_taylor_forward_f32(C.byref(fake), C.byref(mom1), None, None, None, None, 0, 2.0, None,
                                               None, None) == _lib.GWNB_INVALID_ARGUMENT
    assert "saved state" in _lib.last_error()
    # order 2 has no adjoint
    assert lib.gwnb_winding_taylor_forward_f32(C.byref(fake), C.byref(mom2), None, None, None, None, 0, 2.0, None,
                                               C.byref(saved), None) == _lib.GWNB_INVALID_ARGUMENT
    assert "orders 0 and 1" in _lib.last_error()
    assert lib.gwnb_winding_taylor_backward_f32(None, None, C.byref(fake), C.byref(mom1), None, None, None, None,
                                                None, None, None, None) == _lib.GWNB_INVALID_ARGUMENT
    saved.order = 2
    assert lib.gwnb_winding_taylor_backward_f32(C.byref(saved), None, C.byref(fake), C.byref(mom1), None, None,
                                                None, None, None, None, None, None) == _lib.GWNB_INVALID_ARGUMENT
    assert "orders 0 and 1" in _lib.last_error()
    # the BVH must be at the forward pass's revision
    saved.order = 1
    saved.bvh_revision = 4
    assert lib.gwnb_winding_taylor_backward_f32(C.byref(saved), None, C.byref(fake), C.byref(mom1), None, None,
                                                None, None, None, None, None, None) == _lib.GWNB_INVALID_ARGUMENT
    assert "changed since the forward pass" in _lib.last_error()
    # partial output triples are refused
    saved.bvh_revision = 5
    assert lib.gwnb_winding_taylor_backward_f32(C.byref(saved), None, C.byref(fake), C.byref(mom1), None, 8, None,
                                                None, None, None, None, None) == _lib.GWNB_INVALID_ARGUMENT
    assert "all null or all non-null" in _lib.last_error()


def test_spatial_batches_reject_invalid_contracts_before_launch():
    """Distance and ray batches: empty BVH, capacity below the bound, t_max < t_min and null
    storage are refused on the host (tests/unit_gwn_query_distance_ray.cu:563-640)."""
    lib = _lib.load()
    empty = _lib.bvh4_f32()
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(empty), None, None, None, None, 0, float("inf"), None,
                                                None) == _lib.GWNB_INVALID_ARGUMENT
    assert "no queryable data" in _lib.last_error()
    assert lib.gwnb_ray_first_hit_batch_f32(C.byref(empty), None, None, None, None, None, None, None, 0, 0.0,
                                            float("inf"), None, None) == _lib.GWNB_INVALID_ARGUMENT
    fake = _lib.bvh4_f32()
    fake.nodes = 8
    fake.node_count = 3
    fake.primitive_count = 9
    fake.primitive_indices = 8
    fake.triangles = 8
    fake.revision = 5
    fake.internal_stack_bound = 2
    fake.root.reference = 1 << 47
    one = _lib.spatial_options(256, 1, 0)
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(fake), None, None, None, None, 0, 1.0, C.byref(one),
                                                None) == _lib.GWNB_INVALID_ARGUMENT
    assert "Traversal stack capacity" in _lib.last_error()
    assert lib.gwnb_ray_first_hit_batch_f32(C.byref(fake), None, None, None, None, None, None, None, 0, 0.0, 1.0,
                                            C.byref(one), None) == _lib.GWNB_INVALID_ARGUMENT
    assert "Traversal stack capacity" in _lib.last_error()
    # an unknown distance walk is refused
    walk = _lib.spatial_options(256, 64, 1, _lib.GWNB_WALK_TIMED + 1)
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(fake), None, None, None, None, 0, 1.0, C.byref(walk),
                                                None) == _lib.GWNB_INVALID_ARGUMENT
    assert "Unknown traversal" in _lib.last_error()
    # empty batches with a valid capacity are accepted; t_max < t_min (or NaN) is not
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(fake), None, None, None, None, 0, 1.0, None, None) == 0
    assert lib.gwnb_ray_first_hit_batch_f32(C.byref(fake), None, None, None, None, None, None, None, 0, 0.0, 1.0,
                                            None, None) == 0
    for t_min, t_max in ((2.0, 1.0), (0.0, float("nan"))):
        assert lib.gwnb_ray_first_hit_batch_f32(C.byref(fake), None, None, None, None, None, None, None, 0, t_min,
                                                t_max, None, None) == _lib.GWNB_INVALID_ARGUMENT
        assert "t_max >= t_min" in _lib.last_error()
    # non-empty batches with null storage
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(fake), None, None, None, None, 1, 1.0, None,
                                                None) == _lib.GWNB_INVALID_ARGUMENT
    assert lib.gwnb_ray_first_hit_batch_f32(C.byref(fake), 8, None, None, None, None, None, None, 1, 0.0, 1.0,
                                            None, None) == _lib.GWNB_INVALID_ARGUMENT
    assert "non-null storage" in _lib.last_error()
    # a leaf root needs no stack: capacity 1 is accepted
    leaf = _lib.bvh4_f32()
    leaf.primitive_count = 1
    leaf.primitive_indices = 8
    leaf.triangles = 8
    leaf.revision = 5
    leaf.root.reference = (1 << 47) | (1 << 48)
    assert lib.gwnb_unsigned_distance_batch_f32(C.byref(leaf), None, None, None, None, 0, 1.0, C.byref(one),
                                                None) == 0
    assert C.sizeof(_lib.ray_hit_f32) == 32 and api.RAY_HIT_DTYPE.itemsize == 32


def test_spatial_python_mirror_rejects_span_mismatch():
    import torch
    bvh = api.gwn_bvh4_object()
    st = api.gwn_compute_unsigned_distance_batch(bvh, None, None, None, None)
    assert st.error == api.gwn_error.invalid_argument and "no queryable data" in st.message
    st = api.gwn_compute_ray_first_hit_batch(bvh, None, None, None, None, None, None, None)
    assert st.error == api.gwn_error.invalid_argument
    hits = torch.zeros((2, 8), dtype=torch.int32)
    recs = api.ray_hit_records(hits)
    assert recs.shape == (2,) and recs.dtype == api.RAY_HIT_DTYPE


def test_status_mirror():
    assert api.gwn_status().is_ok()
    assert not api.gwn_status(api.gwn_error.internal_error, "x").is_ok()


def test_allocation_failure_injection_arms_and_disarms():
    """gwnb_fail_allocation_after returns the previously armed count and -1 once disarmed (host
    only; the GPU sweep over every entry point is in test_gpu_alloc_failure.py)."""
    lib = _lib.load()
    assert lib.gwnb_fail_allocation_after(-1) == -1
    assert lib.gwnb_fail_allocation_after(5) == -1
    assert lib.gwnb_fail_allocation_after(2) == 5
    assert lib.gwnb_fail_allocation_after(-7) == 2
    assert lib.gwnb_fail_allocation_after(-1) == -1
