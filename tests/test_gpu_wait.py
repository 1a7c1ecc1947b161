"""Bounded device waits: the error path that replaces a hang.

smallgwn's BVH4 collapse spins on its work queue without a limit
(detail/gwn_bvh_build_collapse.cuh:142-144); the radix sort it calls (CUB onesweep) waits on
predecessor tiles the same way. Here every device-side wait -- the decoupled look-back of the radix
sort and of the level-synchronous collapse -- gives up after a number of polls (gwnb_set_wait_limit),
sets a timeout bit and lets the launch complete. The test makes each wait run out on purpose, on a
predecessor tile that nothing publishes (gwnb_wait_timeout_probe, a few microseconds at a limit of
1,000 polls): the call returns GWNB_INTERNAL_ERROR with the timeout, the context stays usable, and a
normal build afterwards is bit-identical to the oracle's. No GPU fault and no unbounded wait are
involved.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from smallgwn_b200 import _lib, api, meshes
from test_gpu_build import build, upload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("stage", [0, 1], ids=["radix_sort", "collapse"])
def test_wait_runs_out_then_build_recovers(cuda, stage):
    lib = _lib.load()
    assert lib.gwnb_set_wait_limit(1000) == _lib.GWNB_OK
    try:
        rc = lib.gwnb_wait_timeout_probe(stage, None)
        assert rc == _lib.GWNB_INTERNAL_ERROR
        assert "timed out" in _lib.last_error()
    finally:
        assert lib.gwnb_set_wait_limit(0) == _lib.GWNB_OK
    cuda.cuda.synchronize()
    # the context is intact: a multi-tile build (10,240 triangles, 3 sort tiles) matches the oracle
    mesh = meshes.to_soa(*meshes.uv_sphere(80, 65, seed=3))
    bvh = build(upload(mesh))
    h = api.bvh_host_arrays(bvh)
    ob = oracle.build_lbvh(mesh, 64)
    np.testing.assert_array_equal(h["primitive_indices"], ob["sorted_ids"])
    np.testing.assert_array_equal(h["nodes"]["reference"], ob["nodes"]["reference"])


def test_probe_rejects_unknown_stage(cuda):
    assert _lib.load().gwnb_wait_timeout_probe(7, None) == _lib.GWNB_INVALID_ARGUMENT
