"""Error paths under device-memory exhaustion, made on the host (no GPU fault).

gwnb_fail_allocation_after(k) lets the next k device allocations of the library succeed and fails
the one after as an out-of-memory allocation would. Each entry point below is run with k = 0, 1,
2, ... until a run needs no more than k allocations; every run that met the failure must
- return cuda_runtime_error with the injected failure in its message,
- leave no device memory of the call in use once its stream has drained (the library pool's
  in-use bytes return to their value before the call), and
- leave the objects it was given as they were (the strong guarantee of smallgwn's builds and
  refits, include/gwn/gwn_bvh_build.cuh:34-39, detail/gwn_bvh_build_impl.cuh:264-273), which the
  next successful call shows by returning the same results as before.
smallgwn's own fault-injection test corrupts device geometry (tests/unit_gwn_bvh.cu:487-501);
device-side corruption is covered in test_gpu_build.py, allocation failures here.
"""
from __future__ import annotations

import numpy as np
import pytest

import smallgwn_b200 as g
from smallgwn_b200 import api, meshes

pytestmark = pytest.mark.gpu


def sweep(cuda, op, after=None, limit=400) -> int:
    """Runs op() with the k-th allocation failing for k = 0, 1, ... and checks every failing run;
    `after` (if given) runs after each failing run to check the objects. Returns how many runs
    met the failure (the op's allocation count)."""
    cuda.cuda.synchronize()
    _, used0 = api.memory_stats()
    for k in range(limit):
        api.fail_allocation_after(k)
        try:
            st = op()
        finally:
            armed = api.fail_allocation_after(-1)
        cuda.cuda.synchronize()
        if armed >= 0:  # the run needed no more than k allocations
            assert st.is_ok(), (k, st.message)
            return k
        assert st.error == g.gwn_error.cuda_runtime_error and "injected" in st.message, (k, st.error, st.message)
        _, used = api.memory_stats()
        assert used == used0, f"allocation {k} failing left {used - used0} bytes in use"
        if after is not None:
            after()
    raise AssertionError("more allocations than the sweep limit")


@pytest.fixture
def scene(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(48, 25, seed=4))
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    moms = {}
    for o in (0, 1, 2):
        moms[o] = g.gwn_bvh4_moment_object(o)
        assert g.gwn_refit_bvh_moment(o, bvh, moms[o]).is_ok()
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, 5000, seed=8)]
    return mesh, geo, bvh, moms, q


def taylor(cuda, bvh, mom, q, **kw):
    out = cuda.full((q[0].numel(),), float("nan"), device="cuda")
    st = g.gwn_compute_winding_number_taylor_batch(mom.order, bvh, mom, *q, out, 2.0, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out.cpu().numpy()


def test_geometry_upload(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(32, 17, seed=2))
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    n = geo.triangle_count()
    fresh = g.gwn_geometry_object()
    count = sweep(cuda, lambda: g.gwn_upload_geometry(fresh, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"],
                                                      mesh["i2"]))
    assert count >= 1 and fresh.triangle_count() == n


@pytest.mark.parametrize("method", [g.gwn_bvh_build_method.k_hploc, g.gwn_bvh_build_method.k_lbvh])
def test_build_keeps_the_previous_tree(cuda, scene, method):
    mesh, geo, bvh, moms, q = scene
    ref = g.gwn_bvh4_object()  # the same build into another object, for the results at the end
    assert g.gwn_build_bvh(geo, ref, g.gwn_bvh_build_options(method=method)).is_ok()
    ref_mom = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, ref, ref_mom).is_ok()
    want = taylor(cuda, ref, ref_mom, q)
    before = api.bvh_host_arrays(bvh)

    def unchanged():
        got = api.bvh_host_arrays(bvh)
        for k in before:
            np.testing.assert_array_equal(got[k], before[k], err_msg=k)

    count = sweep(cuda, lambda: g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=method)), unchanged)
    assert count >= 3
    mom = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
    np.testing.assert_array_equal(taylor(cuda, bvh, mom, q), want)


def test_refit_and_moment_refit(cuda, scene):
    mesh, geo, bvh, moms, q = scene
    want = {o: taylor(cuda, bvh, moms[o], q) for o in (0, 1, 2)}
    sweep(cuda, lambda: g.gwn_refit_bvh(geo, bvh))
    for o in (0, 1, 2):
        m = g.gwn_bvh4_moment_object(o)
        sweep(cuda, lambda: g.gwn_refit_bvh_moment(o, bvh, m))
        np.testing.assert_array_equal(taylor(cuda, bvh, m, q), want[o])


@pytest.mark.parametrize("walk", ["warp", "thread"])
def test_taylor_value_and_gradient_batches(cuda, scene, walk):
    mesh, geo, bvh, moms, q = scene
    want = taylor(cuda, bvh, moms[2], q, traversal=walk)
    out = cuda.empty_like(q[0])
    assert sweep(cuda, lambda: g.gwn_compute_winding_number_taylor_batch(2, bvh, moms[2], *q, out, 2.0,
                                                                         traversal=walk)) >= 1
    grad = [cuda.empty_like(q[0]) for _ in range(3)]
    sweep(cuda, lambda: g.gwn_compute_winding_gradient_taylor_batch(1, bvh, moms[1], *q, *grad, 2.0, traversal=walk))
    np.testing.assert_array_equal(taylor(cuda, bvh, moms[2], q, traversal=walk), want)


def test_exact_distance_and_ray_batches(cuda, scene):
    mesh, geo, bvh, moms, q = scene
    out = cuda.empty_like(q[0])
    sweep(cuda, lambda: g.gwn_compute_winding_number_exact_batch(bvh, *q, out))
    sweep(cuda, lambda: g.gwn_compute_unsigned_distance_batch(bvh, *q, out))
    sweep(cuda, lambda: g.gwn_compute_unsigned_distance_batch(bvh, *q, out, sort_queries=True))
    d = [cuda.randn(q[0].numel(), device="cuda") for _ in range(3)]
    hits = cuda.empty((q[0].numel(), 8), dtype=cuda.int32, device="cuda")
    sweep(cuda, lambda: g.gwn_compute_ray_first_hit_batch(bvh, *q, *d, hits))
    sweep(cuda, lambda: g.gwn_compute_ray_first_hit_batch(bvh, *q, *d, hits, sort_queries=True))


def test_boundary_chain_and_antipodal(cuda):
    mesh = meshes.soup_mesh(24, seed=5)
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    chain = g.gwn_boundary_chain_object()
    assert g.gwn_build_boundary_chain(geo, chain).is_ok()
    rows = chain.edge_count()
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, 2000, seed=3)]
    out = cuda.empty_like(q[0])
    assert g.gwn_compute_winding_number_antipodal_batch(geo, bvh, chain, *q, out).is_ok()
    cuda.cuda.synchronize()
    want = out.cpu().numpy()
    sweep(cuda, lambda: g.gwn_build_boundary_chain(geo, chain))
    assert chain.edge_count() == rows
    sweep(cuda, lambda: g.gwn_compute_winding_number_antipodal_batch(geo, bvh, chain, *q, out))
    grad = [cuda.empty_like(q[0]) for _ in range(3)]
    sweep(cuda, lambda: g.gwn_compute_winding_gradient_antipodal_batch(geo, chain, *q, *grad))
    assert g.gwn_compute_winding_number_antipodal_batch(geo, bvh, chain, *q, out).is_ok()
    cuda.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_adjoint_and_batched_frames(cuda, scene):
    mesh, geo, bvh, moms, q = scene
    out = cuda.empty_like(q[0])
    upstream = cuda.randn(q[0].numel(), device="cuda")
    dv = [cuda.empty(geo.vertex_count(), device="cuda") for _ in range(3)]
    dq = [cuda.empty_like(q[0]) for _ in range(3)]
    saved = {}

    def forward():
        st, saved["state"] = api.gwn_winding_taylor_forward(1, bvh, moms[1], *q, out)
        return st

    sweep(cuda, forward)
    sweep(cuda, lambda: api.gwn_winding_taylor_backward(saved["state"], geo, bvh, moms[1], upstream, *dv, *dq))
    want = [v.cpu().numpy() for v in dv + dq]

    def batch():
        b = api.gwn_batch([(geo, bvh, moms[1], *q, out)])
        st = b.status
        b.release()
        return st

    sweep(cuda, batch)
    b = api.gwn_batch([(geo, bvh, moms[1], *q, out)])
    assert b.ok(), b.status.message
    sweep(cuda, lambda: b.frame())
    b.release()
    assert api.gwn_winding_taylor_backward(saved["state"], geo, bvh, moms[1], upstream, *dv, *dq).is_ok()
    cuda.cuda.synchronize()
    # dL/dV sums its per-triangle terms by atomics, in an order that changes from run to run, and
    # the terms of both signs cancel: the check is on the array's scale (a state damaged by a failed
    # call would be off by far more); dL/dq has no atomics
    for got, w in zip(dv, want[:3]):
        np.testing.assert_allclose(got.cpu().numpy(), w, rtol=1e-3, atol=1e-3 * float(np.abs(w).max()))
    for got, w in zip(dq, want[3:]):
        np.testing.assert_array_equal(got.cpu().numpy(), w)


def test_scene_files_selection_diagnostics_and_batch_upkeep(cuda, scene, tmp_path):
    mesh, geo, bvh, moms, q = scene
    path = tmp_path / "scene.gwnb"
    sweep(cuda, lambda: api.save_scene(path, geo, bvh, [moms[1], moms[2]]))
    kept = {}

    def load():
        st, *kept["objects"] = api.load_scene(path)
        return st

    sweep(cuda, load)
    sweep(cuda, lambda: api.select_taylor_form(geo, bvh, {1: moms[1], 2: moms[2]}, *q, 1e-3)[0])
    counts = [cuda.empty(q[0].numel(), dtype=cuda.int32, device="cuda") for _ in range(3)]
    sweep(cuda, lambda: api.taylor_traversal_stats(bvh, moms[2], *q, *counts))
    sweep(cuda, lambda: api.spatial_traversal_stats(bvh, *q, *counts[:2]))
    sweep(cuda, lambda: api.taylor_form_probe(bvh, moms[2], *q)[0])
    out = cuda.empty_like(q[0])
    b = api.gwn_batch([(geo, bvh, moms[1], *q, out)])
    assert b.ok(), b.status.message
    sweep(cuda, lambda: b.tune(1)[0])
    b.release()


def test_batch_rebuild_under_allocation_failure(cuda):
    """A rebuild that fails part-way keeps what it finished (a mesh whose new tree and moments are
    both in place has them), so device memory is not expected back; instead the batch must either
    run frames or refuse them with an error until a later rebuild completes -- never launch over
    incomplete descriptors."""
    mesh = meshes.to_soa(*meshes.uv_sphere(40, 21, seed=6))
    rng = np.random.default_rng(1)
    moved = [(mesh[k] + rng.normal(0.0, 0.5, mesh[k].size)).astype(np.float32) for k in ("x", "y", "z")]
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, 3000, seed=2)]
    out = cuda.empty_like(q[0])
    refused = 0
    for k in range(400):
        geo = g.gwn_geometry_object()
        assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
        bvh = g.gwn_bvh4_object()
        assert g.gwn_build_bvh(geo, bvh).is_ok()
        mom = g.gwn_bvh4_moment_object(1)
        assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
        b = api.gwn_batch([(geo, bvh, mom, *q, out)])
        assert b.ok(), b.status.message
        # scrambled vertices push the refit tree's cost ratio past 1, so the mesh is rebuilt
        assert g.gwn_update_geometry(geo, *moved).is_ok() and b.frame().is_ok()
        api.fail_allocation_after(k)
        try:
            st, _ = b.rebuild(1.0)
        finally:
            armed = api.fail_allocation_after(-1)
        cuda.cuda.synchronize()
        if armed >= 0:  # the rebuild needed no more than k allocations
            assert st.is_ok(), st.message
            assert b.frame().is_ok() and b.sync().is_ok()
            b.release()
            assert k >= 5 and refused >= 1
            return
        assert st.error == g.gwn_error.cuda_runtime_error and "injected" in st.message, (k, st.message)
        fr = b.frame()
        if not fr.is_ok():
            assert fr.error == g.gwn_error.internal_error and "incomplete" in fr.message, (k, fr.message)
            refused += 1
            st, _ = b.rebuild(1.0)  # finishes what the failed rebuild left
            assert st.is_ok(), st.message
            assert b.frame().is_ok()
        cuda.cuda.synchronize()
        b.release()
    raise AssertionError("more allocations than the sweep limit")
