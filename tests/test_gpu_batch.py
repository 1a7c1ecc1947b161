"""GPU checks of the batched dynamic-mesh frame (gwnb_batch_*).

A frame refits every BVH and its moments and evaluates every mesh's Taylor queries in three
persistent launches. Each mesh's results must equal the per-mesh path -- gwn_refit_bvh,
gwn_refit_bvh_moment and gwn_compute_winding_number_taylor_batch -- on the same deformed vertices:
the batched kernels run the same per-item code with the same summation orders.
"""
from __future__ import annotations

import numpy as np
import pytest

import smallgwn_b200 as g
from smallgwn_b200 import api, meshes

pytestmark = pytest.mark.gpu

ORDER = 1
BETA = 2.0


def make_batch(cuda, sizes, seed=4):
    """Meshes (uv spheres, a soup, a single triangle) in one shared vertex buffer."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, n in enumerate(sizes):
        if n == 0:
            V = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
            F = np.array([[0, 1, 2]])
        elif k % 3 == 2:
            m = meshes.soup_mesh(n, seed=k)
            V = np.stack([m["x"], m["y"], m["z"]], -1)
            F = np.stack([m["i0"], m["i1"], m["i2"]], -1)
        else:
            V, F = meshes.uv_sphere(2 * n, n, seed=10 + k)
        parts.append((V.astype(np.float32) + rng.uniform(-3, 3, size=3).astype(np.float32), F.astype(np.int32)))
    nv = sum(p[0].shape[0] for p in parts)
    X = cuda.empty(3, nv, device="cuda")
    objs = []
    off = 0
    for k, (V, F) in enumerate(parts):
        n = V.shape[0]
        X[:, off:off + n] = cuda.from_numpy(V.T.copy()).cuda()
        idx = [cuda.from_numpy(np.ascontiguousarray(F[:, j])).cuda() for j in range(3)]
        geo = api.gwn_geometry_view(X[0, off:off + n], X[1, off:off + n], X[2, off:off + n], *idx)
        bvh = g.gwn_bvh4_object()
        method = g.gwn_bvh_build_method.k_lbvh if k % 2 else g.gwn_bvh_build_method.k_hploc
        assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=method)).is_ok()
        mom = g.gwn_bvh4_moment_object(ORDER)
        assert g.gwn_refit_bvh_moment(ORDER, bvh, mom).is_ok()
        mesh = {"x": V[:, 0], "y": V[:, 1], "z": V[:, 2], "i0": F[:, 0], "i1": F[:, 1], "i2": F[:, 2]}
        nq = int(rng.integers(500, 6000))
        q = meshes.mixed_queries(mesh, nq, seed=100 + k)
        dq = [cuda.from_numpy(v).cuda() for v in q]
        out = cuda.empty(nq, device="cuda")
        objs.append((geo, bvh, mom, *dq, out))
        off += n
    return X, objs


def per_mesh(cuda, objs, refit: bool):
    """The per-mesh path of plain calls. With refit, the BVH is refit in place and the moments go to a
    moment object of its own: the batch's moment objects stay the ones it was made over."""
    res = []
    for geo, bvh, mom, qx, qy, qz, _ in objs:
        if refit:
            assert g.gwn_refit_bvh(geo, bvh).is_ok()
            mom = g.gwn_bvh4_moment_object(ORDER)
            assert g.gwn_refit_bvh_moment(ORDER, bvh, mom).is_ok()
        o = cuda.empty_like(qx)
        assert g.gwn_compute_winding_number_taylor_batch(ORDER, bvh, mom, qx, qy, qz, o, accuracy_scale=BETA).is_ok()
        res.append(o)
    cuda.cuda.synchronize()
    return [r.cpu().numpy() for r in res]


def outputs(cuda, objs):
    cuda.cuda.synchronize()
    return [o[-1].cpu().numpy() for o in objs]


def deform(X, f):
    # a smooth displacement along a fixed direction field, like the batched benchmark's
    X += 0.02 * cuda_sin(2 * np.pi * f / 10 + X.sum(0, keepdim=True)) * 0.5


def cuda_sin(t):
    return t.sin()


SIZES = [24, 40, 12, 64, 0, 31, 17, 48, 20]


def test_batched_frame_equals_per_mesh_calls(cuda):
    X, objs = make_batch(cuda, SIZES)
    batch = g.gwn_batch(objs, accuracy_scale=BETA)
    assert batch.ok(), batch.status.message
    assert batch.frame().is_ok()
    assert batch.sync().is_ok()
    first = outputs(cuda, objs)
    for a, b in zip(first, per_mesh(cuda, objs, refit=False)):
        np.testing.assert_array_equal(a, b)
    # move the vertices: the batched refit + moments + query equal the per-mesh path
    deform(X, 1)
    assert batch.frame().is_ok()
    assert batch.sync().is_ok()
    second = outputs(cuda, objs)
    assert any(np.max(np.abs(a - b)) > 1e-4 for a, b in zip(first, second))
    for a, b in zip(second, per_mesh(cuda, objs, refit=True)):
        np.testing.assert_array_equal(a, b)
    batch.release()


def test_autotuned_and_graph_captured_frames(cuda):
    X, objs = make_batch(cuda, SIZES, seed=7)
    batch = g.gwn_batch(objs, accuracy_scale=BETA)
    assert batch.ok(), batch.status.message
    st, chosen = batch.tune(repetitions=1)
    assert st.is_ok(), st.message
    assert chosen["frame_ms"] > 0 and chosen["query_block"] in (128, 256)
    deform(X, 2)
    s = cuda.cuda.Stream()
    s.wait_stream(cuda.cuda.current_stream())
    graph = cuda.cuda.CUDAGraph()
    with cuda.cuda.stream(s):
        assert batch.frame(s.cuda_stream).is_ok()  # outside capture first
        s.synchronize()
        with cuda.cuda.graph(graph, stream=s):
            deform(X, 3)
            assert batch.frame(s.cuda_stream).is_ok()
    graph.replay()
    cuda.cuda.synchronize()
    assert batch.sync().is_ok()
    got = outputs(cuda, objs)
    for a, b in zip(got, per_mesh(cuda, objs, refit=True)):
        np.testing.assert_array_equal(a, b)
    # every tuned shape computes the same numbers
    for shape in ((128, 128, 1, 1, 4), (256, 256, 0, 0, 16), (128, 64, 0, 1, 1)):
        assert batch.set_tuning(*shape).is_ok()
        assert batch.frame().is_ok()
        other = outputs(cuda, objs)
        for a, b in zip(other, got):
            np.testing.assert_allclose(a, b, atol=2e-6)
    del graph
    batch.release()


def test_batch_rejects_bad_meshes(cuda):
    X, objs = make_batch(cuda, [12, 16])
    geo, bvh, mom, qx, qy, qz, out = objs[1]
    m0 = g.gwn_bvh4_moment_object(0)
    assert g.gwn_refit_bvh_moment(0, bvh, m0).is_ok()
    bad = g.gwn_batch([objs[0], (geo, bvh, m0, qx, qy, qz, out)])
    assert bad.status.error == g.gwn_error.invalid_argument and "order" in bad.status.message
    assert g.gwn_batch([], accuracy_scale=BETA).status.error == g.gwn_error.invalid_argument


def test_quality_driven_rebuild(cuda):
    """Refit trees keep the rest shape's topology; a deformation that scrambles a mesh raises its
    surface-area cost ratio. rebuild() rebuilds exactly the meshes past the threshold (the caller's
    objects in place), after which the frame again equals the per-mesh path on the same objects and
    the rebuilt trees' ratios are back at 1."""
    X, objs = make_batch(cuda, [24, 40, 31], seed=11)
    batch = g.gwn_batch(objs, accuracy_scale=BETA)
    assert batch.ok(), batch.status.message
    st, ratios = batch.quality()
    assert st.is_ok() and np.allclose(ratios, 1.0, atol=1e-5)
    # scramble the second mesh: every vertex moves to another vertex's position (mirrored in x)
    n0 = objs[0][0].vertex_count()
    n1 = objs[1][0].vertex_count()
    perm = cuda.from_numpy(np.random.default_rng(3).permutation(n1)).cuda()
    sub = X[:, n0:n0 + n1]
    X[:, n0:n0 + n1] = sub[:, perm] * cuda.tensor([[-1.0], [1.0], [1.0]], device="cuda")
    assert batch.frame().is_ok()
    st, ratios = batch.quality()
    assert st.is_ok()
    assert ratios[1] > 2.0 and abs(ratios[0] - 1.0) < 1e-5 and abs(ratios[2] - 1.0) < 1e-5
    old_revision = objs[1][1].accessor().revision
    st, n = batch.rebuild(1.5)
    assert st.is_ok(), st.message
    assert n == 1 and objs[1][1].accessor().revision != old_revision
    st, ratios = batch.quality()
    assert st.is_ok() and np.allclose(ratios, 1.0, atol=1e-5)
    assert batch.frame().is_ok()
    assert batch.sync().is_ok()
    for a, b in zip(outputs(cuda, objs), per_mesh(cuda, objs, refit=True)):
        np.testing.assert_array_equal(a, b)
    batch.release()


def test_replaced_objects_are_refused(cuda):
    """A batch's device descriptors point into the arrays of the BVH and moment objects it was made
    over. Moments refit into a new object in place of one of them (or a BVH built again) leave those
    pointers dangling: every entry point then refuses the batch with invalid_argument instead of
    launching over released arrays, and a new batch over the same objects works."""
    X, objs = make_batch(cuda, [20, 28, 16], seed=5)
    batch = g.gwn_batch(objs, accuracy_scale=BETA)
    assert batch.ok(), batch.status.message
    assert batch.frame().is_ok() and batch.sync().is_ok()
    geo, bvh, mom = objs[1][:3]
    assert g.gwn_refit_bvh_moment(ORDER, bvh, mom).is_ok()  # new moment arrays for mesh 1
    st = batch.frame()
    assert st.error == g.gwn_error.invalid_argument and "mesh 1" in st.message and "replaced" in st.message
    assert batch.run(batch.QUERY).error == g.gwn_error.invalid_argument
    assert batch.sync().error == g.gwn_error.invalid_argument
    assert batch.quality()[0].error == g.gwn_error.invalid_argument
    assert batch.rebuild(1.5)[0].error == g.gwn_error.invalid_argument
    assert batch.tune(repetitions=1)[0].error == g.gwn_error.invalid_argument
    batch.release()
    # a BVH built again is refused the same way
    fresh = g.gwn_batch(objs, accuracy_scale=BETA)
    assert fresh.ok(), fresh.status.message
    assert g.gwn_build_bvh(objs[2][0], objs[2][1], g.gwn_bvh_build_options(method=0)).is_ok()
    assert fresh.frame().error == g.gwn_error.invalid_argument
    fresh.release()
    # objects rebuilt and refit, then a new batch: frames equal the per-mesh path again
    assert g.gwn_refit_bvh_moment(ORDER, objs[2][1], objs[2][2]).is_ok()
    again = g.gwn_batch(objs, accuracy_scale=BETA)
    assert again.ok(), again.status.message
    assert again.frame().is_ok() and again.sync().is_ok()
    for a, b in zip(outputs(cuda, objs), per_mesh(cuda, objs, refit=False)):
        np.testing.assert_array_equal(a, b)
    again.release()
