"""The benchmark's own sizes (1,046,528-triangle displaced sphere, 10M mixed queries, order 2 at
accuracy scale 3.5), checked through properties that hold at any size:

- the sphere is star-shaped about the origin and closed apart from its pole points, which lie on
  the z axis (the missing caps have zero area), so away from the surface and from the axis the
  winding number is the inside indicator |q| < r(theta, phi): every such query is within the
  headline's 1e-3 of it;
- each query's traversal does not depend on its warp mates, so the batch's output is bit-identical
  whether it orders the queries internally or not, and the warp-cooperative and per-thread
  traversals agree bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import api, meshes
from test_gpu_build import upload
from test_gpu_query import assert_agree_or_explained

pytestmark = pytest.mark.gpu

ORDER, BETA, N = 2, 3.5, 10_000_000


@pytest.fixture(scope="module")
def scene(cuda):
    mesh = meshes.sphere_mesh()
    geo = upload(mesh)
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=0, hploc_search_radius=8)).is_ok()
    mom = g.gwn_bvh4_moment_object(ORDER)
    assert g.gwn_refit_bvh_moment(ORDER, bvh, mom).is_ok()
    q = meshes.mixed_queries(mesh, N, seed=2)
    dq = [cuda.from_numpy(v).cuda() for v in q]
    return geo, bvh, mom, q, dq


def taylor(cuda, scene, **kw):
    _, bvh, mom, _, dq = scene
    out = cuda.empty_like(dq[0])
    st = g.gwn_compute_winding_number_taylor_batch(ORDER, bvh, mom, *dq, out, accuracy_scale=BETA, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out


def test_inside_indicator_at_full_size(cuda, scene):
    _, _, _, q, _ = scene
    w = taylor(cuda, scene, precision=g.near_precision.compensated).cpu().numpy().astype(np.float64)
    x, y, z = (v.astype(np.float64) for v in q)
    rho = np.hypot(x, y)
    rad = np.sqrt(x * x + y * y + z * z)
    r = meshes.displaced_radius(np.arctan2(rho, z), np.arctan2(y, x), seed=2)
    # the faceted surface stays within ~1e-4 of r(theta, phi) on this grid; keep 2e-3 clear of
    # it (in radius) and of the z axis that holds the pole points
    clear = (np.abs(rad - r) > 2e-3) & (rho > 2e-3)
    assert clear.sum() > 0.5 * N  # the uniform half and the far tail of the near-surface half
    inside = (rad < r).astype(np.float64)
    err = np.abs(w[clear] - inside[clear])
    assert np.isfinite(w).all()
    assert err.max() <= 1e-3, (err.max(), np.quantile(err, 0.99))
    assert 0.2 < inside[clear].mean() < 0.8  # both classes are well represented


def test_ordering_and_traversal_forms_agree_bit_for_bit(cuda, scene):
    for prec in (g.near_precision.plain, g.near_precision.compensated):
        ordered = taylor(cuda, scene, precision=prec, sort_queries=True)
        unordered = taylor(cuda, scene, precision=prec, sort_queries=False)
        assert cuda.equal(ordered, unordered)
    per_thread = taylor(cuda, scene, precision=g.near_precision.plain, sort_queries=True, per_thread=True)
    warp = taylor(cuda, scene, precision=g.near_precision.plain, sort_queries=True)
    assert cuda.equal(per_thread, warp)


@pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's own kernels (oracle/_ref) not built")
@pytest.mark.parametrize("order", [1, 2])
def test_taylor_matches_reference_kernel_at_size(cuda, order):
    """smallgwn's Taylor batch on the benchmark sphere (its own LBVH and moments, equal to ours up to
    node numbering), accuracy scale 2 as the Taylor-at-scale workload prescribes, 20,000 of its mixed
    queries: every query agrees within 1e-5 + 2e-5 |w|, or the disagreement is explained in FP64 by
    an acceptance test that decides differently under the two moment sets (or sits within rounding
    of its threshold), or by a near-field triangle seen along an edge's line. The max / p99
    difference over all queries and both implementations' errors against FP64 are printed."""
    mesh = meshes.sphere_mesh()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(upload(mesh), bvh, g.gwn_bvh_build_options(method=1)).is_ok()
    mom = g.gwn_bvh4_moment_object(order)
    assert g.gwn_refit_bvh_moment(order, bvh, mom).is_ok()
    R = oracle.Reference(mesh)
    try:
        R.build(1, 8, 64)
        h = api.bvh_host_arrays(bvh)
        rb = R.bvh()
        pairing = oracle.match_wide_nodes(h["nodes"], h["root_reference"], rb["nodes"], rb["root_reference"])
        q = meshes.mixed_queries(mesh, 20_000, seed=2)
        R.refit_moments(order)
        theirs = R.taylor(order, *q, beta=2.0)
        d = [cuda.from_numpy(v).cuda() for v in q]
        out = cuda.empty_like(d[0])
        assert g.gwn_compute_winding_number_taylor_batch(order, bvh, mom, *d, out, accuracy_scale=2.0).is_ok()
        cuda.cuda.synchronize()
        ours = out.cpu().numpy()
        rep = assert_agree_or_explained(ours, theirs, q, h, api.moment_host_array(mom), R.moments(order), pairing,
                                        2.0, allow=("decision", "conditioning", "moments"))
        # order 2: the recentred third moments cancel in FP32 for small nodes far from the origin,
        # so the two climbs' summation orders alone move many queries by up to a few 1e-4 (all of
        # them explained above); what must hold is that neither side is the less accurate one
        print(f"order {order}: {rep['outside'].size} of {ours.size} queries outside 1e-5 + 2e-5 |w|, "
              f"reasons {rep['reasons']}")
        sub = slice(0, 2000)
        ref64 = oracle.exact_winding(mesh, *[v[sub] for v in q], fp64=True)
        e_ours, e_theirs = np.abs(ours[sub] - ref64), np.abs(theirs[sub] - ref64)
        print(f"order {order}: error vs FP64 ours max {e_ours.max():.3e} p99 {np.quantile(e_ours, 0.99):.3e}; "
              f"smallgwn max {e_theirs.max():.3e} p99 {np.quantile(e_theirs, 0.99):.3e}")
        assert np.quantile(e_ours, 0.99) <= 1.25 * np.quantile(e_theirs, 0.99) + 1e-6
        assert e_ours.max() <= 1.25 * e_theirs.max() + 1e-6
    finally:
        R.close()
