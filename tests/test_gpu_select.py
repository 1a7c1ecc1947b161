"""Taylor order and accuracy scale chosen from an error target (gwnb_taylor_select_f32).

On a sample of the caller's queries, against their FP64 exact winding numbers: the choice meets the
bound on the sample, its order's next smaller candidate accuracy scale does not (the smallest
passing scale per order is each order's candidate), the stack capacity is the tree's bound, and the
choice carries over to other queries of the same distribution (within 2x the bound on a disjoint
set). An unreachable bound is refused.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import api, meshes
from test_gpu_build import build, upload

pytestmark = pytest.mark.gpu

SCALES = (1.0, 1.5, 2.0, 2.5, 3.0, 3.25, 3.5, 4.0, 5.0, 6.0, 8.0)


def test_select_meets_the_bound_with_the_smallest_scale(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(128, 64, seed=5))
    geo = upload(mesh)
    bvh = build(geo, g.gwn_bvh_build_method.k_hploc)
    moms = {}
    for o in (0, 1, 2):
        moms[o] = g.gwn_bvh4_moment_object(o)
        assert g.gwn_refit_bvh_moment(o, bvh, moms[o]).is_ok()
    q = meshes.mixed_queries(mesh, 30_000, seed=44)
    sample = [cuda.from_numpy(v[:20_000].copy()).cuda() for v in q]
    st, choice = api.select_taylor_form(geo, bvh, moms, *sample, max_error=1e-3, accuracy_scales=SCALES)
    assert st.is_ok(), st.message
    assert choice["order"] in (0, 1, 2) and choice["max_error"] <= 1e-3 and choice["candidates_passing"] >= 1
    assert choice["stack_capacity"] == bvh.accessor().internal_stack_bound
    ref = oracle.exact_winding(mesh, *[v[:20_000] for v in q], fp64=True)

    def err(order, beta, qs, r):
        d = [cuda.from_numpy(v.copy()).cuda() for v in qs]
        out = cuda.empty_like(d[0])
        assert g.gwn_compute_winding_number_taylor_batch(order, bvh, moms[order], *d, out, accuracy_scale=beta,
                                                         precision=g.near_precision.compensated).is_ok()
        cuda.cuda.synchronize()
        return float(np.abs(out.cpu().numpy() - r).max())

    o, b = choice["order"], choice["accuracy_scale"]
    assert err(o, b, [v[:20_000] for v in q], ref) == pytest.approx(choice["max_error"], rel=1e-6, abs=1e-9)
    smaller = [s for s in SCALES if s < b]
    if smaller:
        assert err(o, smaller[-1], [v[:20_000] for v in q], ref) > 1e-3
    held_out = [v[20_000:] for v in q]
    assert err(o, b, held_out, oracle.exact_winding(mesh, *held_out, fp64=True)) <= 2e-3
    st, _ = api.select_taylor_form(geo, bvh, moms, *sample, max_error=1e-9, accuracy_scales=(1.0, 2.0))
    assert st.error == g.gwn_error.invalid_argument
