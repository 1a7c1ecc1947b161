"""The benchmark-stage harness on the GPU: every stage of smallgwn's harness runs through this
library's public API on a small mesh and writes its row (the two antipodal halves that this library
evaluates in one kernel are written as unavailable with the reason), and the stage outputs are the
library's own results (the Taylor stage's output equals a direct call)."""
from __future__ import annotations

import csv
import io

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import api, meshes, stages

pytestmark = pytest.mark.gpu


def test_all_stages_run_and_write_rows(cuda, tmp_path):
    mesh = meshes.to_soa(*meshes.uv_sphere(48, 25, seed=4))
    opts = stages.options(query_count=3000, warmup_iters=1, measure_iters=3)
    results, context = stages.run_model(mesh, opts)
    names = [r.stage for r in results]
    assert names == [s.format(builder="hploc") for s in stages.STAGES]
    for r in results:
        if r.stage in ("query_antipodal_crossings", "query_antipodal_boundary"):
            assert not r.success and r.error_message == stages.FUSED_ANTIPODAL
        else:
            assert r.success, (r.stage, r.error_message)
            assert len(r.samples_ms) == 3 and r.latency_p50_ms <= r.latency_p95_ms and r.throughput_per_s > 0
    assert 0.05 < context["ray_mix_hit_ratio"] < 0.95
    assert context["boundary_edge_count"] == oracle.boundary_chain(mesh)[0].size
    text = stages.csv_rows(results, context, "uv_sphere_48x25", opts, cuda.cuda.get_device_name(), 0, "t")
    rows = list(csv.DictReader(io.StringIO(text)))
    assert len(rows) == len(stages.STAGES) and rows[0]["stage"] == "bvh_build_hploc"


def test_winding_query_only_and_lbvh(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(32, 17, seed=2))
    opts = stages.options(query_count=2000, warmup_iters=0, measure_iters=2, builder="lbvh", winding_query_only=True)
    results, _ = stages.run_model(mesh, opts)
    assert [r.stage for r in results] == ["query_taylor_o1", "query_antipodal"] and all(r.success for r in results)


def test_reference_query_mix_on_a_closed_sphere(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(40, 21, seed=3))
    n = 2500
    q = [cuda.from_numpy(v).cuda() for v in meshes.reference_mixed_queries(mesh, n, seed=9)]
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    mom = g.gwn_bvh4_moment_object(2)
    assert g.gwn_refit_bvh_moment(2, bvh, mom).is_ok()
    out = cuda.empty(n, device="cuda")
    cfg = api.gwn_query_batch_config(stack_capacity=96)
    assert g.gwn_compute_winding_number_taylor_batch(2, bvh, mom, *q, out, 2.0, config=cfg).is_ok()
    cuda.cuda.synchronize()
    w = out.cpu().numpy()
    # the box centre of a closed sphere is inside, far-field points outside
    assert abs(w[0] - 1.0) < 1e-3
    far = (np.arange(1, n) % 10) >= 7
    assert np.all(np.abs(w[1:][far]) < 1e-2)


def test_per_thread_traversal_stage(cuda):
    mesh = meshes.to_soa(*meshes.uv_sphere(32, 17, seed=2))
    opts = stages.options(query_count=2000, warmup_iters=0, measure_iters=2, traversal="thread",
                          only=("query_taylor_o1", "query_taylor_o2"))
    results, _ = stages.run_model(mesh, opts)
    assert [r.stage for r in results] == ["query_taylor_o1", "query_taylor_o2"] and all(r.success for r in results)


def test_flushed_timing_without_per_call_synchronization(cuda):
    """The comparison timing (L2 flushed before each call, events read after the last call) runs
    the same stages as the harness timing and times every call."""
    mesh = meshes.to_soa(*meshes.uv_sphere(32, 17, seed=2))
    only = ("query_taylor_o2", "query_ray_first_hit")
    base, _ = stages.run_model(mesh, stages.options(query_count=2000, warmup_iters=1, measure_iters=3, only=only))
    res, _ = stages.run_model(mesh, stages.options(query_count=2000, warmup_iters=1, measure_iters=3, only=only,
                                                   flush_l2=True, stream_sync_per_iter=False))
    assert [r.stage for r in res] == list(only) and all(r.success for r in res + base)
    assert all(len(r.samples_ms) == 3 and min(r.samples_ms) > 0 for r in res)


def test_form_probe_matches_traversal_statistics(cuda):
    """The sample of the automatic walk choice, as a diagnostic: on a small ordered batch (128 warps,
    4 units of 32 warps, all sampled) it reads every warp's walk and its largest per-query counts;
    the per-query counts agree with the statistics entry point on the same queries."""
    mesh = meshes.to_soa(*meshes.uv_sphere(40, 21, seed=3))
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    mom = g.gwn_bvh4_moment_object(1)
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
    n = 128 * 32
    q = [cuda.from_numpy(v).cuda() for v in meshes.mixed_queries(mesh, n, seed=6)]
    order = cuda.empty(n, dtype=cuda.int32, device="cuda")
    assert api.query_order(bvh, *q, order).is_ok()
    sq = [d[order.long()].contiguous() for d in q]
    st, pr = api.taylor_form_probe(bvh, mom, *sq, accuracy_scale=2.0, sort_queries=False)
    assert st.is_ok(), st.message
    assert pr["sampled_warps"] == 128
    stats = [cuda.empty(n, dtype=cuda.int32, device="cuda") for _ in range(3)]
    assert api.taylor_traversal_stats(bvh, mom, *sq, *stats, accuracy_scale=2.0).is_ok()
    nodes = stats[0].cpu().numpy().reshape(-1, 32)
    near = stats[2].cpu().numpy().reshape(-1, 32)
    assert pr["lane_max_nodes"] == pytest.approx(nodes.max(axis=1).mean())
    assert pr["lane_max_tris"] == pytest.approx(near.max(axis=1).mean())
    assert pr["warp_nodes"] >= pr["lane_max_nodes"] > 0 and pr["warp_tris"] >= pr["lane_max_tris"]
    st, none = api.taylor_form_probe(bvh, mom, *[v[:31] for v in sq], accuracy_scale=2.0, sort_queries=False)
    assert st.is_ok() and none["sampled_warps"] == 0


@pytest.mark.parametrize("mix", ["harness", "surface"])
def test_walks_agree_and_sample_rule(cuda, mix):
    """Both walks give identical results on a batch of a few resident waves; the sampled statistics
    (units of 32 consecutive ordered warps, every k-th) carry the rule's verdict, 1 exactly when the
    sampled warps walked at least 1.3 times their longest path's nodes and that path met at most 8
    leaf triangles on average."""
    mesh = meshes.to_soa(*meshes.uv_sphere(96, 49, seed=7))
    n = 700_000
    src = (meshes.reference_mixed_queries(mesh, n, seed=11) if mix == "harness"
           else meshes.mixed_queries(mesh, n, seed=12))
    q = [cuda.from_numpy(v).cuda() for v in src]
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    mom = g.gwn_bvh4_moment_object(2)
    assert g.gwn_refit_bvh_moment(2, bvh, mom).is_ok()
    outs = {}
    for walk in ("warp", "thread"):
        o = cuda.full((n,), float("nan"), device="cuda")
        assert g.gwn_compute_winding_number_taylor_batch(2, bvh, mom, *q, o, 2.0, traversal=walk).is_ok()
        cuda.cuda.synchronize()
        outs[walk] = o.cpu().numpy()
    assert not np.isnan(outs["warp"]).any()
    np.testing.assert_array_equal(outs["warp"], outs["thread"])
    st, pr = api.taylor_form_probe(bvh, mom, *q, accuracy_scale=2.0)
    assert st.is_ok() and pr["sampled_warps"] > 0 and pr["sampled_warps"] % 32 == 0
    rule = pr["warp_nodes"] >= 1.3 * pr["lane_max_nodes"] and pr["lane_max_tris"] <= 8.0
    assert pr["per_thread"] == (1.0 if rule else 0.0)
    assert g.gwn_compute_winding_number_taylor_batch(2, bvh, mom, *q, o, 2.0, traversal="sideways").error == \
        g.gwn_error.invalid_argument
