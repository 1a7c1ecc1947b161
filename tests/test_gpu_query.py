"""GPU parity of the winding-number queries against the oracle and smallgwn's own kernels.

Tolerances: every query within 1e-5 + 2e-5 |w| of the other implementation (smallgwn's builder
tests use 2e-5 + 2e-5 |w|, tests/integration_gwn_builder.cu:228-233), with no blanket exemption:
a query outside it must be explained in FP64 (tests/taylor_decisions.py) -- an FP32 solid angle
seen along an edge's line, or, against smallgwn's kernels only, an acceptance test that decides
differently under the two moment sets. Against the oracle's traversal of the same tree the
acceptance test rounds the same way on both sides, so decisions and traversal statistics are
identical. Full descent (beta = 1e6) equals exact within 1e-6 (tests/unit_gwn_bvh_moment.cu:42-114)
and, with the compensated near field, the FP64 oracle within 1e-6 on the small exact workload and
on the golden fixtures; for queries 1e-3 off the surface the records' own rounding sets the bound
NEAR_SURFACE_TOL below. The
FP64 brute force behind every error figure is pinned to the oracle's FP64 restatement of
smallgwn's CPU reference. Contract checks restate tests/unit_gwn_query_winding.cu:222-313,
tests/unit_gwn_bvh_moment.cu:116-268 and tests/unit_gwn_query_stack.cu:246-345; the gradient is
checked against central differences as in tests/unit_gwn_query_gradient.cu:211-267.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from conftest import asym_octahedron, octahedron, single_triangle
from smallgwn_b200 import api, meshes
from taylor_decisions import disagreement_report, explain
from test_gpu_build import WORKLOADS, build, upload

pytestmark = pytest.mark.gpu

EXACT_TOL = 1e-5
# Full descent against exact, and the compensated near field against FP64, for queries 1e-3 off the
# surface (the mixed query sets): both forms evaluate smallgwn's triangle records {v0, v1 - v0,
# v2 - v0}, whose float edges and the float sums b = (v0 - q) + e1, c = (v0 - q) + e2 carry errors
# relative to the distance to the farthest vertex; for a query close to a vertex other than v0 that
# is up to ~2e-6 in the winding number (measured in FP64 over the same records on these meshes).
# Away from the surface (the small exact workload's uniform queries) the bound is smallgwn's 1e-6.
NEAR_SURFACE_TOL = 2.5e-6


class Agreement:
    """FP32-vs-FP32 agreement report: |a - b| <= atol + rtol * max(|a|, |b|) (smallgwn's builder
    tests use 2e-5 + 2e-5 |w|, tests/integration_gwn_builder.cu:228-233)."""

    def __init__(self, a, b, atol=EXACT_TOL, rtol=2e-5):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        self.diff = np.abs(a - b)
        self.bad = self.diff > atol + rtol * np.maximum(np.abs(a), np.abs(b))
        self.bad_count = int(np.count_nonzero(self.bad))
        self.n = int(a.size)

    def __bool__(self) -> bool:
        return self.bad_count == 0

    def __repr__(self) -> str:
        return f"Agreement({self.bad_count}/{self.n} outside, max diff {self.diff.max() if self.n else 0:.3e})"


def within(a, b, atol=EXACT_TOL, rtol=2e-5) -> Agreement:
    return Agreement(a, b, atol, rtol)


def assert_agree_or_explained(a, b, q, h, mom_a, mom_b, pairing, beta, allow, atol=EXACT_TOL, rtol=2e-5,
                              rel=1e-6) -> dict:
    """Every query within atol + rtol |w| of the other implementation, or its disagreement explained
    in FP64 by a reason in `allow` (taylor_decisions.explain over tree h). Returns the report: max
    and p99 of |a - b| over all queries and the count per reason."""
    rep = disagreement_report(a, b, atol, rtol)
    reasons: dict = {}
    for i in rep["outside"]:
        why = explain((q[0][i], q[1][i], q[2][i]), h["nodes"], h["root_reference"], mom_a, mom_b, pairing,
                      h["triangles"], beta, rel=rel, observed=abs(float(a[i]) - float(b[i])))
        assert why in allow, f"query {i} ({q[0][i]}, {q[1][i]}, {q[2][i]}): {a[i]} vs {b[i]}, reason {why}"
        reasons[why] = reasons.get(why, 0) + 1
    rep["reasons"] = reasons
    print(f"max |diff| {rep['max']:.3e}, p99 {rep['p99']:.3e}, explained outside tolerance: {reasons}")
    return rep


def dev(cuda, *arrs):
    return [cuda.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in arrs]


def run_exact(cuda, bvh, q):
    d = dev(cuda, *q)
    out = cuda.empty_like(d[0])
    st = g.gwn_compute_winding_number_exact_batch(bvh, *d, out)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out.cpu().numpy()


def run_taylor(cuda, order, bvh, mom, q, beta, **kw):
    d = dev(cuda, *q)
    out = cuda.empty_like(d[0])
    st = g.gwn_compute_winding_number_taylor_batch(order, bvh, mom, *d, out, accuracy_scale=beta, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out.cpu().numpy()


def moments_of(bvh, order):
    m = g.gwn_bvh4_moment_object(order)
    st = g.gwn_refit_bvh_moment(order, bvh, m)
    assert st.is_ok(), st.message
    return m


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_exact_batch_matches_oracle(cuda, name):
    mesh = WORKLOADS[name]()
    bvh = build(upload(mesh))
    q = meshes.mixed_queries(mesh, 3000, seed=4) if mesh["i0"].size > 100 else meshes.small_queries(3000)
    out = run_exact(cuda, bvh, q)
    ref = oracle.exact_winding(mesh, *q)
    # 513 coincident triangles sum 513 equal solid angles: FP32 rounding grows with the count
    rtol = 1e-4 if name.startswith("equal") else 2e-5
    # the oracle's FP32 brute force loses digits for a query along an edge's line (ours takes those
    # pairs in FP64): every other query agrees within tolerance
    h = api.bvh_host_arrays(bvh)
    mh0 = api.moment_host_array(moments_of(bvh, 0))
    assert_agree_or_explained(out, ref, q, h, mh0, mh0, None, 1e6, allow=("conditioning",), rtol=rtol, rel=0.0)
    # ours is no further from FP64 than the oracle's FP32 brute force (up to rounding), and with
    # the FP64 re-evaluation of cancelling pairs it stays within a few FP32 ulps of the sum
    ref64 = oracle.exact_winding(mesh, *q, fp64=True)
    err = np.abs(out - ref64)
    assert err.max() <= 2 * np.max(np.abs(ref - ref64)) + EXACT_TOL
    if not name.startswith("equal"):
        assert err.max() <= 5e-6, err.max()


def test_exact_batch_small_workload_full(cuda):
    mesh = meshes.small_mesh()
    bvh = build(upload(mesh))
    q = meshes.small_queries(100_000)
    out = run_exact(cuda, bvh, q)
    ref = oracle.exact_winding(mesh, *q)
    err = np.abs(out - ref)
    assert err.max() <= EXACT_TOL, err.max()


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("method", [g.gwn_bvh_build_method.k_lbvh, g.gwn_bvh_build_method.k_hploc])
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40"])
def test_taylor_matches_oracle_traversal(cuda, name, method, order):
    mesh = WORKLOADS[name]()
    bvh = build(upload(mesh), method)
    mom = moments_of(bvh, order)
    h = api.bvh_host_arrays(bvh)
    mh = api.moment_host_array(mom)
    q = meshes.mixed_queries(mesh, 4000, seed=6)
    ref_mom = oracle.moments(order, h["nodes"], h["triangles"])
    scale = np.abs(ref_mom).max(axis=(0, 2), keepdims=True) + 1e-12
    assert np.max(np.abs(mh - ref_mom) / scale) < 1e-4
    ref = oracle.taylor(order, h["nodes"], mh, h["triangles"], h["root_reference"], *q, beta=2.0)
    # same tree and moments, and the acceptance test in one fixed rounding pattern on both sides:
    # every decision is the same, so the only disagreements beyond rounding are near-field
    # triangles seen along an edge's line, where the two FP32 solid-angle formulas both lose digits
    for sort in (True, False):
        out = run_taylor(cuda, order, bvh, mom, q, 2.0, sort_queries=sort)
        assert_agree_or_explained(out, ref, q, h, mh, mh, None, 2.0, allow=("conditioning",), rel=0.0)
    # ...and the compensated near field removes those too
    comp = run_taylor(cuda, order, bvh, mom, q, 2.0, precision=g.near_precision.compensated)
    assert_agree_or_explained(comp, ref, q, h, mh, mh, None, 2.0, allow=("conditioning",), rel=0.0)
    # full descent evaluates every triangle exactly: with the compensated near field it equals the
    # exact batch within the near-surface bound (smallgwn's own check, tests/unit_gwn_bvh_moment.cu
    # :42-114, is 1e-6 on queries away from the surface; see test_full_descent_equals_exact_*)
    full = run_taylor(cuda, order, bvh, mom, q, 1e6, precision=g.near_precision.compensated)
    exact = run_exact(cuda, bvh, q)
    assert np.max(np.abs(full - exact)) <= NEAR_SURFACE_TOL


@pytest.mark.parametrize("method", [g.gwn_bvh_build_method.k_lbvh, g.gwn_bvh_build_method.k_hploc])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_full_descent_equals_exact_on_reference_fixture(cuda, order, method):
    """smallgwn's own check (tests/unit_gwn_bvh_moment.cu:42-114): on the octahedron, with beta =
    1e6 every cluster descends and the Taylor batch equals the exact batch within 1e-6, for every
    order and both builders -- here for both near-field forms."""
    bvh = build(upload(octahedron()), method)
    mom = moments_of(bvh, order)
    q = [np.array([0.13, 3.25], np.float32), np.array([-0.21, -2.5], np.float32), np.array([0.17, 4.75], np.float32)]
    exact = run_exact(cuda, bvh, q)
    for prec in (g.near_precision.plain, g.near_precision.compensated):
        taylor = run_taylor(cuda, order, bvh, mom, q, 1e6, precision=prec)
        assert np.max(np.abs(taylor - exact)) <= 1e-6


def test_full_descent_equals_exact_small_workload(cuda):
    """The small exact workload (icosphere level 4, 5,120 triangles, 100,000 queries in
    [-1.5, 1.5]^3): full-descent Taylor with the compensated near field equals the exact batch within
    1e-6 and the FP64 oracle within 1e-6, over every query."""
    mesh = meshes.small_mesh()
    bvh = build(upload(mesh))
    q = meshes.small_queries(100_000)
    exact = run_exact(cuda, bvh, q)
    ref64 = oracle.exact_winding(mesh, *q, fp64=True)
    for order in (0, 2):
        mom = moments_of(bvh, order)
        full = run_taylor(cuda, order, bvh, mom, q, 1e6, precision=g.near_precision.compensated)
        assert np.max(np.abs(full - exact)) <= 1e-6
        assert np.max(np.abs(full - ref64)) <= 1e-6
    assert np.max(np.abs(exact - ref64)) <= 1e-6


@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40", "octahedron"])
def test_fp64_exact_kernel_matches_oracle(cuda, name):
    """The FP64 brute force that measures every error figure (gwnb_winding_exact_geometry_fp64)
    against the oracle's FP64 restatement of smallgwn's CPU reference (tests/reference_cpu.cuh:22-82
    with Real = double)."""
    mesh = WORKLOADS[name]()
    geo = upload(mesh)
    q = meshes.mixed_queries(mesh, 3000, seed=5) if mesh["i0"].size > 100 else meshes.small_queries(3000)
    d = dev(cuda, *q)
    out = cuda.empty(q[0].size, dtype=cuda.float64, device="cuda")
    assert api.exact_winding_fp64(geo, *d, out).is_ok()
    cuda.cuda.synchronize()
    ref = oracle.exact_winding(mesh, *q, fp64=True)
    # the two FP64 formulas (unit-vector and unnormalised Van Oosterom-Strackee) round apart only
    # where the pair cancels: 1e-10 is 3-4 orders below any FP32 error figure
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-10


def test_fp64_exact_kernel_matches_oracle_at_size(cuda):
    """The same on the 1,046,528-triangle benchmark sphere, 1,000 of its mixed queries."""
    mesh = meshes.sphere_mesh()
    geo = upload(mesh)
    q = [v[:1000].copy() for v in meshes.mixed_queries(mesh, 1000, seed=2)]
    d = dev(cuda, *q)
    out = cuda.empty(1000, dtype=cuda.float64, device="cuda")
    assert api.exact_winding_fp64(geo, *d, out).is_ok()
    cuda.cuda.synchronize()
    ref = oracle.exact_winding(mesh, *q, fp64=True)
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-10


@pytest.mark.parametrize("order", [0, 1, 2])
def test_traversal_statistics_match_oracle(cuda, order):
    mesh = WORKLOADS["uv64x32"]()
    bvh = build(upload(mesh), g.gwn_bvh_build_method.k_hploc)
    mom = moments_of(bvh, order)
    h = api.bvh_host_arrays(bvh)
    mh = api.moment_host_array(mom)
    q = meshes.mixed_queries(mesh, 2000, seed=8)
    d = dev(cuda, *q)
    stats = [cuda.empty(2000, dtype=cuda.int32, device="cuda") for _ in range(3)]
    assert api.taylor_traversal_stats(bvh, mom, *d, *stats, accuracy_scale=2.0).is_ok()
    got = np.stack([s.cpu().numpy() for s in stats], -1)
    _, ref = oracle.taylor(order, h["nodes"], mh, h["triangles"], h["root_reference"], *q, beta=2.0, stats=True)
    # the acceptance test rounds the same way on both sides: identical decisions for every query
    np.testing.assert_array_equal(got, ref.astype(got.dtype))


@pytest.mark.parametrize("method", [g.gwn_bvh_build_method.k_lbvh, g.gwn_bvh_build_method.k_hploc])
def test_far_field_orders_reduce_error(cuda, method):
    mesh = asym_octahedron()
    bvh = build(upload(mesh), method)
    q = [np.array(v, np.float32) for v in ([2.9, -2.7, 0.4, -0.6, 3.2, -2.8, 1.8, -2.1],
                                          [0.4, -0.8, 3.1, -2.9, 2.2, 1.7, -2.6, 2.4],
                                          [1.1, -0.5, 0.8, -1.2, -2.3, 2.5, 2.8, -2.5])]
    ref = oracle.exact_winding(mesh, *q)
    errs = [float(np.mean(np.abs(run_taylor(cuda, o, bvh, moments_of(bvh, o), q, 0.0) - ref))) for o in (0, 1, 2)]
    assert errs[1] < errs[0] and errs[2] < errs[1] and errs[2] < 2e-3


def test_nan_query_propagates(cuda):
    mesh = asym_octahedron()
    bvh = build(upload(mesh))
    mom = moments_of(bvh, 2)
    q = [np.array([np.nan], np.float32), np.array([0.25], np.float32), np.array([3.0], np.float32)]
    assert np.isnan(run_exact(cuda, bvh, q)[0])
    assert np.isnan(run_taylor(cuda, 2, bvh, mom, q, 0.0)[0])


def test_leaf_root_taylor_equals_exact(cuda):
    bvh = build(upload(single_triangle()))
    mom = moments_of(bvh, 2)
    q = [np.array([2.0], np.float32)] * 3
    t = run_taylor(cuda, 2, bvh, mom, q, 0.0)
    e = run_exact(cuda, bvh, q)
    assert t[0] == pytest.approx(e[0], rel=1e-6)


def test_batch_contract(cuda):
    empty_bvh = g.gwn_bvh4_object()
    empty_mom = g.gwn_bvh4_moment_object(0)
    e = cuda.empty(0, device="cuda")
    assert g.gwn_compute_winding_number_taylor_batch(0, empty_bvh, empty_mom, e, e, e, e).error == \
        g.gwn_error.invalid_argument
    assert g.gwn_compute_winding_number_exact_batch(empty_bvh, e, e, e, e).error == g.gwn_error.invalid_argument
    bvh = build(upload(asym_octahedron()))
    mom = moments_of(bvh, 0)
    assert g.gwn_compute_winding_number_taylor_batch(0, bvh, mom, e, e, e, e).is_ok()
    for beta in (-1.0, float("nan")):
        assert g.gwn_compute_winding_number_taylor_batch(0, bvh, mom, e, e, e, e, accuracy_scale=beta).error == \
            g.gwn_error.invalid_argument
    assert g.gwn_compute_winding_number_exact_batch(bvh, e, e, e, e).is_ok()
    one = cuda.empty(1, device="cuda")
    assert g.gwn_compute_winding_number_taylor_batch(0, bvh, mom, e, e, e, one).error == g.gwn_error.invalid_argument
    assert g.gwn_compute_winding_number_exact_batch(bvh, e, e, e, one).error == g.gwn_error.invalid_argument


def test_stale_moments_rejected_after_rebuild_and_refit(cuda):
    geo = upload(octahedron())
    bvh = build(geo)
    mom = moments_of(bvh, 1)
    e = cuda.empty(0, device="cuda")
    assert g.gwn_build_bvh(geo, bvh).is_ok()
    assert not mom.is_valid_for(bvh)
    assert g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, e, e, e, e).error == g.gwn_error.invalid_argument
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok() and mom.is_valid_for(bvh)
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    assert not mom.is_valid_for(bvh)
    assert g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, e, e, e, e).error == g.gwn_error.invalid_argument


def test_stack_capacity_below_bound_rejected(cuda):
    bvh = build(upload(octahedron()))
    assert bvh.accessor().internal_stack_bound > 1
    mom = moments_of(bvh, 1)
    q = dev(cuda, [0.25], [0.25], [2.0])
    out = cuda.empty(1, device="cuda")
    st = g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, *q, out,
                                                   config=g.gwn_query_batch_config(stack_capacity=1))
    assert st.error == g.gwn_error.invalid_argument and "Traversal stack capacity" in st.message


def test_moment_replacement_on_other_stream(cuda):
    s_a, s_b = cuda.cuda.Stream(), cuda.cuda.Stream()
    geo = upload(octahedron(), s_a)
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, stream=s_a).is_ok()
    mom = g.gwn_bvh4_moment_object(0)
    assert g.gwn_refit_bvh_moment(0, bvh, mom, s_a).is_ok()
    n = 1 << 20
    q = [cuda.zeros(n, device="cuda") for _ in range(3)]
    out = cuda.empty(n, device="cuda")
    s_a.synchronize()
    assert g.gwn_compute_winding_number_taylor_batch(0, bvh, mom, *q, out, stream=s_a).is_ok()
    assert g.gwn_refit_bvh_moment(0, bvh, mom, s_b).is_ok()
    assert mom.stream() is s_b and mom.is_valid_for(bvh)
    s_b.synchronize()
    s_a.synchronize()


@pytest.mark.parametrize("order", [1, 2])
def test_gradient_matches_central_differences(cuda, order):
    # an open, inconsistently oriented soup: its winding number varies off the surface (a closed
    # mesh has zero gradient everywhere away from it)
    mesh = meshes.soup_mesh(48, seed=31)
    bvh = build(upload(mesh), g.gwn_bvh_build_method.k_hploc)
    mom = moments_of(bvh, order)
    rng = np.random.default_rng(3)
    d = rng.normal(size=(64, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    radius = np.where(np.arange(64) % 2 == 0, 0.5, 1.5) + rng.uniform(-0.05, 0.05, size=64)
    p = (d * radius[:, None]).astype(np.float32)
    q = [p[:, k].copy() for k in range(3)]
    d = dev(cuda, *q)
    gr = [cuda.empty(64, device="cuda") for _ in range(3)]
    st = g.gwn_compute_winding_gradient_taylor_batch(order, bvh, mom, *d, *gr, accuracy_scale=1e6)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    grad = np.stack([x.cpu().numpy() for x in gr], -1)
    h = 1e-3
    fd = np.zeros_like(grad)
    for k in range(3):
        qp = [c.astype(np.float64) for c in q]
        qm = [c.astype(np.float64) for c in q]
        qp[k] = qp[k] + h
        qm[k] = qm[k] - h
        wp = oracle.exact_winding(mesh, *qp, fp64=True)
        wm = oracle.exact_winding(mesh, *qm, fp64=True)
        fd[:, k] = (wp - wm) / (2 * h)
    scale = np.abs(fd).max() + 1e-6
    assert np.max(np.abs(grad - fd)) / scale < 3e-3


@pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's own kernels (oracle/_ref) not built")
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40"])
def test_queries_match_reference_kernels(cuda, name):
    """Against smallgwn's own kernels on the same inputs and the same LBVH (up to node numbering).
    Every query agrees within 1e-5 + 2e-5 |w|, or its disagreement is explained in FP64
    (taylor_decisions): an acceptance test that decides differently under the two moment sets (whose
    last bits differ with the climbs' summation order) or sits within rounding of its threshold, or
    a near-field triangle seen along an edge's line. The max and p99 difference over all queries
    are printed with the count per reason."""
    mesh = WORKLOADS[name]()
    bvh = build(upload(mesh))
    R = oracle.Reference(mesh)
    R.build(1, 8, 64)
    q = meshes.mixed_queries(mesh, 4000, seed=12)
    h = api.bvh_host_arrays(bvh)
    rb = R.bvh()
    pairing = oracle.match_wide_nodes(h["nodes"], h["root_reference"], rb["nodes"], rb["root_reference"])
    ref64 = oracle.exact_winding(mesh, *q, fp64=True)
    ours, theirs = run_exact(cuda, bvh, q), R.exact(*q)
    # exact: the only disagreements are FP32 cancellation along edge lines, where ours re-evaluates
    # in FP64 and stays within a few ulps of the FP64 sum
    m0 = moments_of(bvh, 0)
    mh0 = api.moment_host_array(m0)
    assert_agree_or_explained(ours, theirs, q, h, mh0, mh0, None, 1e6, allow=("conditioning",), rel=0.0)
    assert np.max(np.abs(ours - ref64)) <= min(5e-6, 2 * np.max(np.abs(theirs - ref64)) + EXACT_TOL)
    for order in (0, 1, 2):
        mom = moments_of(bvh, order)
        ref_m = R.moments(order)
        mh = api.moment_host_array(mom)
        scale = np.abs(ref_m).max(axis=(0, 2), keepdims=True) + 1e-12
        assert np.max(np.abs(mh - ref_m[pairing]) / scale) < 1e-4
        # beta = 2: smallgwn's plain FP32 form on both sides, then our compensated form
        theirs = R.taylor(order, *q, beta=2.0)
        for prec in (g.near_precision.plain, g.near_precision.compensated):
            ours = run_taylor(cuda, order, bvh, mom, q, 2.0, precision=prec)
            assert_agree_or_explained(ours, theirs, q, h, mh, ref_m, pairing, 2.0,
                                      allow=("decision", "conditioning", "moments"))
        # full descent: every triangle exactly, the plain FP32 near field on both sides
        full, full_ref = run_taylor(cuda, order, bvh, mom, q, 1e6), R.taylor(order, *q, beta=1e6)
        assert_agree_or_explained(full, full_ref, q, h, mh, mh, None, 1e6, allow=("conditioning",), rel=0.0)
        e_ours, e_ref = np.abs(full - ref64), np.abs(full_ref - ref64)
        assert np.quantile(e_ours, 0.99) <= 2 * np.quantile(e_ref, 0.99) + 1e-6
        assert e_ours.max() <= 4 * e_ref.max() + EXACT_TOL
        # the compensated near field with FP64 for cancelling pairs is within the near-surface bound
        # of FP64
        comp = run_taylor(cuda, order, bvh, mom, q, 1e6, precision=g.near_precision.compensated,
                          fp64_threshold=1.0 / 16.0)
        assert np.abs(comp - ref64).max() <= NEAR_SURFACE_TOL
    R.close()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_warp_cooperative_equals_per_thread_traversal(cuda, order):
    """The warp-cooperative traversal visits every lane's nodes in that lane's own depth-first
    order, so both traversal kernels produce the same sums."""
    mesh = WORKLOADS["soup40"]()
    bvh = build(upload(mesh), g.gwn_bvh_build_method.k_hploc)
    mom = moments_of(bvh, order)
    q = meshes.mixed_queries(mesh, 5000, seed=17)
    for beta in (1.0, 2.0, 3.5):
        for prec in (g.near_precision.plain, g.near_precision.compensated):
            a = run_taylor(cuda, order, bvh, mom, q, beta, precision=prec)
            b = run_taylor(cuda, order, bvh, mom, q, beta, precision=prec, per_thread=True)
            assert np.mean(a == b) > 0.999 and within(a, b, atol=1e-6, rtol=1e-6)


def test_timed_walk_choice(cuda):
    """GWNB_WALK_TIMED: the first call of a kind walks warp-cooperatively, the second per thread,
    both timed, and later calls take the faster walk. Every call returns what one of the two forced
    walks returns; another accuracy scale is another kind; the gradient batch takes the option too."""
    mesh = WORKLOADS["uv64x32"]()
    bvh = build(upload(mesh), g.gwn_bvh_build_method.k_hploc)
    mom = moments_of(bvh, 2)
    q = meshes.mixed_queries(mesh, 20000, seed=29)
    for beta in (2.0, 3.0):
        forced = [run_taylor(cuda, 2, bvh, mom, q, beta, traversal=w) for w in ("warp", "thread")]
        for _ in range(6):
            got = run_taylor(cuda, 2, bvh, mom, q, beta, traversal="timed")
            assert any(np.array_equal(got, f) for f in forced)
    d = dev(cuda, *q)
    grads = []
    for walk in ("warp", "timed", "timed", "timed"):
        gr = [cuda.empty_like(d[0]) for _ in range(3)]
        st = g.gwn_compute_winding_gradient_taylor_batch(2, bvh, mom, *d, *gr, accuracy_scale=2.0, traversal=walk)
        assert st.is_ok(), st.message
        cuda.cuda.synchronize()
        grads.append(np.stack([v.cpu().numpy() for v in gr]))
    for other in grads[1:]:
        assert np.all(np.isfinite(other)) and within(other, grads[0], atol=1e-6, rtol=1e-6)


@pytest.mark.parametrize("block", [32, 128, 512, 1024])
def test_block_sizes_up_to_1024_give_the_same_results(cuda, block):
    """smallgwn accepts batch block sizes up to 1024 (include/gwn/gwn_query.cuh:37); the kernels here
    run blocks of at most 256 threads, so larger requests launch 256-thread blocks. Every batch
    kind returns the same results for every accepted block size, through the C ABI."""
    mesh = WORKLOADS["uv64x32"]()
    geo = upload(mesh)
    bvh = build(geo, g.gwn_bvh_build_method.k_hploc)
    mom = moments_of(bvh, 1)
    q = meshes.mixed_queries(mesh, 3000, seed=41)
    d = dev(cuda, *q)
    cfg = g.gwn_query_batch_config(block_size=block)
    outs = {}
    for name, fn in (
            ("taylor", lambda o, c: g.gwn_compute_winding_number_taylor_batch(1, bvh, mom, *d, o, config=c)),
            ("exact", lambda o, c: g.gwn_compute_winding_number_exact_batch(bvh, *d, o, config=c)),
            ("distance", lambda o, c: g.gwn_compute_unsigned_distance_batch(bvh, *d, o, config=c))):
        ref, got = cuda.empty_like(d[0]), cuda.empty_like(d[0])
        st = fn(ref, g.gwn_query_batch_config())
        assert st.is_ok(), st.message
        st = fn(got, cfg)
        assert st.is_ok(), (name, st.message)
        cuda.cuda.synchronize()
        assert cuda.equal(ref, got), name
        outs[name] = got
    assert np.isfinite(outs["taylor"].cpu().numpy()).all()
