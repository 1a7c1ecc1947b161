"""GPU parity of the boundary chain and the antipodal winding number / gradient.

Boundary chains equal the oracle's (detail/gwn_boundary_impl.cuh restated) and smallgwn's own rows
exactly, in order. Antipodal values: smallgwn's known answers (tests/unit_gwn_query_antipodal.cu,
tolerance 3e-4 against the exact winding number); the oracle's restatement, which guards the same
ill-conditioned terms with FP64 (same singular axes, NaN pattern and crossing counts; totals within
2e-5, the spherical areas going through two different atan2 implementations); smallgwn's own
kernels (oracle/_ref) through the FP64 truth: an error against the FP64 exact winding number
(values) and against FP64 central differences (gradients) never worse than twice theirs.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from conftest import _mesh, cube, open_cube
from smallgwn_b200 import api, meshes
from test_gpu_build import WORKLOADS, build, upload

pytestmark = pytest.mark.gpu

METHODS = {"lbvh": g.gwn_bvh_build_method.k_lbvh, "hploc": g.gwn_bvh_build_method.k_hploc}
MESHES = dict(WORKLOADS, open_cube=open_cube, cube=cube, soup80=lambda: meshes.soup_mesh(80, seed=21),
              net=lambda: _mesh([0, 1, 0, 1], [0, 0, 1, 1], [0] * 4, [0, 1, 0, 0], [1, 0, 1, 1], [2, 3, 2, 2]))


def dev(cuda, *arrs):
    return [cuda.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in arrs]


def chain_of(geo):
    ch = g.gwn_boundary_chain_object()
    st = g.gwn_build_boundary_chain(geo, ch)
    assert st.is_ok(), st.message
    return ch


def gpu_antipodal(cuda, geo, bvh, ch, q, **kw):
    d = dev(cuda, *q)
    out = cuda.empty_like(d[0])
    st = g.gwn_compute_winding_number_antipodal_batch(geo, bvh, ch, *d, out, **kw)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return out.cpu().numpy()


def gpu_gradient(cuda, geo, ch, q):
    d = dev(cuda, *q)
    gs = [cuda.empty_like(d[0]) for _ in range(3)]
    st = g.gwn_compute_winding_gradient_antipodal_batch(geo, ch, *d, *gs)
    assert st.is_ok(), st.message
    cuda.cuda.synchronize()
    return np.stack([x.cpu().numpy() for x in gs], axis=1)


def queries(mesh, n, seed):
    rng = np.random.default_rng(seed)
    lo = np.array([mesh[k].min() for k in "xyz"], np.float32)
    hi = np.array([mesh[k].max() for k in "xyz"], np.float32)
    c, e = (lo + hi) / 2, (hi - lo) / 2 * 1.3 + 1e-3
    return (c[:, None] + e[:, None] * rng.uniform(-1, 1, (3, n))).astype(np.float32)


@pytest.mark.parametrize("name", list(MESHES))
def test_boundary_chain_equals_oracle(cuda, name):
    mesh = MESHES[name]()
    ch = chain_of(upload(mesh))
    assert ch.has_data()
    ref = oracle.boundary_chain(mesh)
    got = ch.rows()
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    assert ch.accessor().mesh_vertex_count == mesh["x"].size
    assert ch.accessor().mesh_triangle_count == mesh["i0"].size


def test_boundary_chain_of_empty_geometry_is_built_empty():
    geo = g.gwn_geometry_object()
    ch = g.gwn_boundary_chain_object()
    assert g.gwn_build_boundary_chain(geo, ch).is_ok()
    assert ch.has_data() and ch.empty()


def test_known_answers(cuda):
    """unit_gwn_query_antipodal.cu:332-396 and :549-575."""
    qs = [np.array(v, np.float32) for v in ([0.23, 2.2, -0.41, -2.3], [0.17, 0.3, 0.26, -0.4], [0.11, 0.2, 1.7, 0.5])]
    col = [np.array(v, np.float32) for v in ([2, 2, -2, -2], [-1, 1, -1, 1], [2, 2, 2, 2])]
    sing = [np.array(v, np.float32) for v in ([1, -1, 1, -1], [1, 1, -1, -1], [1, 1, 1, 1])]
    for mesh_fn in (cube, open_cube):
        m = mesh_fn()
        geo = upload(m)
        bvh = build(geo)
        ch = chain_of(geo)
        for q in (qs, col):
            assert np.abs(gpu_antipodal(cuda, geo, bvh, ch, q) - oracle.exact_winding(m, *q)).max() <= 3e-4
        if mesh_fn is open_cube:
            assert np.isnan(gpu_antipodal(cuda, geo, bvh, ch, sing)).all()
            assert np.isnan(gpu_gradient(cuda, geo, ch, sing)).all()


def test_gradient_known_answers(cuda):
    """unit_gwn_query_antipodal.cu:398-460: central differences (eps 1e-2, 6e-3) and the mirror
    symmetry of retried queries."""
    m = open_cube()
    geo = upload(m)
    bvh = build(geo)
    ch = chain_of(geo)
    q = [np.array(v, np.float32) for v in ([0.21, 1.3, -1.4, 0.35], [0.18, 0.25, -0.33, 1.4], [0.15, 0.2, 0.42, 1.55])]
    gr = gpu_gradient(cuda, geo, ch, q)
    for ax in range(3):
        p = [v.copy() for v in q]
        n = [v.copy() for v in q]
        p[ax] += 1e-2
        n[ax] -= 1e-2
        fd = (gpu_antipodal(cuda, geo, bvh, ch, p) - gpu_antipodal(cuda, geo, bvh, ch, n)) / 2e-2
        assert np.abs(gr[:, ax] - fd).max() <= 6e-3
    q = [np.array(v, np.float32) for v in ([1, 1, 1, 1], [0.25, -0.25, 0.5, -0.5], [0.2, 0.2, 0.4, 0.4])]
    gr = gpu_gradient(cuda, geo, ch, q)
    assert np.isfinite(gr).all()
    for a, b in ((0, 1), (2, 3)):
        assert abs(gr[a, 0] - gr[b, 0]) <= 1e-6 and abs(gr[a, 1] + gr[b, 1]) <= 1e-6
        assert abs(gr[a, 2] - gr[b, 2]) <= 1e-6


@pytest.mark.parametrize("method", list(METHODS))
@pytest.mark.parametrize("name", ["icosphere4", "uv64x32", "soup40", "soup80", "open_cube", "octahedron"])
def test_equals_oracle(cuda, name, method):
    mesh = MESHES[name]()
    geo = upload(mesh)
    bvh = build(geo, METHODS[method])
    ch = chain_of(geo)
    h = api.bvh_host_arrays(bvh)
    q = queries(mesh, 3000, seed=31)
    ref = oracle.antipodal(mesh, h["nodes"], h["triangles"], h["root_reference"], ch.rows(), *q)
    for sort in (False, True):
        got = gpu_antipodal(cuda, geo, bvh, ch, q, sort_queries=sort)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert np.abs(got[ok] - ref[ok]).max() <= 2e-5
        if ch.empty():  # closed: integral crossing counts, bit for bit
            np.testing.assert_array_equal(got, ref)
    gr = gpu_gradient(cuda, geo, ch, q)
    gref = oracle.antipodal_gradient(mesh, ch.rows(), *q)
    np.testing.assert_array_equal(np.isnan(gr), np.isnan(gref))
    ok = ~np.isnan(gref)
    assert np.abs(gr[ok] - gref[ok]).max() <= 1e-5 * max(1.0, float(np.abs(gref[ok]).max()))


def test_rejects_missing_or_mismatched_boundary(cuda):
    """unit_gwn_query_antipodal.cu:577-669."""
    m = cube()
    geo = upload(m)
    bvh = build(geo)
    d = dev(cuda, [0.23], [0.17], [0.11])
    out = cuda.empty_like(d[0])
    missing = g.gwn_boundary_chain_object()
    assert g.gwn_compute_winding_number_antipodal_batch(geo, bvh, missing, *d, out).error == api.gwn_error.invalid_argument
    mismatched = chain_of(geo)
    mismatched.accessor().mesh_vertex_count += 1
    assert g.gwn_compute_winding_number_antipodal_batch(geo, bvh, mismatched, *d, out).error == \
        api.gwn_error.invalid_argument
    assert "different mesh shape" in g.gwn_compute_winding_gradient_antipodal_batch(geo, mismatched, *d, out, out,
                                                                                     out).message
    mismatched.accessor().mesh_vertex_count -= 1
    assert g.gwn_compute_winding_gradient_antipodal_batch(geo, missing, *d, out, out, out).error == \
        api.gwn_error.invalid_argument
    assert g.gwn_compute_winding_gradient_antipodal_batch(geo, mismatched, *d, None, out, out).error == \
        api.gwn_error.invalid_argument


def fp64_gradient(mesh, q, h=1e-5):
    """Richardson central differences of the FP64 exact winding number, and the mask of queries
    farther than 100 h from the surface."""
    qd = q.astype(np.float64)
    out = np.zeros((q.shape[1], 3))
    for ax in range(3):
        def cd(step):
            a, b = qd.copy(), qd.copy()
            a[ax] += step
            b[ax] -= step
            return (oracle.exact_winding(mesh, *a, fp64=True) - oracle.exact_winding(mesh, *b, fp64=True)) / (2 * step)
        out[:, ax] = (4 * cd(h) - cd(2 * h)) / 3
    return out, oracle.mesh_distance(mesh, *q) > 100 * h


needs_ref = pytest.mark.skipif(oracle.ref_lib() is None, reason="smallgwn's kernels (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("name", ["open_cube", "soup40", "soup80", "uv64x32"])
def test_against_smallgwn_kernels(cuda, name):
    mesh = MESHES[name]()
    geo = upload(mesh)
    bvh = build(geo, METHODS["hploc"])
    ch = chain_of(geo)
    ref = oracle.Reference(mesh)
    ref.build(method=0, radius=8)
    for a, b in zip(ch.rows(), ref.boundary()):
        np.testing.assert_array_equal(a, b)
    q = queries(mesh, 3000, seed=32)
    ours = gpu_antipodal(cuda, geo, bvh, ch, q)
    theirs = ref.antipodal(*q)
    both = ~np.isnan(ours) & ~np.isnan(theirs)
    assert both.mean() >= 0.999
    # against the FP64 exact winding number: never worse than twice smallgwn's error (plus 1e-6)
    exact = oracle.exact_winding(mesh, *q.astype(np.float64), fp64=True)
    e_ours = np.abs(ours - exact)[both]
    e_ref = np.abs(theirs - exact)[both]
    assert (e_ours <= 2 * e_ref + 1e-6).all() and e_ours.max() <= 1e-5
    # gradients against the FP64 truth (Richardson central differences of the FP64 exact winding
    # number) away from the surface: ours evaluates the ill-conditioned terms in FP64, so its error
    # is never worse than twice smallgwn's (plus 1e-4), and small everywhere
    gr = gpu_gradient(cuda, geo, ch, q)
    gt = ref.antipodal_gradient(*q)
    truth, far = fp64_gradient(mesh, q)
    ok = far & ~np.isnan(gt).any(1)
    e_ours = np.abs(gr - truth).max(1)[ok]
    e_ref = np.abs(gt - truth).max(1)[ok]
    assert (e_ours <= 2 * e_ref + 1e-4).all()
    assert np.quantile(e_ours, 0.99) <= 1e-4
    ref.close()
