"""The oracle's boundary chain and antipodal winding numbers (CPU), against smallgwn's known
answers (tests/unit_gwn_boundary.cu, tests/unit_gwn_query_antipodal.cu) and against the exact
winding number."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import _mesh, cube, open_cube
from smallgwn_b200 import meshes

QX = np.array([0.23, 2.2, -0.41, -2.3], np.float32)
QY = np.array([0.17, 0.3, 0.26, -0.4], np.float32)
QZ = np.array([0.11, 0.2, 1.7, 0.5], np.float32)


def rows(chain):
    return sorted(zip(*[a.tolist() for a in chain]))


def antipodal(mesh, *q, method="lbvh"):
    b = oracle.build_bvh(mesh, method)
    return oracle.antipodal(mesh, b["nodes"], b["triangles"], b["root_reference"], oracle.boundary_chain(mesh), *q)


def test_boundary_chain_known_answers():
    """unit_gwn_boundary.cu:94-187: empty and closed meshes give empty chains, the open cube its four
    rim edges, and opposite orientations cancel while repeated ones add up."""
    assert all(a.size == 0 for a in oracle.boundary_chain(_mesh([], [], [], [], [], [])))
    assert all(a.size == 0 for a in oracle.boundary_chain(cube()))
    assert rows(oracle.boundary_chain(open_cube())) == [(4, 7, 1), (5, 4, 1), (6, 5, 1), (7, 6, 1)]
    net = rows(oracle.boundary_chain(_mesh([0, 1, 0, 1], [0, 0, 1, 1], [0] * 4, [0, 1, 0, 0], [1, 0, 1, 1],
                                           [2, 3, 2, 2])))
    assert (0, 1, 2) in net and not any(r[:2] == (1, 0) for r in net)


def test_rows_ascend_by_low_then_high_vertex():
    s, e, m = oracle.boundary_chain(meshes.soup_mesh(40, seed=13))
    lo, hi = np.minimum(s, e).astype(np.uint64), np.maximum(s, e).astype(np.uint64)
    key = (lo << np.uint64(32)) | hi
    assert (np.diff(key.astype(np.int64)) > 0).all() and (m > 0).all()


@pytest.mark.parametrize("mesh_fn", [cube, open_cube])
def test_matches_exact_winding(mesh_fn):
    """unit_gwn_query_antipodal.cu:332-381 (tolerance 3e-4)."""
    m = mesh_fn()
    a = antipodal(m, QX, QY, QZ)
    assert np.abs(a - oracle.exact_winding(m, QX, QY, QZ)).max() <= 3e-4


def test_collinear_boundary_projections_retry():
    """unit_gwn_query_antipodal.cu:383-396."""
    m = open_cube()
    q = [np.array(v, np.float32) for v in ([2, 2, -2, -2], [-1, 1, -1, 1], [2, 2, 2, 2])]
    assert np.abs(antipodal(m, *q) - oracle.exact_winding(m, *q)).max() <= 3e-4


def test_all_axes_singular_give_nan():
    """unit_gwn_query_antipodal.cu:549-575: queries on the rim's corners."""
    m = open_cube()
    q = [np.array(v, np.float32) for v in ([1, -1, 1, -1], [1, 1, -1, -1], [1, 1, 1, 1])]
    assert np.isnan(antipodal(m, *q)).all()
    assert np.isnan(oracle.antipodal_gradient(m, oracle.boundary_chain(m), *q)).all()


def test_gradient_matches_finite_differences():
    """unit_gwn_query_antipodal.cu:398-438 (eps 1e-2, tolerance 6e-3)."""
    m = open_cube()
    q = [np.array(v, np.float32) for v in ([0.21, 1.3, -1.4, 0.35], [0.18, 0.25, -0.33, 1.4], [0.15, 0.2, 0.42, 1.55])]
    g = oracle.antipodal_gradient(m, oracle.boundary_chain(m), *q)
    eps = 1e-2
    for ax in range(3):
        p = [v.copy() for v in q]
        n = [v.copy() for v in q]
        p[ax] += eps
        n[ax] -= eps
        fd = (antipodal(m, *p) - antipodal(m, *n)) / (2 * eps)
        assert np.abs(g[:, ax] - fd).max() <= 6e-3


def test_gradient_retry_keeps_mirror_symmetry():
    """unit_gwn_query_antipodal.cu:440-460: queries whose +z boundary projection is singular."""
    m = open_cube()
    q = [np.array(v, np.float32) for v in ([1, 1, 1, 1], [0.25, -0.25, 0.5, -0.5], [0.2, 0.2, 0.4, 0.4])]
    g = oracle.antipodal_gradient(m, oracle.boundary_chain(m), *q)
    assert np.isfinite(g).all()
    for a, b in ((0, 1), (2, 3)):
        assert abs(g[a, 0] - g[b, 0]) <= 1e-6 and abs(g[a, 1] + g[b, 1]) <= 1e-6 and abs(g[a, 2] - g[b, 2]) <= 1e-6


def test_overflow_gives_nan():
    """unit_gwn_query_antipodal.cu:494-547: capacity 1 below the bound of 32 layers."""
    from spatial_cases import layered
    m = layered(32)
    b = oracle.build_bvh(m, "hploc")
    assert b["internal_stack_bound"] > 1
    q = [np.full(4, 0.25, np.float32), np.full(4, 0.25, np.float32), np.array([-1, -2, -3, -4], np.float32)]
    out = oracle.antipodal(m, b["nodes"], b["triangles"], b["root_reference"], oracle.boundary_chain(m), *q,
                           stack_capacity=1)
    assert np.isnan(out).all()


@pytest.mark.parametrize("method", ["lbvh", "hploc"])
def test_open_soup_against_fp64_exact(method):
    """Away from the surface the antipodal sum and the FP64 exact winding number agree to float
    accuracy of the spherical areas; the crossing term is exactly integral on a closed mesh."""
    soup = meshes.soup_mesh(40, seed=13)
    rng = np.random.default_rng(0)
    q = rng.uniform(-1.5, 1.5, (3, 3000)).astype(np.float32)
    a = antipodal(soup, *q, method=method)
    ex = oracle.exact_winding(soup, *[v.astype(np.float64) for v in q], fp64=True)
    assert not np.isnan(a).any()
    assert np.abs(a - ex).max() <= 3e-4
    closed = meshes.small_mesh()  # icosphere: closed, empty boundary chain
    c = antipodal(closed, *q, method=method)
    assert np.array_equal(c, np.round(c))


def test_guarded_terms_reach_fp64_accuracy():
    """Terms whose atan2 arguments are both small against |s||e| (the edge passes close to the ray
    line) are evaluated in FP64: values within 2e-6 of the FP64 exact winding number and gradients
    within 1e-4 of FP64 central differences, where all-float terms leave errors of order 1 in the
    gradient of 4 % of these queries."""
    soup = meshes.soup_mesh(80, seed=21)
    ch = oracle.boundary_chain(soup)
    b = oracle.build_bvh(soup, "hploc")
    rng = np.random.default_rng(32)
    q = rng.uniform(-1.5, 1.5, (3, 1500)).astype(np.float32)
    a = oracle.antipodal(soup, b["nodes"], b["triangles"], b["root_reference"], ch, *q)
    qd = q.astype(np.float64)
    assert np.abs(a - oracle.exact_winding(soup, *qd, fp64=True)).max() <= 2e-6
    g = oracle.antipodal_gradient(soup, ch, *q)
    h = 1e-5
    truth = np.zeros_like(g, dtype=np.float64)
    for ax in range(3):
        def cd(step):
            p, m = qd.copy(), qd.copy()
            p[ax] += step
            m[ax] -= step
            return (oracle.exact_winding(soup, *p, fp64=True) - oracle.exact_winding(soup, *m, fp64=True)) / (2 * step)
        truth[:, ax] = (4 * cd(h) - cd(2 * h)) / 3
    far = oracle.mesh_distance(soup, *q) > 100 * h
    assert np.abs(g - truth).max(1)[far].max() <= 1e-4
