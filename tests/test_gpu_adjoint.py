"""GPU checks of the Taylor adjoint (gwnb_winding_taylor_forward_f32 / _backward_f32).

The backward pass gives dL/dV and dL/dq of L = sum_q g_q w(q). Checked against:
  * FP64 central differences (Richardson-extrapolated with steps H and H / 2) of the oracle's FP64
    Taylor sum with the float traversal's acceptance decisions frozen -- the piecewise-smooth
    function the adjoint differentiates -- on an open, inconsistently oriented soup (20 % of the
    triangles deleted, 5 % flipped), 64 random vertices and 64 random queries, for the loss over
    the queries the stencil cannot reach across the surface;
  * FP64 central differences of the exact winding number when every slot is descended;
  * the library's Taylor gradient batch and smallgwn's own Taylor query gradient
    (include/gwn/gwn_query.cuh:688-756) for dL/dq = g grad w.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import smallgwn_b200 as g
from smallgwn_b200 import api, meshes

pytestmark = pytest.mark.gpu

# Step of the central differences. Richardson extrapolation leaves an error of about
# 120 (H / d)^4 for a query at distance d from the surface, so the losses below keep only queries
# farther than CLEARANCE * H (relative error below 2e-4).
H = 1e-5
CLEARANCE = 30.0


def setup(cuda, mesh, order, nq, seed, method=g.gwn_bvh_build_method.k_hploc):
    geo = g.gwn_geometry_object()
    assert g.gwn_upload_geometry(geo, mesh["x"], mesh["y"], mesh["z"], mesh["i0"], mesh["i1"], mesh["i2"]).is_ok()
    bvh = g.gwn_bvh4_object()
    assert g.gwn_build_bvh(geo, bvh, g.gwn_bvh_build_options(method=method)).is_ok()
    mom = g.gwn_bvh4_moment_object(order)
    assert g.gwn_refit_bvh_moment(order, bvh, mom).is_ok()
    q = meshes.mixed_queries(mesh, nq, seed=seed)
    w = np.random.default_rng(seed + 1).normal(size=nq).astype(np.float32)
    return geo, bvh, mom, q, w


def run_adjoint(cuda, order, geo, bvh, mom, q, w, beta, **kw):
    d = [cuda.from_numpy(np.ascontiguousarray(v, np.float32)).cuda() for v in q]
    out = cuda.empty_like(d[0])
    st, saved = g.gwn_winding_taylor_forward(order, bvh, mom, *d, out, accuracy_scale=beta, **kw)
    assert st.is_ok(), st.message
    gout = cuda.from_numpy(w).cuda()
    nv = geo.vertex_count()
    dv =[cuda.empty(nv, device="cuda") for _ in range(3)]
    dq = [cuda.empty(len(w), device="cuda") for _ in range(3)]
    st = g.gwn_winding_taylor_backward(saved, geo, bvh, mom, gout, *dv, *dq)
    assert st.is_ok(), st.message
    assert api.sync_bvh_status(bvh).is_ok()
    cuda.cuda.synchronize()
    return (out.cpu().numpy(), np.stack([x.cpu().numpy() for x in dv], -1),
            np.stack([x.cpu().numpy() for x in dq], -1), d)


def richardson(f, h=H):
    """Central difference with Richardson extrapolation: (4 D(h/2) - D(h)) / 3."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def rel_error(adj, fd):
    """Per-sample relative error with a floor of 1 % of the largest derivative of the set."""
    floor = 1e-2 * np.max(np.abs(fd))
    return np.abs(adj - fd) / np.maximum(np.abs(fd), floor)


@pytest.mark.parametrize("order", [0, 1])
def test_adjoint_matches_fp64_central_differences(cuda, order):
    mesh = meshes.soup_mesh(40, seed=13)
    geo, bvh, mom, q, w = setup(cuda, mesh, order, 2000, seed=21)
    # The winding number jumps by 1 across a triangle: a query within the stencil's reach of the
    # surface (a vertex or the query moving by h) has no central difference there. Such queries
    # keep g = 0 (vertex differences) and are not sampled (query differences).
    far = oracle.mesh_distance(mesh, *q) > CLEARANCE * H
    w = np.where(far, w, 0.0).astype(np.float32)
    beta = 2.0
    _, dv, dq, _ = run_adjoint(cuda, order, geo, bvh, mom, q, w, beta)
    h = api.bvh_host_arrays(bvh)
    mh = api.moment_host_array(mom)
    V = np.stack([mesh["x"], mesh["y"], mesh["z"]], -1).astype(np.float64)
    q64 = [v.astype(np.float64) for v in q]
    w64 = w.astype(np.float64)

    def L(Vp, ev=q64, dec=q, gg=w64):
        return float(gg @ oracle.taylor_frozen_f64(order, h["nodes"], mh, h["root_reference"], Vp, mesh,
                                                   h["primitive_indices"], dec, ev, beta=beta))

    rng = np.random.default_rng(5)
    used = np.unique(np.concatenate([mesh["i0"], mesh["i1"], mesh["i2"]]))
    verts = rng.choice(used, 64, replace=False)
    fd_v = np.zeros((64, 3))
    for i, v in enumerate(verts):
        for k in range(3):
            def f(step):
                Vp = V.copy()
                Vp[v, k] += step
                return L(Vp)
            fd_v[i, k] = richardson(f)
    err_v = rel_error(dv[verts], fd_v)
    assert err_v.max() <= 1e-3, (err_v.max(), np.abs(fd_v).max())

    sel = rng.choice(np.flatnonzero(far), 64, replace=False)
    dec = [x[sel] for x in q]
    fd_q = np.zeros((64, 3))
    for k in range(3):
        def f(step):
            ev = [x[sel].astype(np.float64) for x in q]
            ev[k] = ev[k] + step
            return w64[sel] * oracle.taylor_frozen_f64(order, h["nodes"], mh, h["root_reference"], V, mesh,
                                                       h["primitive_indices"], dec, ev, beta=beta)
        fd_q[:, k] = richardson(f)
    err_q = rel_error(dq[sel], fd_q)
    assert err_q.max() <= 1e-3, (err_q.max(), np.abs(fd_q).max())


def test_adjoint_exact_limit_matches_exact_winding_differences(cuda):
    """With every slot descended the function is the exact winding number: its FP64 central
    differences (oracle brute force, no traversal involved) are an independent check."""
    mesh = meshes.soup_mesh(16, seed=3)
    geo, bvh, mom, q, w = setup(cuda, mesh, 1, 256, seed=31)
    w = np.where(oracle.mesh_distance(mesh, *q) > CLEARANCE * H, w, 0.0).astype(np.float32)
    _, dv, dq, _ = run_adjoint(cuda, 1, geo, bvh, mom, q, w, 1e6)
    q64 = [v.astype(np.float64) for v in q]
    w64 = w.astype(np.float64)
    rng = np.random.default_rng(8)
    used = np.unique(np.concatenate([mesh["i0"], mesh["i1"], mesh["i2"]]))
    verts = rng.choice(used, 16, replace=False)
    fd = np.zeros((16, 3))
    for i, v in enumerate(verts):
        for k in range(3):
            def f(step):
                m = dict(mesh)
                key = "xyz"[k]
                m[key] = mesh[key].astype(np.float64).copy()
                m[key][v] += step
                return float(w64 @ oracle.exact_winding(m, *q64, fp64=True))
            fd[i, k] = richardson(f)
    assert rel_error(dv[verts], fd).max() <= 1e-3


@pytest.mark.parametrize("order", [0, 1])
def test_adjoint_query_gradient_is_the_taylor_gradient(cuda, order):
    mesh = meshes.soup_mesh(40, seed=13)
    geo, bvh, mom, q, w = setup(cuda, mesh, order, 4000, seed=41)
    _, _, dq, d = run_adjoint(cuda, order, geo, bvh, mom, q, w, 2.0)
    gr = [cuda.empty(len(w), device="cuda") for _ in range(3)]
    assert g.gwn_compute_winding_gradient_taylor_batch(order, bvh, mom, *d, *gr, accuracy_scale=2.0).is_ok()
    cuda.cuda.synchronize()
    grad = np.stack([x.cpu().numpy() for x in gr], -1)
    ref = w[:, None] * grad
    # the same traversal and far field; the near field differentiates the atan2 form instead of
    # the Biot-Savart form
    scale = np.abs(ref).max()
    assert np.quantile(np.abs(dq - ref), 0.999) <= 1e-4 * scale
    if oracle.ref_lib() is not None:
        R = oracle.Reference(mesh)
        R.build(0, 8, 64)  # H-PLOC, radius 8, 64-bit codes: the tree of setup()
        R.moments(order)
        rg = R.taylor_gradient(order, *q, beta=2.0)
        R.close()
        # smallgwn's BVH is the same tree up to node numbering: same decisions up to rounding
        diff = np.abs(dq - w[:, None] * rg)
        assert np.mean(diff.max(axis=1) <= 1e-4 * scale) >= 0.999


def test_adjoint_contract(cuda):
    mesh = meshes.soup_mesh(16, seed=3)
    geo, bvh, mom, q, w = setup(cuda, mesh, 1, 64, seed=2)
    d = [cuda.from_numpy(np.ascontiguousarray(v, np.float32)).cuda() for v in q]
    out = cuda.empty_like(d[0])
    gout = cuda.from_numpy(w).cuda()
    # order 2 has no adjoint
    m2 = g.gwn_bvh4_moment_object(2)
    assert g.gwn_refit_bvh_moment(2, bvh, m2).is_ok()
    st, saved = g.gwn_winding_taylor_forward(2, bvh, m2, *d, out)
    assert st.error == g.gwn_error.invalid_argument and saved is None
    st, saved = g.gwn_winding_taylor_forward(1, bvh, mom, *d, out)
    assert st.is_ok()
    # skipping both outputs, or either, is allowed
    assert g.gwn_winding_taylor_backward(saved, geo, bvh, mom, gout).is_ok()
    dq = [cuda.empty(64, device="cuda") for _ in range(3)]
    assert g.gwn_winding_taylor_backward(saved, None, bvh, mom, gout, None, None, None, *dq).is_ok()
    # a partial output triple is refused
    st = g.gwn_winding_taylor_backward(saved, geo, bvh, mom, gout, dq[0], None, None)
    assert st.error == g.gwn_error.invalid_argument
    # a refit after the forward pass invalidates its saved state
    assert g.gwn_refit_bvh(geo, bvh).is_ok()
    assert g.gwn_refit_bvh_moment(1, bvh, mom).is_ok()
    st = g.gwn_winding_taylor_backward(saved, geo, bvh, mom, gout, None, None, None, *dq)
    assert st.error == g.gwn_error.invalid_argument and "changed" in st.message
    cuda.cuda.synchronize()


def test_autograd_function_matches_the_c_abi_pair(cuda):
    from smallgwn_b200.autograd import WindingField, winding_number

    mesh = meshes.soup_mesh(24, seed=5)
    faces = np.stack([mesh["i0"], mesh["i1"], mesh["i2"]], -1)
    V = cuda.from_numpy(np.stack([mesh["x"], mesh["y"], mesh["z"]], -1).astype(np.float32)).cuda()
    field = WindingField(V, faces, order=1, accuracy_scale=2.0)
    q = meshes.mixed_queries(mesh, 1000, seed=6)
    Q = cuda.from_numpy(np.stack(q, -1).astype(np.float32)).cuda()
    wts = cuda.from_numpy(np.random.default_rng(1).normal(size=1000).astype(np.float32)).cuda()
    Vp = V.clone().requires_grad_(True)
    Qp = Q.clone().requires_grad_(True)
    out = winding_number(Vp, Qp, field)
    (wts * out).sum().backward()
    ref_out, dv, dq, _ = run_adjoint(cuda, 1, field.geometry, field.bvh, field.moment, q, wts.cpu().numpy(), 2.0)
    np.testing.assert_allclose(out.detach().cpu().numpy(), ref_out, atol=1e-6)
    scale_v = np.abs(dv).max()
    assert np.abs(Vp.grad.cpu().numpy() - dv).max() <= 1e-4 * scale_v
    assert np.abs(Qp.grad.cpu().numpy() - dq).max() <= 1e-4 * np.abs(dq).max()


def test_adjoint_on_the_differentiation_workload_with_step_sweep(cuda):
    """The differentiation workload itself: the 316 x 316 displaced sphere with 20 % of the triangles
    deleted and 5 % flipped (seed 3; 159,242 triangles), order 1, accuracy scale 2, 64 random vertices
    and 64 random queries, losses over 2,048 of its mixed queries farther than 3e-3 from the surface.

    Against FP64 central differences of the frozen-decision Taylor sum, per element, relative error
    with a floor of 1 % of the largest derivative. At the configured step h = 1e-4 the differences
    themselves are not converged for vertex derivatives: their truncation (measured here as the gap
    to the differences at 1e-6, which agree with those at 1e-5 to a few 1e-6) reaches the 1e-2 range,
    so h = 1e-4 cannot check 1e-3. The step sweep shows it: the adjoint matches the converged
    differences (h = 1e-5 and 1e-6) within 1e-3 on every element, and wherever it misses the h = 1e-4
    differences by more than 1e-3, those differences miss the converged ones by as much. Query
    derivatives converge at every step and match within 1e-3 at h = 1e-4 as configured."""
    mesh = meshes.soup_mesh(316, seed=3)
    order, beta = 1, 2.0
    geo, bvh, mom, q, w = setup(cuda, mesh, order, 8000, seed=3)
    dist = oracle.mesh_distance(mesh, *q)
    far = np.flatnonzero(dist > 3e-3)[:2048]
    ws = np.zeros_like(w)
    ws[far] = w[far]
    _, dv, dq, _ = run_adjoint(cuda, order, geo, bvh, mom, q, ws, beta)
    hb, mh = api.bvh_host_arrays(bvh), api.moment_host_array(mom)
    V = np.stack([mesh["x"], mesh["y"], mesh["z"]], -1).astype(np.float64)
    dec = [x[far] for x in q]
    ev0 = [x[far].astype(np.float64) for x in q]
    wf = w[far].astype(np.float64)

    def frozen(Vp, ev, d=dec):
        return oracle.taylor_frozen_f64(order, hb["nodes"], mh, hb["root_reference"], Vp, mesh,
                                        hb["primitive_indices"], d, ev, beta=beta)

    rng = np.random.default_rng(5)
    used = np.unique(np.concatenate([mesh["i0"], mesh["i1"], mesh["i2"]]))
    verts = rng.choice(used, 64, replace=False)
    sel = rng.choice(far.size, 64, replace=False)

    def fd_vertices(h):
        out = np.zeros((64, 3))
        for i, v in enumerate(verts):
            for k in range(3):
                def f(s, v=v, k=k):
                    Vp = V.copy()
                    Vp[v, k] += s
                    return float(wf @ frozen(Vp, ev0))
                out[i, k] = richardson(f, h)
        return out

    def fd_queries(h):
        out = np.zeros((64, 3))
        for k in range(3):
            def f(s, k=k):
                ev = [x[sel].copy() for x in ev0]
                ev[k] = ev[k] + s
                return wf[sel] * frozen(V, ev, [x[sel] for x in dec])
            out[:, k] = richardson(f, h)
        return out

    fdv = {h: fd_vertices(h) for h in (1e-4, 1e-5, 1e-6)}
    adj_v = dv[verts]
    conv = fdv[1e-6]
    assert rel_error(fdv[1e-5], conv).max() <= 1e-4  # the differences have converged by 1e-5
    assert rel_error(adj_v, conv).max() <= 1e-3
    assert rel_error(adj_v, fdv[1e-5]).max() <= 1e-3
    miss = rel_error(adj_v, fdv[1e-4])
    trunc = rel_error(fdv[1e-4], conv)
    bad = miss > 1e-3
    assert np.all(trunc[bad] >= 0.5 * miss[bad])  # every miss at h = 1e-4 is the differences' own error
    print(f"dV per-element max rel: vs FD(1e-4) {miss.max():.3e} (FD(1e-4) vs FD(1e-6) {trunc.max():.3e}), "
          f"vs FD(1e-5) {rel_error(adj_v, fdv[1e-5]).max():.3e}, vs FD(1e-6) {rel_error(adj_v, conv).max():.3e}")
    fq = fd_queries(1e-4)
    assert rel_error(dq[far][sel], fq).max() <= 1e-3
