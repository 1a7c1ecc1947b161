"""Seeded synthetic meshes and query sets for the benchmark workloads (numpy, host side).

All inputs are synthetic; seeds are fixed per workload and use numpy's PCG64 generator.

Workloads
  small   : icosphere, 4 subdivisions (2,562 vertices, 5,120 triangles), unit radius, vertices
            scaled radially by 1 + N(0, 0.01) (seed 0); 100,000 queries uniform in [-1.5, 1.5]^3
            (seed 1).
  sphere  : UV-sphere grid n_phi x n_theta (1024 x 512 -> 1,046,528 triangles), radius
            r(theta, phi) = 1 + 0.1 sum_k a_k sin(m_k theta + p_k) cos(n_k phi + q_k), k = 1..8,
            a_k ~ U(0,1)/k, m_k, n_k integers in [1, 12], phases U[0, 2 pi) (seed 2); queries: half
            uniform in the bounding box scaled by 1.2, half at a surface sample offset along the
            triangle normal by N(0, 1e-3).
  soup    : the displaced sphere on a 316 x 316 grid with 20% of triangles deleted and 5%
            flipped (seed 3).
"""
from __future__ import annotations

import numpy as np


def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere with `level` midpoint subdivisions. Returns (V[n,3] float64, F[m,3] int64)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int64)


def displaced_radius(theta, phi, seed: int) -> np.ndarray:
    """r(theta, phi) = 1 + 0.1 sum_k a_k sin(m_k theta + p_k) cos(n_k phi + q_k), k = 1..8, with
    a_k ~ U(0, 1) / k, integer m_k, n_k in [1, 12] and phases ~ U[0, 2 pi), all drawn from seed."""
    rng = np.random.default_rng(seed)
    k = np.arange(1, 9)
    a = rng.uniform(0.0, 1.0, 8) / k
    m = rng.integers(1, 13, 8)
    n = rng.integers(1, 13, 8)
    p = rng.uniform(0.0, 2.0 * np.pi, 8)
    q = rng.uniform(0.0, 2.0 * np.pi, 8)
    theta = np.asarray(theta, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    s = np.zeros(np.broadcast(theta, phi).shape)
    for i in range(8):
        s += a[i] * np.sin(m[i] * theta + p[i]) * np.cos(n[i] * phi + q[i])
    return 1.0 + 0.1 * s


def uv_sphere(n_phi: int, n_theta: int, seed: int, displaced: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Displaced UV sphere: n_theta rings from pole to pole (poles included), n_phi vertices per
    ring, wrapped in phi; 2 * n_phi * (n_theta - 1) outward-oriented triangles."""
    theta = np.linspace(0.0, np.pi, n_theta)
    phi = np.arange(n_phi) * (2.0 * np.pi / n_phi)
    th, ph = np.meshgrid(theta, phi, indexing="ij")  # [n_theta, n_phi]
    r = displaced_radius(th, ph, seed) if displaced else np.ones_like(th)
    V = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], axis=-1).reshape(-1, 3)
    j = np.arange(n_theta - 1)[:, None]
    i = np.arange(n_phi)[None, :]
    i1 = (i + 1) % n_phi
    v00 = j * n_phi + i
    v01 = j * n_phi + i1
    v10 = (j + 1) * n_phi + i
    v11 = (j + 1) * n_phi + i1
    # outward orientation (theta grows downward from +z)
    t0 = np.stack([v00, v10, v11], axis=-1).reshape(-1, 3)
    t1 = np.stack([v00, v11, v01], axis=-1).reshape(-1, 3)
    F = np.empty((t0.shape[0] * 2, 3), dtype=np.int64)
    F[0::2] = t0
    F[1::2] = t1
    return V, F


def to_soa(V: np.ndarray, F: np.ndarray) -> dict:
    V32 = np.ascontiguousarray(V, dtype=np.float32)
    F32 = np.ascontiguousarray(F, dtype=np.uint32)
    return {"x": np.ascontiguousarray(V32[:, 0]), "y": np.ascontiguousarray(V32[:, 1]),
            "z": np.ascontiguousarray(V32[:, 2]), "i0": np.ascontiguousarray(F32[:, 0]),
            "i1": np.ascontiguousarray(F32[:, 1]), "i2": np.ascontiguousarray(F32[:, 2])}


def small_mesh() -> dict:
    V, F = icosphere(4)
    rng = np.random.default_rng(0)
    V = V * (1.0 + rng.normal(0.0, 0.01, size=(V.shape[0], 1)))
    return to_soa(V, F)


def small_queries(n: int = 100_000) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    rng = np.random.default_rng(1)
    q = rng.uniform(-1.5, 1.5, size=(n, 3)).astype(np.float32)
    return tuple(np.ascontiguousarray(q[:, k]) for k in range(3))


def sphere_mesh(n_phi: int = 1024, n_theta: int = 512, seed: int = 2) -> dict:
    V, F = uv_sphere(n_phi, n_theta, seed)
    return to_soa(V, F)


def triangle_normals(mesh: dict) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=-1).astype(np.float64)
    a, b, c = P[mesh["i0"]], P[mesh["i1"]], P[mesh["i2"]]
    n = np.cross(b - a, c - a)
    area2 = np.linalg.norm(n, axis=1)
    return a, b, c, n, area2


def mixed_queries(mesh: dict, n: int, seed: int, offset_sigma: float = 1e-3,
                  log_offsets: tuple[float, float] | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Half uniform in the bounding box scaled by 1.2 about its centre, half at surface samples
    offset along the unit triangle normal by N(0, offset_sigma) (or by a log-uniform magnitude in
    `log_offsets` with a random sign). Surface samples pick non-degenerate triangles uniformly."""
    rng = np.random.default_rng(seed)
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=-1).astype(np.float64)
    lo, hi = P.min(axis=0), P.max(axis=0)
    ctr, half = (lo + hi) * 0.5, (hi - lo) * 0.5 * 1.2
    n_uni = n // 2
    n_srf = n - n_uni
    out = np.empty((n, 3), dtype=np.float64)
    out[:n_uni] = ctr + rng.uniform(-1.0, 1.0, size=(n_uni, 3)) * half
    a, b, c, nrm, area2 = triangle_normals(mesh)
    good = np.flatnonzero(area2 > 0)
    tri = good[rng.integers(0, good.size, size=n_srf)]
    u = rng.uniform(0.0, 1.0, size=(n_srf, 2))
    flip = u.sum(axis=1) > 1.0
    u[flip] = 1.0 - u[flip]
    pt = a[tri] + u[:, :1] * (b[tri] - a[tri]) + u[:, 1:] * (c[tri] - a[tri])
    unit = nrm[tri] / area2[tri, None]
    if log_offsets is None:
        off = rng.normal(0.0, offset_sigma, size=(n_srf, 1))
    else:
        mag = np.exp(rng.uniform(np.log(log_offsets[0]), np.log(log_offsets[1]), size=(n_srf, 1)))
        off = mag * np.where(rng.uniform(size=(n_srf, 1)) < 0.5, -1.0, 1.0)
    out[n_uni:] = pt + off * unit
    perm = rng.permutation(n)
    out = out[perm].astype(np.float32)
    return tuple(np.ascontiguousarray(out[:, k]) for k in range(3))


class SurfaceSampler:
    """Queries at surface samples offset along the unit normal by a log-uniform magnitude in
    [lo, hi] of random sign (the precision-stress query set); triangles are picked uniformly among
    non-degenerate ones. `sample(n, seed)` returns (qx, qy, qz, signed offsets)."""

    def __init__(self, mesh: dict, lo: float = 1e-6, hi: float = 1e-1) -> None:
        a, b, c, nrm, area2 = triangle_normals(mesh)
        good = np.flatnonzero(area2 > 0)
        self.a, self.ab, self.ac = a[good], (b - a)[good], (c - a)[good]
        self.unit = nrm[good] / area2[good, None]
        self.lo, self.hi = lo, hi

    def sample(self, n: int, seed: int):
        rng = np.random.default_rng(seed)
        tri = rng.integers(0, self.a.shape[0], size=n)
        u = rng.uniform(0.0, 1.0, size=(n, 2))
        flip = u.sum(axis=1) > 1.0
        u[flip] = 1.0 - u[flip]
        mag = np.exp(rng.uniform(np.log(self.lo), np.log(self.hi), size=n))
        off = mag * np.where(rng.uniform(size=n) < 0.5, -1.0, 1.0)
        out = self.a[tri] + u[:, :1] * self.ab[tri] + u[:, 1:] * self.ac[tri] + off[:, None] * self.unit[tri]
        out = out.astype(np.float32)
        return (np.ascontiguousarray(out[:, 0]), np.ascontiguousarray(out[:, 1]), np.ascontiguousarray(out[:, 2]),
                off)


def soup_mesh(n: int = 316, seed: int = 3, delete_frac: float = 0.2, flip_frac: float = 0.05) -> dict:
    V, F = uv_sphere(n, n, seed)
    rng = np.random.default_rng(seed)
    keep = rng.uniform(size=F.shape[0]) >= delete_frac
    F = F[keep]
    flip = rng.uniform(size=F.shape[0]) < flip_frac
    F[flip] = F[flip][:, [0, 2, 1]]
    return to_soa(V, F)


def reference_mixed_queries(mesh: dict, n: int, seed: int = 0xB3A9E5D4) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The mix of smallgwn's benchmark harness (tests/benchmark_utils.cuh:136-208): the box centre,
    then 70% near-field points centre + U(-0.85, 0.85) * extent and 30% far-field points
    centre + (+-U(1.5, 3) + U(-0.25, 0.25)) * extent, drawn here from numpy's PCG64."""
    rng = np.random.default_rng(seed & 0xFFFFFFFFFFFFFFFF)
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=-1).astype(np.float32)
    lo, hi = P.min(axis=0), P.max(axis=0)
    ctr = (lo + hi) * 0.5
    ext = np.maximum(hi - lo, 1e-3)
    out = np.empty((n, 3), dtype=np.float32)
    out[0] = ctr
    idx = np.arange(1, n)
    near = (idx % 10) < 7
    nn = int(near.sum())
    out[1:][near] = ctr + rng.uniform(-0.85, 0.85, size=(nn, 3)) * ext
    nf = n - 1 - nn
    sign = np.where(rng.integers(0, 2, size=(nf, 3)) == 0, -1.0, 1.0)
    out[1:][~near] = ctr + (sign * rng.uniform(1.5, 3.0, size=(nf, 3)) + rng.uniform(-0.25, 0.25, size=(nf, 3))) * ext
    return tuple(np.ascontiguousarray(out[:, k]) for k in range(3))


def _normalize_or(v: np.ndarray, fallback: np.ndarray) -> np.ndarray:
    """Rows of v scaled to unit length; rows of zero (or non-finite) length take `fallback`'s row."""
    n2 = np.einsum("ij,ij->i", v, v)
    good = n2 > 0
    out = np.array(fallback, dtype=v.dtype, copy=True)
    out[good] = v[good] / np.sqrt(n2[good])[:, None]
    return out


def reference_mixed_rays(mesh: dict, n: int, seed: int = 0xB3A9E5D4) -> tuple[np.ndarray, ...]:
    """The ray mix of smallgwn's benchmark harness (tests/benchmark_utils.cuh:210-370) as
    (ox, oy, oz, dx, dy, dz), drawn here from numpy's PCG64: rays 4k and 4k + 1 start at the centroid
    of triangle (ray id mod T) offset by U(0.2, 0.45) x the largest extent along its unit normal (to
    the front for even ids, the back for odd ones) and point at the centroid (4k) or away from it
    (4k + 1), jittered by U(-0.08, 0.08) times a random unit vector; rays 4k + 2 and 4k + 3 start on a
    shell at U(1.6, 3.2) extents from the box centre, 4k + 2 aimed inward with jitter (hit-biased),
    4k + 3 grazing: 0.2 inward + 0.8 of a unit tangent."""
    P = np.stack([mesh["x"], mesh["y"], mesh["z"]], axis=-1).astype(np.float32)
    lo, hi = P.min(axis=0), P.max(axis=0)
    ctr = (lo + hi) * np.float32(0.5)
    ext = np.maximum(hi - lo, np.float32(1e-3))
    ext_max = np.float32(ext.max())
    rng = np.random.default_rng((seed ^ 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF)
    ids = np.arange(n, dtype=np.int64)
    o = np.empty((n, 3), np.float32)
    d = np.empty((n, 3), np.float32)

    def unit(k):
        return _normalize_or(rng.uniform(-1, 1, size=(k, 3)).astype(np.float32),
                             np.tile(np.float32([1, 0, 0]), (k, 1)))

    T = int(mesh["i0"].size)
    tri_rays = ((ids % 4) < 2) & (T > 0)
    k = int(tri_rays.sum())
    if k:
        sel = ids[tri_rays]
        t = sel % T
        a, b, c = (P[np.asarray(mesh[f"i{j}"])[t].astype(np.int64)] for j in range(3))
        cen = (a + b + c) / np.float32(3)
        nrm = np.cross(b - a, c - a).astype(np.float32)
        ru = unit(k)
        nrm = _normalize_or(nrm, ru)
        side = np.where((sel & 1) == 0, np.float32(1), np.float32(-1))[:, None]
        off = rng.uniform(0.2, 0.45, size=(k, 1)).astype(np.float32) * ext_max
        org = cen + side * off * nrm
        dr = cen - org
        dr[(sel % 4) == 1] *= -1
        dr = dr + rng.uniform(-0.08, 0.08, size=(k, 3)).astype(np.float32) * ru
        o[tri_rays], d[tri_rays] = org, _normalize_or(dr, -side * nrm)
    m = n - k
    if m:
        sel = ids[~tri_rays]
        outward = unit(m)
        shell = rng.uniform(1.6, 3.2, size=(m, 1)).astype(np.float32)
        org = ctr + outward * shell * ext
        inward = _normalize_or(ctr - org, np.tile(np.float32([0, 0, 1]), (m, 1)))
        j = unit(m)
        jit = rng.uniform(-0.08, 0.08, size=(m, 3)).astype(np.float32)
        tang = _normalize_or(np.cross(inward, j).astype(np.float32), np.tile(np.float32([1, 0, 0]), (m, 1)))
        dr = np.where(((sel % 4) == 2)[:, None], inward + jit * j, np.float32(0.2) * inward + np.float32(0.8) * tang)
        o[~tri_rays], d[~tri_rays] = org, _normalize_or(dr.astype(np.float32), inward)
    return tuple(np.ascontiguousarray(a[:, i]) for a in (o, d) for i in range(3))
