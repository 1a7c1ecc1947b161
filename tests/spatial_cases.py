"""Known-answer cases of the distance and ray queries, restated from smallgwn's
tests/unit_gwn_query_distance_ray.cu (the analytic meshes and the expected values those tests
assert). Shared by the CPU oracle tests and the GPU parity tests.

Each ray case: (ox, oy, oz, dx, dy, dz, t_min, t_max) -> expected (status, t, primitive_id) with a
tolerance on t; each distance case: (qx, qy, qz, band) -> expected distance.
"""
from __future__ import annotations

import numpy as np

INF = float("inf")
INVALID = 0xFFFFFFFF


def layered(n: int, x_scale: float = 1.0) -> dict:
    """n unit right triangles stacked at z = 0, 1, ..., n-1 (unit_gwn_query_distance_ray.cu:38-57)."""
    x, y, z, i0, i1, i2 = [], [], [], [], [], []
    for t in range(n):
        v = len(x)
        x += [0.0, 1.0 * x_scale, 0.0]
        y += [0.0, 0.0, 1.0]
        z += [float(t)] * 3
        i0.append(v)
        i1.append(v + 1)
        i2.append(v + 2)
    return {"x": np.array(x, np.float32), "y": np.array(y, np.float32), "z": np.array(z, np.float32),
            "i0": np.array(i0, np.uint32), "i1": np.array(i1, np.uint32), "i2": np.array(i2, np.uint32)}


def tiny_triangle(scale: float) -> dict:
    """One right triangle of leg `scale` in the z = 0 plane (:318-377)."""
    return {"x": np.array([0, scale, 0], np.float32), "y": np.array([0, 0, scale], np.float32),
            "z": np.zeros(3, np.float32), "i0": np.array([0], np.uint32), "i1": np.array([1], np.uint32),
            "i2": np.array([2], np.uint32)}


def octahedron() -> dict:
    """The oblique-hit octahedron of :408-431."""
    return {"x": np.array([1, -1, 0, 0, 0, 0], np.float32), "y": np.array([0, 0, 1, -1, 0, 0], np.float32),
            "z": np.array([0, 0, 0, 0, 1, -1], np.float32),
            "i0": np.array([0, 2, 1, 3, 2, 1, 3, 0], np.uint32), "i1": np.array([2, 1, 3, 0, 0, 2, 1, 3], np.uint32),
            "i2": np.array([4, 4, 4, 4, 5, 5, 5, 5], np.uint32)}


def unit_quad() -> dict:
    """Two triangles sharing the diagonal of the unit square (:433-456)."""
    return {"x": np.array([0, 1, 1, 0], np.float32), "y": np.array([0, 0, 1, 1], np.float32),
            "z": np.zeros(4, np.float32), "i0": np.array([0, 0], np.uint32), "i1": np.array([1, 2], np.uint32),
            "i2": np.array([2, 3], np.uint32)}


# (name, mesh factory, builder "lbvh"/"hploc", stack capacity, rays, distances)
# ray: ((ox, oy, oz, dx, dy, dz, t_min, t_max), (status, t, primitive_id, t_tol, uv))
# distance: ((qx, qy, qz, band), expected)
CASES = [
    ("leaf_root", lambda: layered(1), "lbvh", 64,
     [((0.25, 0.25, 1, 0, 0, -1, 0, INF), (1, 1.0, 0, 0.0, (0.25, 0.25, 1e-6))),
      ((0.25, 0.25, 1, 0, 0, -1, 1, 1), (1, 1.0, 0, 0.0, None)),
      ((0.25, 0.25, 1, 0, 0, 0, 0, 10), (0, -1.0, INVALID, 0.0, None)),
      ((0.25, 0.25, 1, 1e-30, 0, -1, 0, 2), (1, 1.0, 0, 1e-6, None)),
      ((0.25, 0.25, 0, 1, 0, 0, 0, 2), (0, -1.0, INVALID, 0.0, None)),
      ((0.25, 0.25, 1e-6, 0, 0, -1, 0, 1e-5), (1, 1e-6, 0, 1e-10, None))],
     [((0.25, 0.25, 2, INF), 2.0), ((2, 0, 0, INF), 1.0), ((0.25, 0.25, 2, 0.5), 0.5),
      ((0.25, 0.25, 2, -4), 0.0)]),
    ("tiny_1e-10", lambda: tiny_triangle(1e-10), "lbvh", 64,
     [((0.25e-10, 0.25e-10, 1, 0, 0, -1, 0, 2), (1, 1.0, 0, 1e-6, (0.25, 0.25, 1e-6)))], []),
    ("subnormal_1e-20", lambda: tiny_triangle(1e-20), "lbvh", 64,
     [((0.25e-20, 0.25e-20, 1, 0, 0, -1, 0, 2), (1, 1.0, 0, 0.0, (0.25, 0.25, 1e-5)))], []),
    ("layered_12_lbvh", lambda: layered(12), "lbvh", 64,
     [((0.25, 0.25, 20, 0, 0, -1, 0, INF), (1, 9.0, 11, 0.0, None)),
      ((2, 2, 20, 0, 0, -1, 0, INF), (0, -1.0, INVALID, 0.0, None)),
      ((0, 0.25, 20, 0, 0, -1, 0, INF), (1, 9.0, 11, 0.0, None))],
     [((0.25, 0.25, 10.25, 2), 0.25), ((0.25, 0.25, 30, 2), 2.0), ((0, 0.25, 10.25, 2), 0.25)]),
    ("layered_12_hploc", lambda: layered(12), "hploc", 64,
     [((0.25, 0.25, 20, 0, 0, -1, 0, INF), (1, 9.0, 11, 0.0, None)),
      ((2, 2, 20, 0, 0, -1, 0, INF), (0, -1.0, INVALID, 0.0, None)),
      ((0, 0.25, 20, 0, 0, -1, 0, INF), (1, 9.0, 11, 0.0, None))],
     [((0.25, 0.25, 10.25, 2), 0.25), ((0.25, 0.25, 30, 2), 2.0), ((0, 0.25, 10.25, 2), 0.25)]),
    ("octahedron", octahedron, "hploc", 64,
     [((2, 2, 2, -1, -1, -1, 0, INF), (1, 5.0 / 3.0, 0, 1e-5, None)),
      ((2, 0.2, 0.1, -1, 0, 0, 0, INF), (1, 1.3, 0, 1e-5, None)),
      ((2, 2, 2, 1, 1, 1, 0, INF), (0, -1.0, INVALID, 0.0, None))],
     [((0, 0, 0, INF), float(1 / np.sqrt(3)))]),
    # the grazing hit on the shared diagonal: smallgwn accepts either triangle, the lower id wins here
    ("shared_edge", unit_quad, "hploc", 64,
     [((0.5, 0.5, 1, 0, 0, -1, 0, 2), (1, 1.0, 0, 0.0, None))],
     [((0.5, 0.5, 0, INF), 0.0)]),
    ("thin_bounds", lambda: layered(16, 1e-25), "hploc", 64,
     [((0.25e-25, 0.25, -1, 0, 0, 1, 0.5, 2), (1, 1.0, 0, 0.0, None))], []),
    ("negative_entry", lambda: layered(16), "hploc", 64,
     [((0.25, 0.25, 20, 0, 0, 1, -30, 0), (1, -20.0, 0, 0.0, None))], []),
    ("leaf_children_capacity_1", lambda: layered(4), "lbvh", 1,
     [((0.25, 0.25, 5, 0, 0, -1, 0, INF), (1, 2.0, 3, 0.0, None))],
     [((0.25, 0.25, 3.5, INF), 0.5)]),
]
