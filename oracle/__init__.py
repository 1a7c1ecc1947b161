"""The oracle: CPU restatement of smallgwn's winding-number path, plus smallgwn's own kernels.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline, never by the product (smallgwn_b200/). Two libraries back it:
  * _build/liboracle.so   gwn_oracle.c (C, OpenMP): exact winding FP32/FP64, Morton codes, stable
                          sort, Karras LBVH, H-PLOC, BVH4 collapse, triangle records, Taylor
                          moments and Taylor traversal with per-query counts, unsigned distance,
                          ray first hit, boundary chains and antipodal winding numbers;
  * _ref/libgwnref.so     smallgwn's CUDA implementation compiled from its headers (ref_shim.cu),
                          present when the reference project was available at build time.
Parity pins: tests/test_oracle.py checks the C restatement against analytic known answers and
against golden vectors recorded from smallgwn's own kernels (tests/golden/).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_ORACLE = None
_REF = None

NODE_DTYPE = np.dtype([("bounds", np.float32, (6,)), ("reference", np.uint64)])
BNODE_DTYPE = np.dtype((np.uint32, 4))


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        from .build import build_oracle

        path = build_oracle()
        _ORACLE = C.CDLL(str(path))
        _ORACLE.oracle_max_threads.restype = C.c_int
        _ORACLE.oracle_hploc.restype = C.c_int
        _ORACLE.oracle_collapse.restype = C.c_int
        _ORACLE.oracle_triangles.restype = C.c_int
    return _ORACLE


def ref_lib() -> C.CDLL | None:
    """smallgwn's own kernels (oracle/_ref/libgwnref.so) or None when not built."""
    global _REF
    if _REF is None:
        path = HERE / "_ref" / "libgwnref.so"
        if not path.exists():
            return None
        _REF = C.CDLL(str(path))
        _REF.ref_last_message.restype = C.c_char_p
    return _REF


_REF_CPU = None


def ref_cpu_lib() -> C.CDLL | None:
    """smallgwn's own CPU reference code (oracle/_ref/libgwnrefcpu.so) or None when not built."""
    global _REF_CPU
    if _REF_CPU is None:
        path = HERE / "_ref" / "libgwnrefcpu.so"
        if not path.exists():
            return None
        lib = C.CDLL(str(path))
        lib.refcpu_set_threads.restype = C.c_int
        lib.refcpu_set_threads.argtypes = [C.c_int]
        lib.refcpu_exact.restype = C.c_int
        lib.refcpu_exact.argtypes = [C.c_void_p] * 3 + [C.c_uint64] + [C.c_void_p] * 3 + [C.c_uint64] + \
            [C.c_void_p] * 3 + [C.c_uint64, C.c_void_p]
        lib.refcpu_hdk_create.restype = C.c_void_p
        lib.refcpu_hdk_create.argtypes = [C.c_void_p] * 3 + [C.c_uint64] + [C.c_void_p] * 3 + [C.c_uint64, C.c_int]
        lib.refcpu_hdk_query.restype = C.c_int
        lib.refcpu_hdk_query.argtypes = [C.c_void_p] * 4 + [C.c_uint64, C.c_float, C.c_void_p]
        lib.refcpu_hdk_destroy.argtypes = [C.c_void_p]
        _REF_CPU = lib
    return _REF_CPU


def reference_cpu_exact(mesh: dict, qx, qy, qz, threads: int = 0) -> np.ndarray:
    """smallgwn's own CPU exact brute force (tests/reference_cpu.cuh:84-114), FP32."""
    lib = ref_cpu_lib()
    lib.refcpu_set_threads(int(threads))
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    q = [_f32(v) for v in (qx, qy, qz)]
    out = np.empty(q[0].size, np.float32)
    if lib.refcpu_exact(_p(x), _p(y), _p(z), x.size, _p(i0), _p(i1), _p(i2), i0.size, _p(q[0]), _p(q[1]), _p(q[2]),
                        out.size, _p(out)) != 0:
        raise RuntimeError("reference CPU exact batch failed")
    return out


class ReferenceHDK:
    """smallgwn's CPU Taylor path: the vendored SideFX HDK solid-angle tree of a mesh
    (tests/reference_hdk.cuh:18-89), built once, queried at an accuracy scale."""

    def __init__(self, mesh: dict, order: int, threads: int = 0):
        self.lib = ref_cpu_lib()
        if self.lib is None:
            raise RuntimeError("oracle/_ref/libgwnrefcpu.so is not built")
        self.threads = self.lib.refcpu_set_threads(int(threads))
        x, y, z = (_f32(mesh[k]) for k in "xyz")
        i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
        self.h = self.lib.refcpu_hdk_create(_p(x), _p(y), _p(z), x.size, _p(i0), _p(i1), _p(i2), i0.size, int(order))
        if not self.h:
            raise RuntimeError("reference HDK tree construction failed")

    def query(self, qx, qy, qz, beta: float) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        out = np.empty(q[0].size, np.float32)
        if self.lib.refcpu_hdk_query(self.h, _p(q[0]), _p(q[1]), _p(q[2]), out.size, C.c_float(beta), _p(out)) != 0:
            raise RuntimeError("reference HDK query failed")
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.refcpu_hdk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def exact_winding(mesh: dict, qx, qy, qz, threads: int = 0, fp64: bool = False) -> np.ndarray:
    """tests/reference_cpu.cuh:84-114 restated: brute-force exact winding, FP32 or FP64."""
    threads = threads or max_threads()
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    n = len(qx)
    if fp64:
        x, y, z = (np.ascontiguousarray(mesh[k], dtype=np.float64) for k in "xyz")
        q = [np.ascontiguousarray(v, dtype=np.float64) for v in (qx, qy, qz)]
        out = np.empty(n, np.float64)
        lib().oracle_exact_winding_f64(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2),
                                       C.c_uint64(i0.size), _p(q[0]), _p(q[1]), _p(q[2]), _p(out),
                                       C.c_uint64(n), C.c_int(threads))
        return out
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    q = [_f32(v) for v in (qx, qy, qz)]
    out = np.empty(n, np.float32)
    lib().oracle_exact_winding_f32(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2),
                                   C.c_uint64(i0.size), _p(q[0]), _p(q[1]), _p(q[2]), _p(out), C.c_uint64(n),
                                   C.c_int(threads))
    return out


def exact_records(tris: np.ndarray, qx, qy, qz, threads: int = 0) -> np.ndarray:
    """Exact winding over leaf-ordered records (gwn_query_winding_impl.cuh:377-389)."""
    threads = threads or max_threads()
    t = np.ascontiguousarray(tris, dtype=np.float32)
    q = [_f32(v) for v in (qx, qy, qz)]
    out = np.empty(len(q[0]), np.float32)
    lib().oracle_exact_records(_p(t), C.c_uint64(t.shape[0]), _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(len(out)),
                               _p(out), C.c_int(threads))
    return out


def morton(mesh: dict, bits: int = 64) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Triangle AABBs (nt, 6), Morton codes (uint64 storage) and scene (min, max, inv)."""
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    nt = i0.size
    aabbs = np.empty((nt, 6), np.float32)
    codes = np.empty(nt, np.uint64)
    scene = np.empty(9, np.float32)
    lib().oracle_scene_and_morton(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2), C.c_uint64(nt),
                                  C.c_int(bits), _p(aabbs), _p(codes), _p(scene))
    return aabbs, codes, scene


def sort_pairs(codes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    c = np.ascontiguousarray(codes, dtype=np.uint64)
    out = np.empty_like(c)
    ids = np.empty(c.size, np.uint32)
    lib().oracle_sort_pairs(_p(c), C.c_uint64(c.size), _p(out), _p(ids))
    return out, ids


def karras(sorted_codes: np.ndarray, bits: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    c = np.ascontiguousarray(sorted_codes, dtype=np.uint64)
    n = c.size
    nodes = np.zeros((max(n - 1, 0), 4), np.uint32)
    ip = np.empty(max(n - 1, 0), np.uint32)
    lp = np.empty(n, np.uint32)
    lib().oracle_karras(_p(c), C.c_int(bits), C.c_uint64(n), _p(nodes), _p(ip), _p(lp))
    return nodes, ip, lp


def binary_bounds(nodes: np.ndarray, leaf_aabbs: np.ndarray, root: int) -> np.ndarray:
    n = leaf_aabbs.shape[0]
    out = np.zeros((max(n - 1, 0), 6), np.float32)
    lib().oracle_binary_bounds(_p(np.ascontiguousarray(nodes, np.uint32)), C.c_uint64(n),
                               _p(np.ascontiguousarray(leaf_aabbs, np.float32)), C.c_uint32(root), _p(out))
    return out


def hploc(sorted_codes: np.ndarray, bits: int, leaf_aabbs: np.ndarray, radius: int):
    c = np.ascontiguousarray(sorted_codes, dtype=np.uint64)
    n = c.size
    nodes = np.zeros((max(n - 1, 0), 4), np.uint32)
    bounds = np.zeros((max(n - 1, 0), 6), np.float32)
    root = C.c_uint32(0)
    rc = lib().oracle_hploc(_p(c), C.c_int(bits), C.c_uint64(n), _p(np.ascontiguousarray(leaf_aabbs, np.float32)),
                            C.c_uint32(radius), _p(nodes), _p(bounds), C.byref(root))
    if rc != 0:
        raise RuntimeError("oracle H-PLOC did not converge")
    return nodes, bounds, int(root.value)


def collapse(bin_nodes: np.ndarray, bin_bounds: np.ndarray, leaf_aabbs: np.ndarray, root: int):
    n = leaf_aabbs.shape[0]
    out = np.zeros((max(n - 1, 1), 4), NODE_DTYPE)
    cnt = C.c_uint64(0)
    ib = C.c_uint32(0)
    pb = C.c_uint32(0)
    lib().oracle_collapse(_p(np.ascontiguousarray(bin_nodes, np.uint32)),
                          _p(np.ascontiguousarray(bin_bounds, np.float32)),
                          _p(np.ascontiguousarray(leaf_aabbs, np.float32)), C.c_uint64(n), C.c_uint32(root), _p(out),
                          C.byref(cnt), C.byref(ib), C.byref(pb))
    return out[: cnt.value], int(ib.value), int(pb.value)


def triangles(mesh: dict, ids: np.ndarray) -> np.ndarray:
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    ids = _u32(ids)
    out = np.zeros((ids.size, 9), np.float32)
    bad = lib().oracle_triangles(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2), C.c_uint64(i0.size),
                                 _p(ids), _p(out))
    if bad:
        raise ValueError("invalid triangle index")
    return out


def moments(order: int, nodes: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """smallgwn-layout moment nodes, shape (nodes, fields, 4)."""
    F = {0: 7, 1: 13, 2: 23}[order]
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    out = np.zeros((nd.shape[0], F, 4), np.float32)
    t = np.ascontiguousarray(tris, np.float32)
    lib().oracle_moments(C.c_int(order), _p(nd), C.c_uint64(nd.shape[0]), _p(t), C.c_uint64(t.shape[0]), _p(out))
    return out


def taylor(order: int, nodes: np.ndarray, mom: np.ndarray, tris: np.ndarray, root_ref: int, qx, qy, qz,
           beta: float = 2.0, stack_capacity: int = 256, threads: int = 0, stats: bool = False):
    """gwn_winding_taylor_impl restated; with stats also (nodes entered, far children, exact tris)."""
    threads = threads or max_threads()
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    m = np.ascontiguousarray(mom, np.float32)
    t = np.ascontiguousarray(tris, np.float32)
    q = [_f32(v) for v in (qx, qy, qz)]
    n = q[0].size
    out = np.empty(n, np.float32)
    st = np.zeros((n, 3), np.uint32) if stats else None
    lib().oracle_taylor(C.c_int(order), _p(nd), C.c_uint64(nd.shape[0]), _p(m), _p(t), C.c_uint64(t.shape[0]),
                        C.c_uint64(root_ref), _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(n), C.c_float(beta),
                        C.c_int(stack_capacity), _p(out), _p(st), C.c_int(threads))
    return (out, st) if stats else out


def taylor_frozen_f64(order: int, nodes: np.ndarray, mom: np.ndarray, root_ref: int, vertices: np.ndarray,
                      mesh: dict, primitive_indices: np.ndarray, decide, evaluate, beta: float = 2.0,
                      threads: int = 0) -> np.ndarray:
    """FP64 Taylor winding numbers (orders 0, 1) with the float traversal's acceptance decisions
    frozen: decisions from the float moment nodes `mom` at the float points `decide`, the sum in
    FP64 at the points `evaluate` with moments recomputed from the FP64 `vertices` (V, 3). Central
    differences of it are the checker of the adjoint."""
    threads = threads or max_threads()
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    m = np.ascontiguousarray(mom, np.float32)
    v = [np.ascontiguousarray(vertices[:, k], np.float64) for k in range(3)]
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    prim = _u32(primitive_indices)
    d = [_f32(x) for x in decide]
    e = [np.ascontiguousarray(x, np.float64) for x in evaluate]
    n = d[0].size
    out = np.empty(n, np.float64)
    lib().oracle_taylor_frozen_f64(C.c_int(order), _p(nd), C.c_uint64(nd.shape[0]), C.c_uint64(root_ref), _p(m),
                                   _p(v[0]), _p(v[1]), _p(v[2]), _p(i0), _p(i1), _p(i2), _p(prim),
                                   C.c_uint64(prim.size), _p(d[0]), _p(d[1]), _p(d[2]), _p(e[0]), _p(e[1]), _p(e[2]),
                                   C.c_uint64(n), C.c_float(beta), _p(out), C.c_int(threads))
    return out


def mesh_distance(mesh: dict, qx, qy, qz, threads: int = 0) -> np.ndarray:
    """Unsigned distance of each point to the mesh (FP64 brute force)."""
    threads = threads or max_threads()
    v = [np.ascontiguousarray(mesh[k], np.float64) for k in "xyz"]
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    q = [np.ascontiguousarray(x, np.float64) for x in (qx, qy, qz)]
    out = np.empty(q[0].size, np.float64)
    lib().oracle_mesh_distance_f64(_p(v[0]), _p(v[1]), _p(v[2]), C.c_uint64(v[0].size), _p(i0), _p(i1), _p(i2),
                                   C.c_uint64(i0.size), _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(q[0].size), _p(out),
                                   C.c_int(threads))
    return out


def unsigned_distance(nodes: np.ndarray, tris: np.ndarray, root_ref: int, qx, qy, qz,
                      culling_band: float = float("inf"), stack_capacity: int = 256, threads: int = 0,
                      stats: bool = False):
    """gwn_unsigned_distance_impl restated (detail/gwn_query_distance_impl.cuh:40-160); with stats
    also (internal nodes entered, triangles evaluated) per query."""
    threads = threads or max_threads()
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    t = np.ascontiguousarray(tris, np.float32)
    q = [_f32(v) for v in (qx, qy, qz)]
    n = q[0].size
    out = np.empty(n, np.float32)
    st = np.zeros((n, 2), np.uint32) if stats else None
    lib().oracle_unsigned_distance(_p(nd), C.c_uint64(nd.shape[0]), _p(t), C.c_uint64(t.shape[0]),
                                   C.c_uint64(root_ref), _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(n),
                                   C.c_float(culling_band), C.c_int(stack_capacity), _p(out), _p(st),
                                   C.c_int(threads))
    return (out, st) if stats else out


def distance_brute(tris: np.ndarray, qx, qy, qz, culling_band: float = float("inf"), threads: int = 0) -> np.ndarray:
    """Minimum over every record of the same float point-triangle distance (no traversal)."""
    threads = threads or max_threads()
    t = np.ascontiguousarray(tris, np.float32)
    q = [_f32(v) for v in (qx, qy, qz)]
    out = np.empty(q[0].size, np.float32)
    lib().oracle_distance_brute(_p(t), C.c_uint64(t.shape[0]), _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(out.size),
                                C.c_float(culling_band), _p(out), C.c_int(threads))
    return out


def boundary_chain(mesh: dict) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """detail/gwn_boundary_impl.cuh restated: (start, end, multiplicity) rows of the algebraic
    boundary of the oriented triangle chain, in ascending (low, high) vertex order."""
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    nt = C.c_uint64(i0.size)
    lib().oracle_boundary_chain.restype = C.c_uint64
    rows = int(lib().oracle_boundary_chain(_p(i0), _p(i1), _p(i2), nt, None, None, None))
    start = np.empty(rows, np.uint32)
    end = np.empty(rows, np.uint32)
    mult = np.empty(rows, np.uint64)
    lib().oracle_boundary_chain(_p(i0), _p(i1), _p(i2), nt, _p(start), _p(end), _p(mult))
    return start, end, mult


def antipodal(mesh: dict, nodes: np.ndarray, tris: np.ndarray, root_ref: int, chain, qx, qy, qz,
              stack_capacity: int = 256, threads: int = 0) -> np.ndarray:
    """gwn_winding_number_antipodal_impl restated (detail/gwn_query_winding_antipodal_impl.cuh:
    380-568): signed +axis ray crossings through the BVH plus the boundary spherical-area term,
    axes z, x, y until one is not singular; NaN when none is."""
    threads = threads or max_threads()
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    t = np.ascontiguousarray(tris, np.float32)
    s, e, m = (np.ascontiguousarray(a) for a in chain)
    q = [_f32(v) for v in (qx, qy, qz)]
    out = np.empty(q[0].size, np.float32)
    lib().oracle_antipodal(_p(x), _p(y), _p(z), _p(nd), C.c_uint64(nd.shape[0]), _p(t), C.c_uint64(t.shape[0]),
                           C.c_uint64(root_ref), _p(s), _p(e), _p(m), C.c_uint64(s.size), _p(q[0]), _p(q[1]),
                           _p(q[2]), C.c_uint64(out.size), C.c_int(stack_capacity), _p(out), C.c_int(threads))
    return out


def antipodal_gradient(mesh: dict, chain, qx, qy, qz, threads: int = 0) -> np.ndarray:
    """gwn_winding_gradient_point_antipodal_impl restated (:261-372): (n, 3) gradients of the
    boundary term, NaN rows where every axis is singular."""
    threads = threads or max_threads()
    x, y, z = (_f32(mesh[k]) for k in "xyz")
    s, e, m = (np.ascontiguousarray(a) for a in chain)
    q = [_f32(v) for v in (qx, qy, qz)]
    g = [np.empty(q[0].size, np.float32) for _ in range(3)]
    lib().oracle_antipodal_gradient(_p(x), _p(y), _p(z), _p(s), _p(e), _p(m), C.c_uint64(s.size), _p(q[0]), _p(q[1]),
                                    _p(q[2]), C.c_uint64(q[0].size), _p(g[0]), _p(g[1]), _p(g[2]), C.c_int(threads))
    return np.stack(g, axis=1)


# gwn::gwn_ray_first_hit_result<float, uint32_t> (include/gwn/gwn_query.cuh:63-96), 32 bytes.
HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32), ("nx", np.float32),
                      ("ny", np.float32), ("nz", np.float32), ("primitive_id", np.uint32), ("status", np.uint8),
                      ("pad", np.uint8, (3,))])


def ray_first_hit(nodes: np.ndarray, tris: np.ndarray, primitive_indices: np.ndarray, root_ref: int, ox, oy, oz,
                  dx, dy, dz, t_min: float = 0.0, t_max: float = float("inf"), stack_capacity: int = 256,
                  threads: int = 0, stats: bool = False):
    """gwn_ray_first_hit_impl restated (detail/gwn_query_ray_impl.cuh:376-560, canonical traversal;
    equal-t hits resolved to the lower original primitive id)."""
    threads = threads or max_threads()
    nd = np.ascontiguousarray(nodes.reshape(-1, 4), dtype=NODE_DTYPE)
    t = np.ascontiguousarray(tris, np.float32)
    prim = _u32(primitive_indices)
    r = [_f32(v) for v in (ox, oy, oz, dx, dy, dz)]
    n = r[0].size
    out = np.zeros(n, HIT_DTYPE)
    st = np.zeros((n, 2), np.uint32) if stats else None
    lib().oracle_ray_first_hit(_p(nd), C.c_uint64(nd.shape[0]), _p(t), _p(prim), C.c_uint64(t.shape[0]),
                               C.c_uint64(root_ref), *[_p(v) for v in r], C.c_uint64(n), C.c_float(t_min),
                               C.c_float(t_max), C.c_int(stack_capacity), _p(out), _p(st), C.c_int(threads))
    return (out, st) if stats else out


def ray_brute(tris: np.ndarray, primitive_indices: np.ndarray, ox, oy, oz, dx, dy, dz, t_min: float = 0.0,
              t_max: float = float("inf"), threads: int = 0) -> np.ndarray:
    """Nearest hit over every record with the same per-triangle test and tie rule (no traversal)."""
    threads = threads or max_threads()
    t = np.ascontiguousarray(tris, np.float32)
    prim = _u32(primitive_indices)
    r = [_f32(v) for v in (ox, oy, oz, dx, dy, dz)]
    out = np.zeros(r[0].size, HIT_DTYPE)
    lib().oracle_ray_brute(_p(t), _p(prim), C.c_uint64(t.shape[0]), *[_p(v) for v in r], C.c_uint64(out.size),
                           C.c_float(t_min), C.c_float(t_max), _p(out), C.c_int(threads))
    return out


def build_bvh(mesh: dict, method: str = "lbvh", bits: int = 64, radius: int = 8) -> dict:
    """build_lbvh, or the same pipeline with H-PLOC (radius) in place of Karras' builder."""
    if method == "lbvh":
        return build_lbvh(mesh, bits)
    out = build_lbvh(mesh, bits)
    if out["sorted_ids"].size > 1:
        bn, bb, root = hploc(out["sorted_codes"], bits, out["sorted_aabbs"], radius)
        nodes, ib, pb = collapse(bn, bb, out["sorted_aabbs"], root)
        out.update(binary_nodes=bn, binary_bounds=bb, nodes=nodes, internal_stack_bound=ib, packed_stack_bound=pb)
    return out


def build_lbvh(mesh: dict, bits: int = 64) -> dict:
    """Full CPU pipeline: Morton, stable sort, Karras, bounds, BVH4 collapse, triangle records."""
    aabbs, codes, scene = morton(mesh, bits)
    sc, ids = sort_pairs(codes)
    saabb = aabbs[ids]
    n = ids.size
    out = {"sorted_codes": sc, "sorted_ids": ids, "sorted_aabbs": saabb, "scene": scene}
    if n == 1:
        out.update(nodes=np.zeros((0, 4), NODE_DTYPE), internal_stack_bound=0, packed_stack_bound=0,
                   root_reference=(1 << 47) | (1 << 48))
    else:
        bn, ip, lp = karras(sc, bits)
        bb = binary_bounds(bn, saabb, 0)
        nodes, ib, pb = collapse(bn, bb, saabb, 0)
        out.update(binary_nodes=bn, binary_bounds=bb, nodes=nodes, internal_stack_bound=ib, packed_stack_bound=pb,
                   root_reference=(1 << 47))
    out["triangles"] = triangles(mesh, ids)
    return out


# ---- smallgwn's own kernels (oracle/_ref) -------------------------------------------------------


class Reference:
    """Handle on smallgwn's CUDA implementation for one mesh (needs a GPU and oracle/_ref)."""

    def __init__(self, mesh: dict):
        self.lib = ref_lib()
        if self.lib is None:
            raise RuntimeError("oracle/_ref/libgwnref.so is not built")
        self.mesh = mesh
        x, y, z = (_f32(mesh[k]) for k in "xyz")
        i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
        self._keep = (x, y, z, i0, i1, i2)
        h = C.c_void_p()
        self._check(self.lib.ref_create(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2),
                                        C.c_uint64(i0.size), C.byref(h)))
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(f"reference call failed ({rc}): {self.lib.ref_last_message().decode()}")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, method: int = 1, radius: int = 8, bits: int = 64) -> None:
        self._check(self.lib.ref_build(self.h, C.c_int(method), C.c_uint32(radius), C.c_int(bits)))

    def bvh(self) -> dict:
        nn = C.c_uint64()
        ib = C.c_uint32()
        pb = C.c_uint32()
        rr = C.c_uint64()
        rb = np.zeros(6, np.float32)
        self._check(self.lib.ref_bvh_info(self.h, C.byref(nn), C.byref(ib), C.byref(pb), C.byref(rr), _p(rb)))
        nt = self._keep[3].size
        nodes = np.zeros((nn.value, 4), NODE_DTYPE)
        prims = np.zeros(nt, np.uint32)
        tris = np.zeros((nt, 9), np.float32)
        self._check(self.lib.ref_bvh_copy(self.h, _p(nodes), _p(prims), _p(tris)))
        return {"nodes": nodes, "primitive_indices": prims, "triangles": tris, "root_reference": rr.value,
                "root_bounds": rb, "internal_stack_bound": ib.value, "packed_stack_bound": pb.value}

    def set_queries(self, qx, qy, qz) -> None:
        """Device-resident query batch for dynamic_frame."""
        q = [_f32(v) for v in (qx, qy, qz)]
        self._check(self.lib.ref_set_queries(self.h, _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(q[0].size)))

    def dynamic_frame(self, x, y, z, order: int, beta: float) -> None:
        """smallgwn's dynamic stage for one frame: host positions up, refit, moment refit, Taylor batch."""
        v = [_f32(a) for a in (x, y, z)]
        self._check(self.lib.ref_dynamic_frame(self.h, _p(v[0]), _p(v[1]), _p(v[2]), C.c_uint64(v[0].size),
                                               C.c_int(order), C.c_float(beta)))

    def refit_moments(self, order: int) -> None:
        """smallgwn's moment refit of `order` on its current BVH (kept on the device)."""
        self._check(self.lib.ref_moment(self.h, C.c_int(order)))

    def moments(self, order: int) -> np.ndarray:
        self._check(self.lib.ref_moment(self.h, C.c_int(order)))
        F = {0: 7, 1: 13, 2: 23}[order]
        nn = C.c_uint64()
        dummy = C.c_uint32()
        rr = C.c_uint64()
        rb = np.zeros(6, np.float32)
        self._check(self.lib.ref_bvh_info(self.h, C.byref(nn), C.byref(dummy), C.byref(dummy), C.byref(rr), _p(rb)))
        out = np.zeros((nn.value, F, 4), np.float32)
        self._check(self.lib.ref_moment_copy(self.h, C.c_int(order), _p(out)))
        return out

    def exact(self, qx, qy, qz) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        out = np.empty(q[0].size, np.float32)
        self._check(self.lib.ref_exact(self.h, _p(q[0]), _p(q[1]), _p(q[2]), _p(out), C.c_uint64(out.size)))
        return out

    def taylor(self, order: int, qx, qy, qz, beta: float = 2.0) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        out = np.empty(q[0].size, np.float32)
        self._check(self.lib.ref_taylor(self.h, C.c_int(order), _p(q[0]), _p(q[1]), _p(q[2]), _p(out),
                                        C.c_uint64(out.size), C.c_float(beta)))
        return out

    def taylor_gradient(self, order: int, qx, qy, qz, beta: float = 2.0) -> np.ndarray:
        """smallgwn's Taylor query gradient, shape (n, 3)."""
        q = [_f32(v) for v in (qx, qy, qz)]
        g = [np.empty(q[0].size, np.float32) for _ in range(3)]
        self._check(self.lib.ref_taylor_gradient(self.h, C.c_int(order), _p(q[0]), _p(q[1]), _p(q[2]), _p(g[0]),
                                                 _p(g[1]), _p(g[2]), C.c_uint64(q[0].size), C.c_float(beta)))
        return np.stack(g, -1)

    def time_taylor(self, order: int, qx, qy, qz, beta: float, warmup: int, iters: int) -> float:
        q = [_f32(v) for v in (qx, qy, qz)]
        ms = C.c_float()
        self._check(self.lib.ref_time_taylor(self.h, C.c_int(order), _p(q[0]), _p(q[1]), _p(q[2]),
                                             C.c_uint64(q[0].size), C.c_float(beta), C.c_int(warmup), C.c_int(iters),
                                             C.byref(ms)))
        return float(ms.value)

    def time_exact(self, qx, qy, qz, warmup: int, iters: int) -> float:
        q = [_f32(v) for v in (qx, qy, qz)]
        ms = C.c_float()
        self._check(self.lib.ref_time_exact(self.h, _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(q[0].size),
                                            C.c_int(warmup), C.c_int(iters), C.byref(ms)))
        return float(ms.value)

    def distance(self, qx, qy, qz, culling_band: float = float("inf")) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        out = np.empty(q[0].size, np.float32)
        self._check(self.lib.ref_distance(self.h, _p(q[0]), _p(q[1]), _p(q[2]), _p(out), C.c_uint64(out.size),
                                          C.c_float(culling_band)))
        return out

    def ray(self, ox, oy, oz, dx, dy, dz, t_min: float = 0.0, t_max: float = float("inf")) -> np.ndarray:
        r = [_f32(v) for v in (ox, oy, oz, dx, dy, dz)]
        out = np.zeros(r[0].size, HIT_DTYPE)
        self._check(self.lib.ref_ray(self.h, *[_p(v) for v in r], _p(out), C.c_uint64(out.size), C.c_float(t_min),
                                     C.c_float(t_max)))
        return out

    def time_spatial(self, qx, qy, qz, dirs=None, culling_band: float = float("inf"), t_min: float = 0.0,
                     t_max: float = float("inf"), warmup: int = 2, iters: int = 5) -> float:
        """Average ms of smallgwn's distance batch (dirs None) or ray batch on device-resident inputs."""
        q = [_f32(v) for v in (qx, qy, qz)]
        d = [_f32(v) for v in dirs] if dirs is not None else q
        ms = C.c_float()
        self._check(self.lib.ref_time_spatial(self.h, C.c_int(1 if dirs is not None else 0), *[_p(v) for v in q],
                                              *[_p(v) for v in d], C.c_uint64(q[0].size), C.c_float(culling_band),
                                              C.c_float(t_min), C.c_float(t_max), C.c_int(warmup), C.c_int(iters),
                                              C.byref(ms)))
        return float(ms.value)

    def boundary(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """smallgwn's boundary chain of this mesh (rows as its kernels emit them)."""
        cnt = C.c_uint64()
        self._check(self.lib.ref_boundary(self.h, None, None, None, C.byref(cnt)))
        n = cnt.value
        s, e, m = np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, np.uint64)
        self._check(self.lib.ref_boundary(self.h, _p(s), _p(e), _p(m), C.byref(cnt)))
        return s, e, m

    def antipodal(self, qx, qy, qz) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        out = np.empty(q[0].size, np.float32)
        self._check(self.lib.ref_antipodal(self.h, _p(q[0]), _p(q[1]), _p(q[2]), _p(out), C.c_uint64(out.size)))
        return out

    def antipodal_gradient(self, qx, qy, qz) -> np.ndarray:
        q = [_f32(v) for v in (qx, qy, qz)]
        g = [np.empty(q[0].size, np.float32) for _ in range(3)]
        self._check(self.lib.ref_antipodal_gradient(self.h, _p(q[0]), _p(q[1]), _p(q[2]), _p(g[0]), _p(g[1]),
                                                    _p(g[2]), C.c_uint64(q[0].size)))
        return np.stack(g, axis=1)

    def time_antipodal(self, qx, qy, qz, warmup: int = 2, iters: int = 5) -> float:
        q = [_f32(v) for v in (qx, qy, qz)]
        ms = C.c_float()
        self._check(self.lib.ref_time_antipodal(self.h, _p(q[0]), _p(q[1]), _p(q[2]), C.c_uint64(q[0].size),
                                                C.c_int(warmup), C.c_int(iters), C.byref(ms)))
        return float(ms.value)

    def time_build(self, method: int, radius: int, bits: int, iters: int) -> float:
        ms = C.c_float()
        self._check(self.lib.ref_time_build(self.h, C.c_int(method), C.c_uint32(radius), C.c_int(bits),
                                            C.c_int(iters), C.byref(ms)))
        return float(ms.value)

    def time_refit(self, order: int = -1, iters: int = 5) -> float:
        """Device ms of gwn_refit_bvh (order -1) or gwn_refit_bvh_moment<order> on the built BVH."""
        ms = C.c_float()
        self._check(self.lib.ref_time_refit(self.h, C.c_int(order), C.c_int(iters), C.byref(ms)))
        return float(ms.value)

    def update_refit(self, x, y, z) -> None:
        xs, ys, zs = (_f32(v) for v in (x, y, z))
        self._check(self.lib.ref_update_refit(self.h, _p(xs), _p(ys), _p(zs), C.c_uint64(xs.size)))

    def preprocess(self, bits: int = 64):
        nt = self._keep[3].size
        codes = np.zeros(nt, np.uint64)
        ids = np.zeros(nt, np.uint32)
        aabbs = np.zeros((nt, 6), np.float32)
        self._check(self.lib.ref_preprocess(self.h, C.c_int(bits), _p(codes), _p(ids), _p(aabbs)))
        return codes, ids, aabbs


def ref_binary(method: int, bits: int, sorted_codes: np.ndarray, sorted_aabbs: np.ndarray, radius: int = 8):
    lib_ = ref_lib()
    if lib_ is None:
        raise RuntimeError("oracle/_ref/libgwnref.so is not built")
    c = np.ascontiguousarray(sorted_codes, np.uint64)
    a = np.ascontiguousarray(sorted_aabbs, np.float32)
    n = c.size
    nodes = np.zeros((n - 1, 4), np.uint32)
    bounds = np.zeros((n - 1, 6), np.float32)
    root = C.c_uint32()
    rc = lib_.ref_binary(C.c_int(method), C.c_int(bits), C.c_uint64(n), _p(c), _p(a), C.c_uint32(radius), _p(nodes),
                         _p(bounds), C.byref(root))
    if rc != 0:
        raise RuntimeError(f"reference binary build failed: {lib_.ref_last_message().decode()}")
    return nodes, bounds, int(root.value)


def ref_exact_f64(mesh: dict, qx, qy, qz) -> np.ndarray:
    lib_ = ref_lib()
    if lib_ is None:
        raise RuntimeError("oracle/_ref/libgwnref.so is not built")
    x, y, z = (np.ascontiguousarray(mesh[k], dtype=np.float64) for k in "xyz")
    i0, i1, i2 = _u32(mesh["i0"]), _u32(mesh["i1"]), _u32(mesh["i2"])
    q = [np.ascontiguousarray(v, dtype=np.float64) for v in (qx, qy, qz)]
    out = np.empty(q[0].size, np.float64)
    rc = lib_.ref_exact_f64(_p(x), _p(y), _p(z), C.c_uint64(x.size), _p(i0), _p(i1), _p(i2), C.c_uint64(i0.size),
                            _p(q[0]), _p(q[1]), _p(q[2]), _p(out), C.c_uint64(out.size))
    if rc != 0:
        raise RuntimeError(f"reference FP64 exact failed: {lib_.ref_last_message().decode()}")
    return out


# ---- canonical forms for comparisons up to node numbering -----------------------------------------


def canonical_wide(nodes: np.ndarray, root_ref: int) -> list:
    """Nested tuple of (child kind, primitive offset/count or subtree) per slot, depth first."""
    import sys

    sys.setrecursionlimit(100000)
    nd = nodes.reshape(-1, 4)

    def walk(i: int):
        res = []
        for s in range(4):
            r = int(nd[i, s]["reference"])
            if not (r >> 47) & 1:
                res.append(None)
            elif (r >> 48) == 0:
                res.append(walk(r & ((1 << 47) - 1)))
            else:
                res.append(("L", r & ((1 << 47) - 1), r >> 48))
        return tuple(res)

    if (root_ref >> 48) != 0:
        return [("L", root_ref & ((1 << 47) - 1), root_ref >> 48)]
    return [walk(root_ref & ((1 << 47) - 1))]


def binary_leaf_sets(nodes: np.ndarray, root: int) -> set:
    """Set of frozensets of leaf ids under every internal node (numbering independent)."""
    nd = np.asarray(nodes, np.uint32).reshape(-1, 4)
    n = nd.shape[0]
    order = []
    stack = [root]
    while stack:
        v = stack.pop()
        order.append(v)
        if nd[v, 1] == 1:
            stack.append(int(nd[v, 0]))
        if nd[v, 3] == 1:
            stack.append(int(nd[v, 2]))
    leaves = {}
    for v in reversed(order):
        s = []
        for idx, kind in ((nd[v, 0], nd[v, 1]), (nd[v, 2], nd[v, 3])):
            s += [int(idx)] if kind == 2 else leaves[int(idx)]
        leaves[v] = s
    assert len(order) == n, "binary tree does not reach every internal node"
    return {frozenset(v) for v in leaves.values()}


def binary_leaf_set_hashes(nodes: np.ndarray, root: int, seed: int = 0x5EED) -> np.ndarray:
    """Numbering-independent fingerprint of a binary tree for million-leaf trees: per internal node
    the sum (mod 2^64) of one random 64-bit word per leaf under it, mixed with the leaf count,
    sorted. Two trees with the same family of leaf sets give equal arrays; two that differ in any
    node's leaf set collide with probability about 2^-64 per pair. Vectorised bottom-up over the
    breadth-first levels; raises if the tree does not reach every internal node."""
    nd = np.asarray(nodes, np.uint32).reshape(-1, 4)
    n_int = nd.shape[0]
    words = np.random.default_rng(seed).integers(0, np.iinfo(np.uint64).max, n_int + 1, dtype=np.uint64,
                                                 endpoint=True)
    levels = []
    frontier = np.array([root], np.int64)
    seen = 0
    while frontier.size:
        levels.append(frontier)
        seen += frontier.size
        if seen > n_int:
            raise AssertionError("binary tree revisits internal nodes")
        kids = [nd[frontier, 0][nd[frontier, 1] == 1], nd[frontier, 2][nd[frontier, 3] == 1]]
        frontier = np.concatenate(kids).astype(np.int64)
    if seen != n_int:
        raise AssertionError("binary tree does not reach every internal node")
    h = np.zeros(n_int, np.uint64)
    cnt = np.zeros(n_int, np.uint64)
    for lev in reversed(levels):
        for side in (0, 2):
            idx = nd[lev, side].astype(np.int64)
            leaf = nd[lev, side + 1] == 2
            h[lev] += np.where(leaf, words[np.minimum(idx, n_int)], h[np.minimum(idx, n_int - 1)])
            cnt[lev] += np.where(leaf, np.uint64(1), cnt[np.minimum(idx, n_int - 1)])
    return np.sort(h ^ (cnt * np.uint64(0x9E3779B97F4A7C15)))


def match_wide_nodes(nodes_a: np.ndarray, root_a: int, nodes_b: np.ndarray, root_b: int) -> np.ndarray:
    """Pair the nodes of two structurally identical BVH4s by walking both from the root in slot
    order. Returns idx with nodes_b[idx[i]] corresponding to nodes_a[i]; raises if the trees differ."""
    na = nodes_a.reshape(-1, 4)
    nb = nodes_b.reshape(-1, 4)
    if na.shape[0] != nb.shape[0]:
        raise AssertionError("node counts differ")
    idx = np.full(na.shape[0], -1, np.int64)
    if na.shape[0] == 0:
        return idx
    off = (1 << 47) - 1
    stack = [(int(root_a) & off, int(root_b) & off)]
    while stack:
        i, j = stack.pop()
        idx[i] = j
        for s in range(4):
            ra, rb = int(na[i, s]["reference"]), int(nb[j, s]["reference"])
            va, vb = (ra >> 47) & 1, (rb >> 47) & 1
            if va != vb or (ra >> 48) != (rb >> 48):
                raise AssertionError(f"trees differ at node {i}/{j} slot {s}")
            if va and (ra >> 48) == 0:
                stack.append((ra & off, rb & off))
            elif va and (ra & off) != (rb & off):
                raise AssertionError(f"leaf ranges differ at node {i}/{j} slot {s}")
    if (idx < 0).any():
        raise AssertionError("unreachable nodes")
    return idx
