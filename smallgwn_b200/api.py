"""Python mirror of smallgwn's public API over libgwnb.so.

Names, argument meaning and error behaviour follow smallgwn's C++ API
(include/gwn/gwn_geometry.cuh, gwn_bvh.cuh, gwn_bvh_build.cuh, gwn_bvh_refit.cuh, gwn_query.cuh):
every call returns a ``gwn_status``; objects own device storage, are rebound to the stream of the
last successful mutating call and are replaced atomically (staging and swap) so a failed call
leaves the previous state intact. Device buffers are torch CUDA tensors (or raw device pointers).
Only width 4, float32 positions and uint32 indices are provided, as in the C ABI.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib


class gwn_error(enum.IntEnum):
    success = 0
    invalid_argument = 1
    cuda_runtime_error = 2
    internal_error = 3


@dataclass
class gwn_status:
    """Mirror of gwn::gwn_status (include/gwn/gwn_utils.cuh:223-283)."""
    error: gwn_error = gwn_error.success
    message: str = ""

    def is_ok(self) -> bool:
        return self.error == gwn_error.success

    @staticmethod
    def ok() -> "gwn_status":
        return gwn_status()

    def __bool__(self) -> bool:  # truthiness = success, for terse checks
        return self.is_ok()


def _status(rc: int) -> gwn_status:
    if rc == _lib.GWNB_OK:
        return gwn_status()
    return gwn_status(gwn_error(rc), _lib.last_error())


class gwn_bvh_build_method(enum.IntEnum):
    """Mirror of gwn::gwn_bvh_build_method (include/gwn/gwn_bvh_build.cuh:15-20)."""
    k_hploc = 0
    k_lbvh = 1


@dataclass
class gwn_bvh_build_options:
    """Mirror of gwn::gwn_bvh_build_options (include/gwn/gwn_bvh_build.cuh:22-28)."""
    method: int = gwn_bvh_build_method.k_hploc
    hploc_search_radius: int = 8


@dataclass(frozen=True)
class gwn_query_batch_config:
    """Mirror of gwn::gwn_query_batch_config (include/gwn/gwn_query.cuh:48-61)."""
    block_size: int = 256
    stack_capacity: int = 64


class near_precision(enum.IntEnum):
    plain = _lib.GWNB_NEAR_PLAIN
    compensated = _lib.GWNB_NEAR_COMPENSATED


# Compensated near field: (query, triangle) pairs whose numerator and denominator are both below
# this fraction of |a||b||c| are evaluated in FP64 (about 0.03 pairs per near-surface query).
FP64_THRESHOLD = 1.0 / 16.0


def _stream(stream) -> int | None:
    if stream is None:
        return None  # cudaStreamLegacy / stream 0
    if isinstance(stream, int):
        return stream or None
    handle = getattr(stream, "cuda_stream", None)
    if handle is not None:
        return int(handle) or None
    raise TypeError(f"unsupported stream object {stream!r}")


def _ptr(buf) -> int | None:
    if buf is None:
        return None
    if isinstance(buf, int):
        return buf or None
    dp = getattr(buf, "data_ptr", None)
    if dp is not None:
        if not buf.is_cuda:
            raise ValueError("device buffers must be CUDA tensors")
        if not buf.is_contiguous():
            raise ValueError("device buffers must be contiguous")
        return int(dp()) or None
    raise TypeError(f"unsupported device buffer {type(buf)!r}")


def _numel(buf) -> int:
    if buf is None:
        return 0
    return int(buf.numel())


def _host(arr, dtype) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(arr), dtype=dtype)
    return a


class _stream_mixin:
    def __init__(self) -> None:
        self._stream = None

    def stream(self):
        return self._stream

    def set_stream(self, stream) -> None:
        self._stream = stream


class gwn_geometry_object(_stream_mixin):
    """Mirror of gwn::gwn_geometry_object<float, uint32_t> (include/gwn/gwn_geometry.cuh:98-149)."""

    def __init__(self) -> None:
        super().__init__()
        self._view = _lib.geometry_f32()

    def accessor(self) -> _lib.geometry_f32:
        return self._view

    def vertex_count(self) -> int:
        return int(self._view.vertex_count)

    def triangle_count(self) -> int:
        return int(self._view.triangle_count)

    def has_data(self) -> bool:
        return self.vertex_count() != 0 or self.triangle_count() != 0

    def clear(self) -> None:
        if self.has_data():
            _lib.load().gwnb_geometry_release_f32(C.byref(self._view), _stream(self._stream))
        self._view = _lib.geometry_f32()

    def __del__(self) -> None:
        try:
            self.clear()
        except Exception:
            pass


class gwn_geometry_view:
    """Non-owning geometry over caller device buffers (torch CUDA tensors: float32 x, y, z and
    int32/uint32 i0, i1, i2), e.g. slices of one shared vertex buffer; accepted wherever a
    gwn_geometry_object is. The tensors are held, so they outlive the view."""

    def __init__(self, x, y, z, i0, i1, i2) -> None:
        n, t = _numel(x), _numel(i0)
        if not (_numel(y) == n == _numel(z)) or not (_numel(i1) == t == _numel(i2)):
            raise ValueError("geometry view: SoA spans must have identical lengths")
        self._keep = (x, y, z, i0, i1, i2)
        self._view = _lib.geometry_f32(_ptr(x), _ptr(y), _ptr(z), n, _ptr(i0), _ptr(i1), _ptr(i2), t)

    def accessor(self) -> _lib.geometry_f32:
        return self._view

    def vertex_count(self) -> int:
        return int(self._view.vertex_count)

    def triangle_count(self) -> int:
        return int(self._view.triangle_count)


def gwn_upload_geometry(obj: gwn_geometry_object, x, y, z, i0, i1, i2, stream=None) -> gwn_status:
    """Upload host SoA positions and indices; replaces ``obj`` only on success."""
    lib = _lib.load()
    xs, ys, zs = (_host(a, np.float32) for a in (x, y, z))
    a0, a1, a2 = (_host(a, np.uint32) for a in (i0, i1, i2))
    if not (xs.size == ys.size == zs.size):
        return gwn_status(gwn_error.invalid_argument, "Vertex SoA spans must have identical lengths.")
    if not (a0.size == a1.size == a2.size):
        return gwn_status(gwn_error.invalid_argument, "Triangle SoA spans must have identical lengths.")
    staging = _lib.geometry_f32()
    rc = lib.gwnb_geometry_upload_f32(
        C.byref(staging), xs.ctypes.data or None, ys.ctypes.data or None, zs.ctypes.data or None, xs.size,
        a0.ctypes.data or None, a1.ctypes.data or None, a2.ctypes.data or None, a0.size, _stream(stream))
    if rc != _lib.GWNB_OK:
        return _status(rc)
    obj.clear()
    obj._view = staging
    obj.set_stream(stream)
    return gwn_status()


def gwn_upload_geometry_from_eigen(obj: gwn_geometry_object, vertices, triangles, stream=None) -> gwn_status:
    """Upload an N x 3 vertex matrix and an M x 3 triangle matrix (any array-like: numpy arrays as
    libigl's bindings return them, row- or column-major). Checks and messages follow smallgwn's
    include/gwn/gwn_eigen_bridge.cuh:26-132: floating-point indices must be finite and
    integer-valued, every index in [0, vertex_count); replaces ``obj`` only on success."""
    V = np.asarray(vertices)
    F = np.asarray(triangles)
    if V.ndim != 2 or F.ndim != 2 or V.shape[1] != 3 or F.shape[1] != 3:
        return gwn_status(gwn_error.invalid_argument, "Eigen inputs must be Nx3 vertices and Mx3 triangles.")
    nv = V.shape[0]
    if nv > 0 and nv - 1 > 0xFFFFFFFF:
        return gwn_status(gwn_error.invalid_argument, "Vertex count exceeds index range.")
    bad = gwn_status(gwn_error.invalid_argument, "Eigen triangle indices must be integer-valued in [0, vertex_count).")
    if F.size:
        if F.dtype.kind == "f":
            with np.errstate(invalid="ignore"):
                if not (np.isfinite(F).all() and (np.floor(F) == F).all()):
                    return bad
        elif F.dtype.kind not in "iu":
            return bad
        if F.min() < 0 or F.max() >= nv:
            return bad
    Fi = F.astype(np.uint32)
    Vf = V.astype(np.float32)
    return gwn_upload_geometry(obj, Vf[:, 0], Vf[:, 1], Vf[:, 2], Fi[:, 0], Fi[:, 1], Fi[:, 2], stream)


def gwn_update_geometry(obj: gwn_geometry_object, x, y, z, stream=None) -> gwn_status:
    """Copy new host (numpy) or device (torch CUDA) positions into an uploaded geometry."""
    lib = _lib.load()
    if hasattr(x, "is_cuda") and x.is_cuda:
        n = _numel(x)
        if not (_numel(y) == n == _numel(z)):
            return gwn_status(gwn_error.invalid_argument, "Vertex SoA spans must have identical lengths.")
        rc = lib.gwnb_geometry_update_device_f32(C.byref(obj._view), _ptr(x), _ptr(y), _ptr(z), n, _stream(stream))
    else:
        xs, ys, zs = (_host(a, np.float32) for a in (x, y, z))
        if not (xs.size == ys.size == zs.size):
            return gwn_status(gwn_error.invalid_argument, "Vertex SoA spans must have identical lengths.")
        rc = lib.gwnb_geometry_update_f32(C.byref(obj._view), xs.ctypes.data or None, ys.ctypes.data or None,
                                          zs.ctypes.data or None, xs.size, _stream(stream))
        obj._keepalive = (xs, ys, zs)  # host memory must outlive the asynchronous copy
    if rc == _lib.GWNB_OK:
        obj.set_stream(stream)
    return _status(rc)


def _assign(view, value) -> None:
    """Overwrites a view structure in place, so that C code holding its address (a batch lends the
    BVH and moment objects of its meshes) keeps seeing the object rather than a dropped copy."""
    C.memmove(C.addressof(view), C.addressof(value), C.sizeof(view))


class gwn_bvh4_object(_stream_mixin):
    """Mirror of gwn::gwn_bvh4_object<float, uint32_t> (include/gwn/gwn_bvh.cuh:329-381)."""

    def __init__(self) -> None:
        super().__init__()
        self._view = _lib.bvh4_f32()

    def accessor(self) -> _lib.bvh4_f32:
        return self._view

    def has_data(self) -> bool:
        v = self._view
        if v.revision == 0 or not (v.root.reference >> 47) & 1 or v.primitive_count == 0:
            return False
        return True

    def clear(self) -> None:
        if self._view.primitive_count or self._view.aux:
            _lib.load().gwnb_bvh4_release_f32(C.byref(self._view), _stream(self._stream))
        _assign(self._view, _lib.bvh4_f32())

    def __del__(self) -> None:
        try:
            self.clear()
        except Exception:
            pass


def gwn_build_bvh(geometry: gwn_geometry_object, bvh: gwn_bvh4_object,
                  options: gwn_bvh_build_options | None = None, stream=None, morton_bits: int = 64) -> gwn_status:
    """Build a BVH4 (LBVH or H-PLOC binary builder + wide collapse). Strong guarantee."""
    opt = options or gwn_bvh_build_options()
    staging = _lib.bvh4_f32()
    rc = _lib.load().gwnb_bvh4_build_f32(C.byref(geometry._view), int(opt.method), int(opt.hploc_search_radius),
                                         int(morton_bits), C.byref(staging), _stream(stream))
    if rc != _lib.GWNB_OK:
        return _status(rc)
    bvh.clear()
    _assign(bvh._view, staging)
    bvh.set_stream(stream)
    return gwn_status()


def gwn_refit_bvh(geometry: gwn_geometry_object, bvh: gwn_bvh4_object, stream=None) -> gwn_status:
    """Refit bounds and triangle records in place (synchronizes, publishes a new revision)."""
    before = bvh._view.revision
    rc = _lib.load().gwnb_bvh4_refit_f32(C.byref(geometry._view), C.byref(bvh._view), _stream(stream))
    if rc == _lib.GWNB_OK or (before != 0 and bvh._view.revision == 0):
        bvh.set_stream(stream)
    return _status(rc)


class gwn_bvh4_moment_object(_stream_mixin):
    """Mirror of gwn::gwn_bvh4_moment_object<Order, float, uint32_t> (include/gwn/gwn_bvh.cuh:387-430)."""

    def __init__(self, order: int) -> None:
        super().__init__()
        if order not in (0, 1, 2):
            raise ValueError("Taylor order must be 0, 1, or 2.")
        self.order = order
        self._view = _lib.moment4_f32(order=order)

    def accessor(self) -> _lib.moment4_f32:
        return self._view

    def has_data(self) -> bool:
        return self._view.bvh_revision != 0

    def is_valid_for(self, bvh: gwn_bvh4_object) -> bool:
        return bvh.has_data() and self._view.bvh_revision == bvh._view.revision

    def clear(self) -> None:
        if self._view.nodes or self._view.aux:
            _lib.load().gwnb_moment4_release_f32(C.byref(self._view), _stream(self._stream))
        _assign(self._view, _lib.moment4_f32(order=self.order))

    def __del__(self) -> None:
        try:
            self.clear()
        except Exception:
            pass


def gwn_refit_bvh_moment(order: int, bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object, stream=None) -> gwn_status:
    """Compute Taylor moments of ``order`` aligned to ``bvh``; replaces ``moment`` on success."""
    if moment.order != order:
        return gwn_status(gwn_error.invalid_argument, "Moment object order does not match the requested order.")
    staging = _lib.moment4_f32(order=order)
    rc = _lib.load().gwnb_moment4_refit_f32(C.byref(bvh._view), order, C.byref(staging), _stream(stream))
    if rc != _lib.GWNB_OK:
        return _status(rc)
    moment.clear()
    _assign(moment._view, staging)
    moment.set_stream(stream)
    return gwn_status()


def _check_spans(qx, qy, qz, out) -> gwn_status | None:
    n = _numel(qx)
    if not (_numel(qy) == n == _numel(qz)):
        return gwn_status(gwn_error.invalid_argument, "Query SoA spans must have identical lengths.")
    if _numel(out) != n:
        return gwn_status(gwn_error.invalid_argument, "Output span size must match query count.")
    return None


def gwn_compute_winding_number_exact_batch(bvh: gwn_bvh4_object, qx, qy, qz, out, stream=None,
                                           config: gwn_query_batch_config = gwn_query_batch_config()) -> gwn_status:
    """Exact winding numbers of a device batch (asynchronous)."""
    lib = _lib.load()
    if not bvh.has_data():
        return gwn_status(gwn_error.invalid_argument, "BVH object contains no queryable data.")
    bad = _check_spans(qx, qy, qz, out)
    if bad is not None:
        return bad
    rc = lib.gwnb_winding_exact_batch_f32(C.byref(bvh._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(out),
                                          _numel(out), int(config.block_size), _stream(stream))
    return _status(rc)


# gwnb_taylor_options::per_thread: "timed" takes the faster of the two walks, chosen from the timed
# first two calls of the same kind (identical results either way)
TRAVERSALS = {"warp": _lib.GWNB_WALK_WARP, "thread": _lib.GWNB_WALK_THREAD, "timed": _lib.GWNB_WALK_TIMED}


def _options(config: gwn_query_batch_config, sort_queries: bool, precision: int, fp64_threshold: float,
             per_thread: bool = False, traversal: str = "warp"):
    walk = 1 if per_thread else TRAVERSALS[traversal]
    return _lib.taylor_options(int(config.block_size), int(config.stack_capacity), 1 if sort_queries else 0,
                               int(precision), float(fp64_threshold), walk)


def gwn_compute_winding_number_taylor_batch(order: int, bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object,
                                            qx, qy, qz, out, accuracy_scale: float = 2.0, stream=None,
                                            config: gwn_query_batch_config = gwn_query_batch_config(),
                                            sort_queries: bool = True, precision: int = near_precision.plain,
                                            fp64_threshold: float = FP64_THRESHOLD, per_thread: bool = False,
                                            traversal: str = "warp") -> gwn_status:
    """Taylor-approximated winding numbers of a device batch (asynchronous). ``traversal``: "warp"
    (the default: 32 ordered queries per warp walk one traversal together), "thread" (one
    independent walk per query; also ``per_thread=True``) or "timed" (the faster of the two for
    calls of this kind, from the timed first two); all give identical results."""
    if moment.order != order:
        return gwn_status(gwn_error.invalid_argument, "Moment object order does not match the requested order.")
    if traversal not in TRAVERSALS:
        return gwn_status(gwn_error.invalid_argument, f"Unknown traversal {traversal!r}.")
    bad = _check_spans(qx, qy, qz, out)
    if bad is not None:
        return bad
    opt = _options(config, sort_queries, precision, fp64_threshold, per_thread, traversal)
    rc = _lib.load().gwnb_winding_taylor_batch_f32(
        C.byref(bvh._view), C.byref(moment._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(out), _numel(out),
        float(accuracy_scale), C.byref(opt), _stream(stream))
    return _status(rc)


def gwn_compute_winding_gradient_taylor_batch(order: int, bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object,
                                              qx, qy, qz, gx, gy, gz, accuracy_scale: float = 2.0, stream=None,
                                              config: gwn_query_batch_config = gwn_query_batch_config(),
                                              sort_queries: bool = True, traversal: str = "warp") -> gwn_status:
    """Gradient of the Taylor winding number with respect to the query point (``traversal`` as for
    the value batch)."""
    if moment.order != order:
        return gwn_status(gwn_error.invalid_argument, "Moment object order does not match the requested order.")
    if traversal not in TRAVERSALS:
        return gwn_status(gwn_error.invalid_argument, f"Unknown traversal {traversal!r}.")
    for g in (gx, gy, gz):
        bad = _check_spans(qx, qy, qz, g)
        if bad is not None:
            return bad
    opt = _options(config, sort_queries, near_precision.plain, FP64_THRESHOLD, traversal=traversal)
    rc = _lib.load().gwnb_winding_gradient_taylor_batch_f32(
        C.byref(bvh._view), C.byref(moment._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(gx), _ptr(gy), _ptr(gz),
        _numel(qx), float(accuracy_scale), C.byref(opt), _stream(stream))
    return _status(rc)


def taylor_traversal_stats(bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object, qx, qy, qz, nodes, far, near,
                           accuracy_scale: float = 2.0, stream=None) -> gwn_status:
    """Per-query counts of nodes entered, far-field children accepted and exact triangles."""
    rc = _lib.load().gwnb_winding_taylor_stats_f32(
        C.byref(bvh._view), C.byref(moment._view), _ptr(qx), _ptr(qy), _ptr(qz), _numel(qx), float(accuracy_scale),
        _ptr(nodes), _ptr(far), _ptr(near), _stream(stream))
    return _status(rc)


def taylor_form_probe(bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object, qx, qy, qz, accuracy_scale: float = 2.0,
                      precision: int = near_precision.plain, sort_queries: bool = True,
                      stream=None) -> tuple[gwn_status, dict]:
    """Sampled walk statistics (gwnb_taylor_form_probe_f32): per sampled warp, the nodes and leaf
    triangles the warp-cooperative walk takes and the largest per-query node and triangle counts (the
    per-thread walk's lockstep work), the number of sampled warps, and per_thread = 1 when the
    per-thread traversal suits the batch."""
    out = (C.c_double * 6)()
    opt = _options(gwn_query_batch_config(stack_capacity=max(64, bvh.accessor().internal_stack_bound)), sort_queries,
                   precision, FP64_THRESHOLD)
    rc = _lib.load().gwnb_taylor_form_probe_f32(C.byref(bvh._view), C.byref(moment._view), _ptr(qx), _ptr(qy),
                                                _ptr(qz), _numel(qx), float(accuracy_scale), C.byref(opt), out,
                                                _stream(stream))
    keys = ("warp_nodes", "warp_tris", "lane_max_nodes", "lane_max_tris", "sampled_warps", "per_thread")
    return _status(rc), dict(zip(keys, list(out)))


def select_taylor_form(geometry: gwn_geometry_object, bvh: gwn_bvh4_object, moments: dict, qx, qy, qz,
                       max_error: float, accuracy_scales=(1.0, 1.5, 2.0, 2.5, 3.0, 3.25, 3.5, 4.0, 5.0, 6.0, 8.0),
                       precision: int = near_precision.compensated, stream=None) -> tuple[gwn_status, dict]:
    """Taylor order and accuracy scale for an error bound, chosen on a device sample of queries
    (gwnb_taylor_select_f32): ``moments`` maps the orders to consider to their moment objects. Returns
    (status, {order, accuracy_scale, max_error, sample_ms, stack_capacity, candidates_passing})."""
    arr = (C.POINTER(_lib.moment4_f32) * 3)()
    for o, m in moments.items():
        arr[int(o)] = C.pointer(m._view)
    betas = (C.c_float * len(accuracy_scales))(*accuracy_scales)
    out = _lib.taylor_choice()
    rc = _lib.load().gwnb_taylor_select_f32(C.byref(geometry._view), C.byref(bvh._view), arr, _ptr(qx), _ptr(qy),
                                            _ptr(qz), _numel(qx), float(max_error), betas, len(accuracy_scales),
                                            int(precision), C.byref(out), _stream(stream))
    return _status(rc), {f: getattr(out, f) for f, _ in _lib.taylor_choice._fields_}


def exact_winding_fp64(geometry: gwn_geometry_object, qx, qy, qz, out, stream=None) -> gwn_status:
    """FP64 exact winding numbers of the float mesh (float32 queries, float64 output tensor)."""
    bad = _check_spans(qx, qy, qz, out)
    if bad is not None:
        return bad
    rc = _lib.load().gwnb_winding_exact_geometry_fp64(C.byref(geometry._view), _ptr(qx), _ptr(qy), _ptr(qz),
                                                      _ptr(out), _numel(out), _stream(stream))
    return _status(rc)


# gwn::gwn_ray_first_hit_status / gwn_ray_first_hit_result<float, uint32_t>
# (include/gwn/gwn_query.cuh:63-96): one 32-byte record per ray.
class gwn_ray_first_hit_status(enum.IntEnum):
    k_miss = _lib.GWNB_RAY_MISS
    k_hit = _lib.GWNB_RAY_HIT
    k_overflow = _lib.GWNB_RAY_OVERFLOW


RAY_HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32),
                          ("geometric_normal_x", np.float32), ("geometric_normal_y", np.float32),
                          ("geometric_normal_z", np.float32), ("primitive_id", np.uint32), ("status", np.uint8),
                          ("padding", np.uint8, (3,))])
RAY_HIT_WORDS = 8  # four-byte words per record


def ray_hit_records(out) -> np.ndarray:
    """Host copy of a ray-hit output buffer (CUDA tensor of 8 four-byte words per ray) as a numpy
    structured array with the fields of gwn_ray_first_hit_result."""
    raw = out.detach().contiguous().view(-1).cpu().numpy().view(np.uint8)
    return raw.view(RAY_HIT_DTYPE)


def _ray_rows(out) -> int:
    n = _numel(out)
    if out is not None and out.element_size() != 4:
        raise ValueError("ray-hit output must be a tensor of 4-byte words (8 per ray)")
    return n // RAY_HIT_WORDS


def _spatial_options(config: gwn_query_batch_config, sort_queries: bool, traversal: str = "warp"):
    return _lib.spatial_options(int(config.block_size), int(config.stack_capacity), 1 if sort_queries else 0,
                                TRAVERSALS[traversal])


class gwn_boundary_chain_object(_stream_mixin):
    """Mirror of gwn::gwn_boundary_chain_object<uint32_t> (include/gwn/gwn_boundary.cuh:61-110): the
    algebraic boundary of an oriented triangle chain (directed edges with positive multiplicity).
    ``has_data()`` means built; a closed mesh has ``has_data()`` and ``edge_count() == 0``."""

    def __init__(self) -> None:
        super().__init__()
        self._view = _lib.boundary_chain_u32()

    def accessor(self) -> _lib.boundary_chain_u32:
        return self._view

    def has_data(self) -> bool:
        return bool(self._view.is_built)

    def edge_count(self) -> int:
        return int(self._view.edge_count)

    def empty(self) -> bool:
        return self.edge_count() == 0

    def rows(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Host copy of the (start, end, multiplicity) rows."""
        n = self.edge_count()
        if n == 0:
            return np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint64)
        v = self._view
        return (np.frombuffer(_copy_to_host(v.start_vertex, 4 * n), np.uint32),
                np.frombuffer(_copy_to_host(v.end_vertex, 4 * n), np.uint32),
                np.frombuffer(_copy_to_host(v.multiplicity, 8 * n), np.uint64))

    def clear(self) -> None:
        if self.has_data():
            _lib.load().gwnb_boundary_chain_release_u32(C.byref(self._view), _stream(self._stream))
        self._view = _lib.boundary_chain_u32()

    def __del__(self) -> None:
        try:
            self.clear()
        except Exception:
            pass


def gwn_build_boundary_chain(geometry, out: gwn_boundary_chain_object, stream=None) -> gwn_status:
    """Build the algebraic boundary chain of an uploaded geometry; replaces ``out`` only on success
    (include/gwn/gwn_boundary.cuh:116-125)."""
    staging = _lib.boundary_chain_u32()
    rc = _lib.load().gwnb_boundary_chain_build_u32(C.byref(geometry.accessor()), C.byref(staging), _stream(stream))
    if rc != _lib.GWNB_OK:
        return _status(rc)
    out.clear()
    out._view = staging
    out.set_stream(stream)
    return gwn_status()


def gwn_compute_winding_number_antipodal_batch(geometry, bvh: gwn_bvh4_object, boundary: gwn_boundary_chain_object,
                                               qx, qy, qz, out, stream=None,
                                               config: gwn_query_batch_config = gwn_query_batch_config(),
                                               sort_queries: bool = False) -> gwn_status:
    """Antipodal winding numbers of a device batch (asynchronous): signed +z (+x, +y on retry) ray
    crossings through the BVH plus the boundary spherical-area term; NaN where every axis is
    singular (include/gwn/gwn_query.cuh:497-556)."""
    n = _numel(qx)
    if not (_numel(qy) == n == _numel(qz)):
        return gwn_status(gwn_error.invalid_argument, "Query SoA spans require identical lengths.")
    if _numel(out) != n:
        return gwn_status(gwn_error.invalid_argument, "Output span size differs from query count.")
    opt = _spatial_options(config, sort_queries)
    rc = _lib.load().gwnb_winding_antipodal_batch_f32(C.byref(geometry.accessor()), C.byref(bvh._view),
                                                      C.byref(boundary._view), _ptr(qx), _ptr(qy), _ptr(qz),
                                                      _ptr(out), n, C.byref(opt), _stream(stream))
    return _status(rc)


def gwn_compute_winding_gradient_antipodal_batch(geometry, boundary: gwn_boundary_chain_object, qx, qy, qz, gx, gy,
                                                 gz, stream=None,
                                                 config: gwn_query_batch_config = gwn_query_batch_config()
                                                 ) -> gwn_status:
    """Gradient of the antipodal boundary term (include/gwn/gwn_query.cuh:596-654)."""
    n = _numel(qx)
    if not (_numel(qy) == n == _numel(qz)):
        return gwn_status(gwn_error.invalid_argument, "Query SoA spans require identical lengths.")
    if not (_numel(gx) == n == _numel(gy) == _numel(gz)):
        return gwn_status(gwn_error.invalid_argument, "Output span sizes differ from query count.")
    rc = _lib.load().gwnb_winding_gradient_antipodal_batch_f32(
        C.byref(geometry.accessor()), C.byref(boundary._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(gx), _ptr(gy),
        _ptr(gz), n, int(config.block_size), _stream(stream))
    return _status(rc)


def gwn_compute_unsigned_distance_batch(bvh: gwn_bvh4_object, qx, qy, qz, out, culling_band: float = float("inf"),
                                        stream=None, config: gwn_query_batch_config = gwn_query_batch_config(),
                                        sort_queries: bool = False, traversal: str = "warp") -> gwn_status:
    """Unsigned point-to-mesh distances of a device batch, at most ``culling_band`` (asynchronous).
    ``sort_queries`` traverses in Hilbert order of the points (results stay at input positions);
    such a batch is walked by ``traversal``: "warp" (32 neighbouring queries per warp walk one
    traversal), "thread" (one walk per query) or "timed" (the faster of the two for calls of this
    kind, from the timed first two); identical results."""
    if not bvh.has_data():
        return gwn_status(gwn_error.invalid_argument, "BVH object contains no queryable data.")
    if traversal not in TRAVERSALS:
        return gwn_status(gwn_error.invalid_argument, f"Unknown traversal {traversal!r}.")
    bad = _check_spans(qx, qy, qz, out)
    if bad is not None:
        return bad
    opt = _spatial_options(config, sort_queries, traversal)
    rc = _lib.load().gwnb_unsigned_distance_batch_f32(C.byref(bvh._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(out),
                                                      _numel(out), float(culling_band), C.byref(opt), _stream(stream))
    return _status(rc)


def gwn_compute_ray_first_hit_batch(bvh: gwn_bvh4_object, ox, oy, oz, dx, dy, dz, out, t_min: float = 0.0,
                                    t_max: float = float("inf"), stream=None,
                                    config: gwn_query_batch_config = gwn_query_batch_config(),
                                    sort_queries: bool = False) -> gwn_status:
    """Nearest ray-triangle hits of a device batch on [t_min, t_max] (asynchronous). ``out`` holds
    8 four-byte words per ray (a gwn_ray_first_hit_result record; see ray_hit_records)."""
    if not bvh.has_data():
        return gwn_status(gwn_error.invalid_argument, "BVH object contains no queryable data.")
    n = _numel(ox)
    if any(_numel(a) != n for a in (oy, oz, dx, dy, dz)) or _ray_rows(out) != n or \
            (out is not None and _numel(out) % RAY_HIT_WORDS != 0):
        return gwn_status(gwn_error.invalid_argument, "ray first-hit: mismatched span sizes")
    opt = _spatial_options(config, sort_queries)
    rc = _lib.load().gwnb_ray_first_hit_batch_f32(C.byref(bvh._view), _ptr(ox), _ptr(oy), _ptr(oz), _ptr(dx),
                                                  _ptr(dy), _ptr(dz), _ptr(out), n, float(t_min), float(t_max),
                                                  C.byref(opt), _stream(stream))
    return _status(rc)


def spatial_traversal_stats(bvh: gwn_bvh4_object, qx, qy, qz, nodes, tris, dx=None, dy=None, dz=None,
                            culling_band: float = float("inf"), t_min: float = 0.0, t_max: float = float("inf"),
                            stream=None) -> gwn_status:
    """Per-query internal nodes entered and triangles tested by the distance batch (no directions)
    or the ray batch (directions given); int32 CUDA tensors `nodes`, `tris`."""
    kind = _lib.GWNB_SPATIAL_RAY if dx is not None else _lib.GWNB_SPATIAL_DISTANCE
    rc = _lib.load().gwnb_spatial_stats_f32(C.byref(bvh._view), kind, _ptr(qx), _ptr(qy), _ptr(qz), _ptr(dx),
                                            _ptr(dy), _ptr(dz), _numel(qx), float(culling_band), float(t_min),
                                            float(t_max), _ptr(nodes), _ptr(tris), _stream(stream))
    return _status(rc)


def ray_order(bvh: gwn_bvh4_object, ox, oy, oz, dx, dy, dz, order, stream=None) -> gwn_status:
    """Traversal order of a ray batch (direction cell, then origin Hilbert index); `order` is an
    int32 CUDA tensor."""
    rc = _lib.load().gwnb_ray_order_f32(C.byref(bvh._view), _ptr(ox), _ptr(oy), _ptr(oz), _ptr(dx), _ptr(dy), _ptr(dz),
                                        _numel(ox), _ptr(order), _stream(stream))
    return _status(rc)


# ---- mesh and scene files ---------------------------------------------------------------------------

def read_ply(path) -> dict:
    """Triangle mesh of a PLY file (ASCII or binary; polygons split into fans) as the SoA dict the
    upload takes (x, y, z float32; i0, i1, i2 uint32). Raises ValueError on a refused file, as
    smallgwn's test loader returns no mesh (tests/test_mesh_io.cpp:43-92)."""
    lib = _lib.load()
    m = _lib.host_mesh_f32()
    rc = lib.gwnb_mesh_read_ply(str(path).encode(), C.byref(m))
    if rc != _lib.GWNB_OK:
        raise ValueError(_lib.last_error())
    try:
        nv, nt = int(m.vertex_count), int(m.triangle_count)
        fa = C.POINTER(C.c_float)
        ua = C.POINTER(C.c_uint32)
        out = {k: np.ctypeslib.as_array(C.cast(getattr(m, k), fa), (nv,)).copy() for k in "xyz"}
        out.update({k: np.ctypeslib.as_array(C.cast(getattr(m, k), ua), (nt,)).copy() for k in ("i0", "i1", "i2")})
    finally:
        lib.gwnb_host_mesh_free(C.byref(m))
    return out


def write_ply(path, mesh: dict, binary: bool = True) -> None:
    """Write a SoA mesh dict as PLY (float positions, uint32 index lists)."""
    arrs = {k: np.ascontiguousarray(mesh[k], np.float32) for k in "xyz"}
    arrs.update({k: np.ascontiguousarray(mesh[k], np.uint32) for k in ("i0", "i1", "i2")})
    m = _lib.host_mesh_f32(arrs["x"].ctypes.data, arrs["y"].ctypes.data, arrs["z"].ctypes.data, arrs["x"].size,
                           arrs["i0"].ctypes.data, arrs["i1"].ctypes.data, arrs["i2"].ctypes.data, arrs["i0"].size)
    rc = _lib.load().gwnb_mesh_write_ply(str(path).encode(), C.byref(m), 1 if binary else 0)
    if rc != _lib.GWNB_OK:
        raise ValueError(_lib.last_error())


def save_scene(path, geometry, bvh: gwn_bvh4_object, moments=(), stream=None) -> gwn_status:
    """Save geometry, BVH and moment objects (at most one per order) to one file."""
    ms = list(moments)
    arr = (C.POINTER(_lib.moment4_f32) * max(len(ms), 1))(*[C.pointer(m._view) for m in ms])
    rc = _lib.load().gwnb_scene_save_f32(str(path).encode(), C.byref(geometry.accessor()), C.byref(bvh._view), arr,
                                         len(ms), _stream(stream))
    return _status(rc)


def load_scene(path, stream=None):
    """Load a scene file: (status, geometry object, BVH object, {order: moment object}) with the
    moments refit from the loaded BVH and checked equal to the saved ones."""
    g = _lib.geometry_f32()
    b = _lib.bvh4_f32()
    ms = (_lib.moment4_f32 * 3)()
    mask = C.c_int(0)
    rc = _lib.load().gwnb_scene_load_f32(str(path).encode(), C.byref(g), C.byref(b), ms, C.byref(mask),
                                         _stream(stream))
    if rc != _lib.GWNB_OK:
        return _status(rc), None, None, {}
    geo = gwn_geometry_object()
    geo._view = g
    geo.set_stream(stream)
    bvh = gwn_bvh4_object()
    _assign(bvh._view, b)
    bvh.set_stream(stream)
    moments = {}
    for order in range(3):
        if mask.value & (1 << order):
            mo = gwn_bvh4_moment_object(order)
            _assign(mo._view, ms[order])
            mo.set_stream(stream)
            moments[order] = mo
    return gwn_status(), geo, bvh, moments


def query_order(bvh: gwn_bvh4_object, qx, qy, qz, order, stream=None) -> gwn_status:
    """Traversal-coherent (Hilbert) order of a query batch; `order` is an int32 CUDA tensor."""
    rc = _lib.load().gwnb_query_order_f32(C.byref(bvh._view), _ptr(qx), _ptr(qy), _ptr(qz), _numel(qx), _ptr(order),
                                          _stream(stream))
    return _status(rc)


def fp64_fallback_count(bvh: gwn_bvh4_object, stream=None) -> int:
    n = C.c_uint64(0)
    rc = _lib.load().gwnb_bvh4_fp64_fallback_count(C.byref(bvh._view), C.byref(n), _stream(stream))
    if rc != _lib.GWNB_OK:
        raise RuntimeError(_lib.last_error())
    return int(n.value)


def refit_bvh_async(geometry: gwn_geometry_object, bvh: gwn_bvh4_object, stream=None) -> gwn_status:
    """Stream-ordered refit without host synchronization (graph capturable)."""
    return _status(_lib.load().gwnb_bvh4_refit_async_f32(C.byref(geometry._view), C.byref(bvh._view),
                                                        _stream(stream)))


def refit_bvh_moment_async(bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object, stream=None) -> gwn_status:
    """Refit an existing moment object for the BVH's current geometry without synchronization."""
    return _status(_lib.load().gwnb_moment4_refit_async_f32(C.byref(bvh._view), C.byref(moment._view),
                                                           _stream(stream)))


def memory_stats() -> tuple[int, int]:
    """(bytes the library's device memory pool holds, bytes in live allocations), current device."""
    r, u = C.c_uint64(), C.c_uint64()
    rc = _lib.load().gwnb_memory_stats(C.byref(r), C.byref(u))
    if rc != _lib.GWNB_OK:
        raise RuntimeError(_lib.last_error())
    return int(r.value), int(u.value)


def launch_count() -> int:
    """Kernel launches the library has issued in this process (graph-captured launches count once)."""
    return int(_lib.load().gwnb_launch_count())


def fp32_fma_peak(iters: int = 16384, stream=None) -> tuple[float, float]:
    """Measured FP32 FMA throughput of the current GPU: (TFLOP/s, ms of the timed launch)."""
    tf, ms = C.c_double(), C.c_double()
    rc = _lib.load().gwnb_fp32_fma_peak(int(iters), C.byref(tf), C.byref(ms), _stream(stream))
    if rc != _lib.GWNB_OK:
        raise RuntimeError(_lib.last_error())
    return float(tf.value), float(ms.value)


def fail_allocation_after(count: int) -> int:
    """Failure injection (gwnb_fail_allocation_after): the library's device allocation after the
    next `count` fails as out of memory; a negative count disarms. Returns the previously armed
    count (-1: none armed, or it has fired)."""
    return int(_lib.load().gwnb_fail_allocation_after(int(count)))


def memory_trim(keep_bytes: int = 0) -> gwn_status:
    """Return the pool's cached device memory to the driver down to keep_bytes (or what is in use)."""
    return _status(_lib.load().gwnb_memory_trim(int(keep_bytes)))


def sync_bvh_status(bvh: gwn_bvh4_object, stream=None) -> gwn_status:
    """Synchronize, publish device-side root bounds and turn device error bits into a status."""
    return _status(_lib.load().gwnb_bvh4_sync_status_f32(C.byref(bvh._view), _stream(stream)))


# ---- adjoint of the Taylor batch ------------------------------------------------------------------

class gwn_taylor_saved:
    """What a forward pass keeps for its backward pass: the query buffers (held here, so they stay
    alive) and the BVH revision; the backward pass recomputes the traversal."""

    def __init__(self, queries) -> None:
        self._view = _lib.taylor_saved_f32()
        self._queries = queries


def gwn_winding_taylor_forward(order: int, bvh: gwn_bvh4_object, moment: gwn_bvh4_moment_object, qx, qy, qz, out,
                               accuracy_scale: float = 2.0, stream=None,
                               config: gwn_query_batch_config = gwn_query_batch_config(),
                               sort_queries: bool = True, precision: int = near_precision.plain,
                               fp64_threshold: float = FP64_THRESHOLD) -> tuple[gwn_status, gwn_taylor_saved | None]:
    """Taylor winding numbers (orders 0 and 1) plus the saved state of their backward pass."""
    if moment.order != order:
        return gwn_status(gwn_error.invalid_argument, "Moment object order does not match the requested order."), None
    bad = _check_spans(qx, qy, qz, out)
    if bad is not None:
        return bad, None
    saved = gwn_taylor_saved((qx, qy, qz))
    opt = _options(config, sort_queries, precision, fp64_threshold, False)
    rc = _lib.load().gwnb_winding_taylor_forward_f32(
        C.byref(bvh._view), C.byref(moment._view), _ptr(qx), _ptr(qy), _ptr(qz), _ptr(out), _numel(out),
        float(accuracy_scale), C.byref(opt), C.byref(saved._view), _stream(stream))
    st = _status(rc)
    return st, (saved if st.is_ok() else None)


def gwn_winding_taylor_backward(saved: gwn_taylor_saved, geometry: gwn_geometry_object | None, bvh: gwn_bvh4_object,
                                moment: gwn_bvh4_moment_object, grad_out, dvx=None, dvy=None, dvz=None, dqx=None,
                                dqy=None, dqz=None, stream=None) -> gwn_status:
    """dL/dV (vertex_count floats per axis, overwritten) and dL/dq (query count per axis) of
    L = sum_q grad_out[q] * w(q); pass None for a triple to skip it."""
    if saved is None:
        return gwn_status(gwn_error.invalid_argument, "Taylor backward: saved state must be non-null.")
    if _numel(grad_out) != int(saved._view.count):
        return gwn_status(gwn_error.invalid_argument, "Upstream gradient size must match the query count.")
    geo = C.byref(geometry._view) if geometry is not None else None
    rc = _lib.load().gwnb_winding_taylor_backward_f32(
        C.byref(saved._view), geo, C.byref(bvh._view), C.byref(moment._view), _ptr(grad_out), _ptr(dvx), _ptr(dvy),
        _ptr(dvz), _ptr(dqx), _ptr(dqy), _ptr(dqz), _stream(stream))
    return _status(rc)


# ---- batched dynamic meshes ---------------------------------------------------------------------------

class gwn_batch:
    """Many meshes refit and queried per frame in three persistent launches (gwnb_batch_*).

    ``meshes`` is a list of (geometry, bvh, moment, qx, qy, qz, out): each BVH built from its
    geometry, each moment object refit for it (one Taylor order for all), queries and outputs CUDA
    tensors. The objects and tensors must outlive the batch; frames refit the BVHs and moments in
    place. ``frame()`` is asynchronous and capturable in a CUDA graph once a frame or a tuning has
    run outside capture."""

    def __init__(self, meshes, accuracy_scale: float = 2.0, stream=None, precision: int = near_precision.plain,
                 fp64_threshold: float = FP64_THRESHOLD) -> None:
        self._handle = C.c_void_p()
        self._keep = list(meshes)
        arr = (_lib.batch_mesh_f32 * len(meshes))()
        for i, (geo, bvh, mom, qx, qy, qz, out) in enumerate(meshes):
            if _numel(out) != _numel(qx) or _numel(qy) != _numel(qx) or _numel(qz) != _numel(qx):
                raise ValueError(f"batch mesh {i}: query/output spans must have identical lengths")
            arr[i] = _lib.batch_mesh_f32(geo._view, C.pointer(bvh._view), C.pointer(mom._view), _ptr(qx), _ptr(qy),
                                         _ptr(qz), _ptr(out), _numel(qx))
        opt = _options(gwn_query_batch_config(), True, precision, fp64_threshold, False)
        rc = _lib.load().gwnb_batch_create_f32(arr, len(meshes), float(accuracy_scale), C.byref(opt),
                                               C.byref(self._handle), _stream(stream))
        self.status = _status(rc)
        self._stream = stream

    def ok(self) -> bool:
        return self.status.is_ok() and bool(self._handle)

    def tune(self, repetitions: int = 3, stream=None) -> tuple[gwn_status, dict]:
        t = _lib.batch_tuning()
        rc = _lib.load().gwnb_batch_tune_f32(self._handle, int(repetitions), C.byref(t), _stream(stream))
        return _status(rc), {f: getattr(t, f) for f, _ in _lib.batch_tuning._fields_}

    def set_tuning(self, refit_block: int, query_block: int, per_thread: int, sorted_queries: int,
                   grid_scale: int) -> gwn_status:
        t = _lib.batch_tuning(refit_block, query_block, per_thread, sorted_queries, grid_scale, 0.0)
        return _status(_lib.load().gwnb_batch_set_tuning_f32(self._handle, C.byref(t)))

    def frame(self, stream=None) -> gwn_status:
        return _status(_lib.load().gwnb_batch_frame_f32(self._handle, _stream(stream)))

    REFIT, MOMENTS, QUERY = _lib.GWNB_BATCH_REFIT, _lib.GWNB_BATCH_MOMENTS, _lib.GWNB_BATCH_QUERY

    def run(self, stages: int, stream=None) -> gwn_status:
        """Selected stages of a frame (REFIT | MOMENTS | QUERY)."""
        return _status(_lib.load().gwnb_batch_run_f32(self._handle, int(stages), _stream(stream)))

    def sync(self, stream=None) -> gwn_status:
        return _status(_lib.load().gwnb_batch_sync_f32(self._handle, _stream(stream)))

    def quality(self, stream=None) -> tuple[gwn_status, list]:
        """Per mesh, the BVH's surface-area cost now over its cost when built (gwnb_batch_quality_f32)."""
        out = (C.c_float * len(self._keep))()
        rc = _lib.load().gwnb_batch_quality_f32(self._handle, out, _stream(stream))
        return _status(rc), list(out)

    def rebuild(self, threshold: float, method: int = gwn_bvh_build_method.k_hploc, radius: int = 8,
                stream=None) -> tuple[gwn_status, int]:
        """Rebuild the BVHs (and moments) whose cost ratio exceeds ``threshold``; the mesh objects are
        updated in place. A frame graph captured before a rebuild that rebuilt anything must be
        captured again."""
        n = C.c_uint32()
        rc = _lib.load().gwnb_batch_rebuild_f32(self._handle, float(threshold), int(method), int(radius), C.byref(n),
                                                _stream(stream))
        return _status(rc), int(n.value)

    def release(self, stream=None) -> None:
        if self._handle:
            _lib.load().gwnb_batch_release_f32(self._handle, _stream(stream if stream is not None else self._stream))
            self._handle = C.c_void_p()

    def __del__(self) -> None:
        try:
            self.release()
        except Exception:
            pass


# ---- host views of device state (tests, diagnostics) ------------------------------------------------

NODE_DTYPE = np.dtype([("bounds", np.float32, (6,)), ("reference", np.uint64)])
TRI_DTYPE = np.dtype((np.float32, 9))


def _copy_to_host(ptr: int, nbytes: int) -> bytes:
    import torch

    if nbytes == 0:
        return b""
    buf = torch.empty(nbytes, dtype=torch.uint8)
    torch.cuda.synchronize()
    cudart = _cudart()
    rc = cudart.cudaMemcpy(C.c_void_p(buf.data_ptr()), C.c_void_p(ptr), C.c_size_t(nbytes), 2)
    if rc != 0:
        raise RuntimeError(f"cudaMemcpy failed ({rc})")
    return buf.numpy().tobytes()


_cudart_lib = None


def _cudart():
    global _cudart_lib
    if _cudart_lib is None:
        import glob
        import os

        cands = []
        try:
            import torch

            cands += glob.glob(os.path.join(os.path.dirname(torch.__file__), "lib", "libcudart*.so*"))
        except Exception:
            pass
        cands += glob.glob("/usr/local/cuda/lib64/libcudart.so*")
        for c in cands:
            try:
                _cudart_lib = C.CDLL(c)
                break
            except OSError:
                continue
        if _cudart_lib is None:
            raise RuntimeError("libcudart not found")
        _cudart_lib.cudaMemcpy.restype = C.c_int
        _cudart_lib.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return _cudart_lib


def bvh_host_arrays(bvh: gwn_bvh4_object) -> dict:
    """Copy nodes, primitive order and triangle records of a BVH to host numpy arrays."""
    v = bvh._view
    nodes = np.frombuffer(_copy_to_host(v.nodes, int(v.node_count) * 128), dtype=NODE_DTYPE).reshape(-1, 4)
    prims = np.frombuffer(_copy_to_host(v.primitive_indices, int(v.primitive_count) * 4), dtype=np.uint32)
    tris = np.frombuffer(_copy_to_host(v.triangles, int(v.primitive_count) * 36), dtype=np.float32).reshape(-1, 9)
    return {"nodes": nodes, "primitive_indices": prims, "triangles": tris,
            "root_reference": int(v.root.reference),
            "root_bounds": np.array([getattr(v.root.bounds, f) for f, _ in _lib.aabb_f32._fields_], np.float32),
            "internal_stack_bound": int(v.internal_stack_bound), "packed_stack_bound": int(v.packed_stack_bound),
            "revision": int(v.revision)}


def moment_host_array(moment: gwn_bvh4_moment_object) -> np.ndarray:
    """Copy smallgwn-layout moment nodes to host: shape (nodes, fields, 4)."""
    v = moment._view
    fields = {0: 7, 1: 13, 2: 23}[moment.order]
    raw = _copy_to_host(v.nodes, int(v.node_count) * fields * 16)
    return np.frombuffer(raw, dtype=np.float32).reshape(-1, fields, 4)
