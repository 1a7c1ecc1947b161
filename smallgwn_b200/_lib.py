"""ctypes binding of libgwnb.so (include/gwnb.h).

The structures below mirror the C declarations field by field. Loading fails loudly when the
library has not been built: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libgwnb.so"

GWNB_OK = 0
GWNB_INVALID_ARGUMENT = 1
GWNB_CUDA_RUNTIME_ERROR = 2
GWNB_INTERNAL_ERROR = 3

GWNB_METHOD_HPLOC = 0
GWNB_METHOD_LBVH = 1

GWNB_NEAR_PLAIN = 0
GWNB_NEAR_COMPENSATED = 1

GWNB_WALK_WARP = 0
GWNB_WALK_THREAD = 1
GWNB_WALK_TIMED = 2

GWNB_BATCH_REFIT = 1
GWNB_BATCH_MOMENTS = 2
GWNB_BATCH_QUERY = 4

GWNB_RAY_MISS = 0
GWNB_RAY_HIT = 1
GWNB_RAY_OVERFLOW = 2

GWNB_SPATIAL_DISTANCE = 0
GWNB_SPATIAL_RAY = 1


class aabb_f32(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")]


class child_f32(C.Structure):
    _fields_ = [("bounds", aabb_f32), ("reference", C.c_uint64)]


class node4_f32(C.Structure):
    _fields_ = [("children", child_f32 * 4)]


class triangle_f32(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("v0_x", "v0_y", "v0_z", "e1_x", "e1_y", "e1_z", "e2_x", "e2_y", "e2_z")]


class geometry_f32(C.Structure):
    _fields_ = [
        ("vertex_x", C.c_void_p), ("vertex_y", C.c_void_p), ("vertex_z", C.c_void_p),
        ("vertex_count", C.c_uint64),
        ("tri_i0", C.c_void_p), ("tri_i1", C.c_void_p), ("tri_i2", C.c_void_p),
        ("triangle_count", C.c_uint64),
    ]


class bvh4_f32(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p),
        ("node_count", C.c_uint64),
        ("node_capacity", C.c_uint64),
        ("primitive_indices", C.c_void_p),
        ("triangles", C.c_void_p),
        ("primitive_count", C.c_uint64),
        ("root", child_f32),
        ("internal_stack_bound", C.c_uint32),
        ("packed_stack_bound", C.c_uint32),
        ("revision", C.c_uint64),
        ("aux", C.c_void_p),
    ]


class moment4_f32(C.Structure):
    _fields_ = [
        ("order", C.c_int),
        ("nodes", C.c_void_p),
        ("node_count", C.c_uint64),
        ("bvh_revision", C.c_uint64),
        ("aux", C.c_void_p),
    ]


class taylor_options(C.Structure):
    _fields_ = [
        ("block_size", C.c_int),
        ("stack_capacity", C.c_int),
        ("sort_queries", C.c_int),
        ("near_precision", C.c_int),
        ("fp64_threshold", C.c_float),
        ("per_thread", C.c_int),
    ]


class taylor_saved_f32(C.Structure):
    _fields_ = [
        ("query_x", C.c_void_p),
        ("query_y", C.c_void_p),
        ("query_z", C.c_void_p),
        ("count", C.c_uint64),
        ("accuracy_scale", C.c_float),
        ("order", C.c_int),
        ("bvh_revision", C.c_uint64),
        ("options", taylor_options),
    ]


class batch_mesh_f32(C.Structure):
    _fields_ = [
        ("geometry", geometry_f32),
        ("bvh", C.POINTER(bvh4_f32)),
        ("moment", C.POINTER(moment4_f32)),
        ("query_x", C.c_void_p),
        ("query_y", C.c_void_p),
        ("query_z", C.c_void_p),
        ("output", C.c_void_p),
        ("query_count", C.c_uint64),
    ]


class taylor_choice(C.Structure):
    _fields_ = [
        ("order", C.c_int),
        ("accuracy_scale", C.c_float),
        ("max_error", C.c_float),
        ("sample_ms", C.c_float),
        ("stack_capacity", C.c_int),
        ("candidates_passing", C.c_int),
    ]


class batch_tuning(C.Structure):
    _fields_ = [
        ("refit_block", C.c_int),
        ("query_block", C.c_int),
        ("per_thread", C.c_int),
        ("sorted", C.c_int),
        ("grid_scale", C.c_int),
        ("frame_ms", C.c_float),
    ]


class spatial_options(C.Structure):
    _fields_ = [
        ("block_size", C.c_int),
        ("stack_capacity", C.c_int),
        ("sort_queries", C.c_int),
        ("per_thread", C.c_int),
    ]


class ray_hit_f32(C.Structure):
    _fields_ = [
        ("t", C.c_float), ("u", C.c_float), ("v", C.c_float),
        ("geometric_normal_x", C.c_float), ("geometric_normal_y", C.c_float), ("geometric_normal_z", C.c_float),
        ("primitive_id", C.c_uint32), ("status", C.c_uint8), ("padding", C.c_uint8 * 3),
    ]


class boundary_chain_u32(C.Structure):
    _fields_ = [
        ("start_vertex", C.c_void_p),
        ("end_vertex", C.c_void_p),
        ("multiplicity", C.c_void_p),
        ("edge_count", C.c_uint64),
        ("mesh_vertex_count", C.c_uint64),
        ("mesh_triangle_count", C.c_uint64),
        ("is_built", C.c_int),
    ]


class host_mesh_f32(C.Structure):
    _fields_ = [
        ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("vertex_count", C.c_uint64),
        ("i0", C.c_void_p), ("i1", C.c_void_p), ("i2", C.c_void_p), ("triangle_count", C.c_uint64),
    ]


class binary_node(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("left_index", "left_kind", "right_index", "right_kind")]


assert C.sizeof(child_f32) == 32 and C.sizeof(node4_f32) == 128 and C.sizeof(triangle_f32) == 36
assert C.sizeof(ray_hit_f32) == 32

P = C.c_void_p
U64 = C.c_uint64
U32 = C.c_uint32
I = C.c_int
F = C.c_float

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "gwnb_last_error_message": (C.c_char_p, []),
    "gwnb_last_cuda_error": (I, []),
    "gwnb_version": (C.c_char_p, []),
    "gwnb_cuda_runtime_version": (C.c_int, []),
    "gwnb_memory_stats": (C.c_int, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "gwnb_memory_trim": (C.c_int, [C.c_uint64]),
    "gwnb_fail_allocation_after": (C.c_int64, [C.c_int64]),
    "gwnb_launch_count": (C.c_uint64, []),
    "gwnb_fp32_fma_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    "gwnb_set_wait_limit": (C.c_int, [C.c_int64]),
    "gwnb_batch_quality_f32": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_void_p]),
    "gwnb_batch_rebuild_f32": (C.c_int, [C.c_void_p, C.c_float, C.c_int, C.c_uint32, C.POINTER(C.c_uint32),
                                         C.c_void_p]),
    "gwnb_taylor_select_f32": (C.c_int, [C.POINTER(geometry_f32), C.POINTER(bvh4_f32), C.POINTER(C.POINTER(moment4_f32)),
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_float,
                                         C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(taylor_choice),
                                         C.c_void_p]),
    "gwnb_wait_timeout_probe": (C.c_int, [C.c_int, C.c_void_p]),
    "gwnb_geometry_upload_f32": (I, [C.POINTER(geometry_f32), P, P, P, U64, P, P, P, U64, P]),
    "gwnb_geometry_update_f32": (I, [C.POINTER(geometry_f32), P, P, P, U64, P]),
    "gwnb_geometry_update_device_f32": (I, [C.POINTER(geometry_f32), P, P, P, U64, P]),
    "gwnb_geometry_release_f32": (None, [C.POINTER(geometry_f32), P]),
    "gwnb_bvh4_build_f32": (I, [C.POINTER(geometry_f32), I, U32, I, C.POINTER(bvh4_f32), P]),
    "gwnb_bvh4_release_f32": (None, [C.POINTER(bvh4_f32), P]),
    "gwnb_build_preprocess_f32": (I, [C.POINTER(geometry_f32), I, P, P, P, P]),
    "gwnb_build_binary_lbvh": (I, [P, I, U64, P, P, P, P, P]),
    "gwnb_build_binary_hploc": (I, [P, I, U64, P, U32, P, P, P, C.POINTER(U32), P]),
    "gwnb_radix_sort_pairs": (I, [P, P, P, P, U64, I, I, P]),
    "gwnb_bvh4_refit_f32": (I, [C.POINTER(geometry_f32), C.POINTER(bvh4_f32), P]),
    "gwnb_bvh4_refit_async_f32": (I, [C.POINTER(geometry_f32), C.POINTER(bvh4_f32), P]),
    "gwnb_bvh4_sync_status_f32": (I, [C.POINTER(bvh4_f32), P]),
    "gwnb_moment4_refit_f32": (I, [C.POINTER(bvh4_f32), I, C.POINTER(moment4_f32), P]),
    "gwnb_moment4_refit_async_f32": (I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P]),
    "gwnb_moment4_release_f32": (None, [C.POINTER(moment4_f32), P]),
    "gwnb_moment_node_bytes": (U64, [I]),
    "gwnb_winding_exact_batch_f32": (I, [C.POINTER(bvh4_f32), P, P, P, P, U64, I, P]),
    "gwnb_winding_taylor_batch_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, P, U64, F, C.POINTER(taylor_options), P]),
    "gwnb_winding_gradient_taylor_batch_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, P, P, P, U64, F, C.POINTER(taylor_options), P]),
    "gwnb_winding_taylor_stats_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, U64, F, P, P, P, P]),
    "gwnb_taylor_form_probe_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, U64, F, C.POINTER(taylor_options),
            C.POINTER(C.c_double), P]),
    "gwnb_bvh4_fp64_fallback_count": (I, [C.POINTER(bvh4_f32), C.POINTER(U64), P]),
    "gwnb_winding_exact_geometry_fp64": (I, [C.POINTER(geometry_f32), P, P, P, P, U64, P]),
    "gwnb_query_order_f32": (I, [C.POINTER(bvh4_f32), P, P, P, U64, P, P]),
    "gwnb_unsigned_distance_batch_f32": (
        I, [C.POINTER(bvh4_f32), P, P, P, P, U64, F, C.POINTER(spatial_options), P]),
    "gwnb_ray_first_hit_batch_f32": (
        I, [C.POINTER(bvh4_f32), P, P, P, P, P, P, P, U64, F, F, C.POINTER(spatial_options), P]),
    "gwnb_boundary_chain_build_u32": (I, [C.POINTER(geometry_f32), C.POINTER(boundary_chain_u32), P]),
    "gwnb_boundary_chain_release_u32": (None, [C.POINTER(boundary_chain_u32), P]),
    "gwnb_winding_antipodal_batch_f32": (
        I, [C.POINTER(geometry_f32), C.POINTER(bvh4_f32), C.POINTER(boundary_chain_u32), P, P, P, P, U64,
            C.POINTER(spatial_options), P]),
    "gwnb_winding_gradient_antipodal_batch_f32": (
        I, [C.POINTER(geometry_f32), C.POINTER(boundary_chain_u32), P, P, P, P, P, P, U64, I, P]),
    "gwnb_mesh_read_ply": (I, [C.c_char_p, C.POINTER(host_mesh_f32)]),
    "gwnb_host_mesh_free": (None, [C.POINTER(host_mesh_f32)]),
    "gwnb_mesh_write_ply": (I, [C.c_char_p, C.POINTER(host_mesh_f32), I]),
    "gwnb_scene_save_f32": (
        I, [C.c_char_p, C.POINTER(geometry_f32), C.POINTER(bvh4_f32), C.POINTER(C.POINTER(moment4_f32)), I, P]),
    "gwnb_scene_load_f32": (
        I, [C.c_char_p, C.POINTER(geometry_f32), C.POINTER(bvh4_f32), C.POINTER(moment4_f32), C.POINTER(I), P]),
    "gwnb_ray_order_f32": (I, [C.POINTER(bvh4_f32), P, P, P, P, P, P, U64, P, P]),
    "gwnb_spatial_stats_f32": (
        I, [C.POINTER(bvh4_f32), I, P, P, P, P, P, P, U64, F, F, F, P, P, P]),
    "gwnb_winding_taylor_batch_noalloc_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, P, U64, F, C.POINTER(taylor_options), P]),
    "gwnb_winding_taylor_forward_f32": (
        I, [C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P, P, P, P, U64, F, C.POINTER(taylor_options),
            C.POINTER(taylor_saved_f32), P]),
    "gwnb_winding_taylor_backward_f32": (
        I, [C.POINTER(taylor_saved_f32), C.POINTER(geometry_f32), C.POINTER(bvh4_f32), C.POINTER(moment4_f32), P,
            P, P, P, P, P, P, P]),
    "gwnb_batch_create_f32": (
        I, [C.POINTER(batch_mesh_f32), C.c_uint32, F, C.POINTER(taylor_options), C.POINTER(P), P]),
    "gwnb_batch_tune_f32": (I, [P, I, C.POINTER(batch_tuning), P]),
    "gwnb_batch_set_tuning_f32": (I, [P, C.POINTER(batch_tuning)]),
    "gwnb_batch_frame_f32": (I, [P, P]),
    "gwnb_batch_run_f32": (I, [P, C.c_uint, P]),
    "gwnb_batch_sync_f32": (I, [P, P]),
    "gwnb_batch_release_f32": (I, [P, P]),
}

_lib: C.CDLL | None = None


def library_path() -> Path:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load libgwnb.so and bind every entry point of include/gwnb.h. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(
            f"{_LIB_PATH} is missing: build it with `python -m smallgwn_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(str(_LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().gwnb_last_error_message().decode(errors="replace")
