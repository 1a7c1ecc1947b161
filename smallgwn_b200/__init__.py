"""smallgwn_b200 -- B200-native (sm_100a) generalized winding numbers behind smallgwn's API.

The product is libgwnb.so (CUDA kernels + the C ABI of include/gwnb.h). This package builds it
(`build.py`), binds it with ctypes (`_lib.py`) and mirrors smallgwn's public API in Python
(`api.py`) for tests and benchmarks. `meshes.py` generates the seeded synthetic workloads.
"""
from .api import (  # noqa: F401
    gwn_batch,
    gwn_boundary_chain_object,
    gwn_build_boundary_chain,
    gwn_bvh4_moment_object,
    gwn_bvh4_object,
    gwn_bvh_build_method,
    gwn_bvh_build_options,
    gwn_build_bvh,
    gwn_compute_ray_first_hit_batch,
    gwn_compute_winding_gradient_antipodal_batch,
    gwn_compute_winding_number_antipodal_batch,
    gwn_compute_unsigned_distance_batch,
    gwn_compute_winding_gradient_taylor_batch,
    gwn_compute_winding_number_exact_batch,
    gwn_compute_winding_number_taylor_batch,
    gwn_error,
    gwn_geometry_object,
    gwn_geometry_view,
    gwn_query_batch_config,
    gwn_ray_first_hit_status,
    gwn_refit_bvh,
    gwn_refit_bvh_moment,
    gwn_status,
    gwn_taylor_saved,
    gwn_update_geometry,
    gwn_upload_geometry,
    gwn_upload_geometry_from_eigen,
    gwn_winding_taylor_backward,
    gwn_winding_taylor_forward,
    load_scene,
    near_precision,
    ray_hit_records,
    read_ply,
    save_scene,
    write_ply,
)
