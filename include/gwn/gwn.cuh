#pragma once

/// \file gwn.cuh
/// \brief Umbrella header of the drop-in API (smallgwn's include/gwn/gwn.cuh). Link against
/// libgwnb.so; a plain C++20 host compiler is enough (no --expt-relaxed-constexpr needed).

#include "gwn_boundary.cuh"
#include "gwn_bvh.cuh"
#include "gwn_bvh_build.cuh"
#include "gwn_bvh_refit.cuh"
#include "gwn_geometry.cuh"
#include "gwn_mesh_io.cuh"
#include "gwn_query.cuh"
#include "gwn_utils.cuh"
