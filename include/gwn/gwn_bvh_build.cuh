#pragma once

/// \file gwn_bvh_build.cuh
/// \brief gwn_build_bvh with the k_lbvh / k_hploc binary builders and the BVH4 collapse.
///
/// Signature and options as smallgwn's include/gwn/gwn_bvh_build.cuh:15-39; implemented by
/// gwnb_bvh4_build_f32. Strong guarantee: \p bvh is replaced (and rebound to \p stream) only on
/// success.

#include <cuda_runtime_api.h>

#include <cstdint>

#include "gwn_bvh.cuh"
#include "gwn_geometry.cuh"

namespace gwn {

enum class gwn_bvh_build_method : std::uint8_t {
    k_hploc,
    k_lbvh,
};

struct gwn_bvh_build_options {
    gwn_bvh_build_method method = gwn_bvh_build_method::k_hploc;
    std::uint32_t hploc_search_radius = 8;
};

template <int Width, gwn_real_type Real, gwn_index_type Index, gwn_index_type MortonCode = std::uint64_t>
[[nodiscard]] gwn_status gwn_build_bvh(
    gwn_geometry_object<Real, Index> const &geometry, gwn_bvh_object<Width, Real, Index> &bvh,
    gwn_bvh_build_options const options = {}, cudaStream_t const stream = gwn_default_stream()
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        (void)geometry;
        (void)bvh;
        (void)options;
        (void)stream;
        return detail::unsupported_instantiation();
    } else {
        gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
        gwnb_bvh4_f32 staging{};
        int const method = options.method == gwn_bvh_build_method::k_hploc   ? GWNB_METHOD_HPLOC
                           : options.method == gwn_bvh_build_method::k_lbvh ? GWNB_METHOD_LBVH
                                                                            : -1;
        int const rc = gwnb_bvh4_build_f32(&g, method, options.hploc_search_radius,
                                           static_cast<int>(sizeof(MortonCode) * 8), &staging,
                                           detail::gwnb_stream(stream));
        if (rc != GWNB_OK)
            return detail::gwnb_to_status(rc);
        gwn_bvh_object<Width, Real, Index> replacement;
        detail::from_gwnb(staging, replacement.accessor());
        detail::object_access::aux(replacement) = staging.aux;
        detail::object_access::capacity(replacement) = staging.node_capacity;
        replacement.set_stream(stream);
        swap(bvh, replacement);
        return gwn_status::ok();
    }
}

} // namespace gwn
