#pragma once

/// \file gwn_bvh_refit.cuh
/// \brief gwn_refit_bvh (bounds + triangle records, in place) and gwn_refit_bvh_moment<Order>.
///
/// Semantics of smallgwn's include/gwn/gwn_bvh_refit.cuh:25-51: refit keeps hierarchy, primitive
/// order and stack bounds, publishes a new revision (so moments formed earlier become stale) and
/// makes the BVH unqueryable when a device-side failure happens after mutation began; moment refit
/// replaces the moment object with coefficients aligned to the BVH's current revision.

#include <cuda_runtime_api.h>

#include "gwn_bvh.cuh"
#include "gwn_geometry.cuh"

namespace gwn {

template <int Width, gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] gwn_status gwn_refit_bvh(gwn_geometry_object<Real, Index> const &geometry,
                                       gwn_bvh_object<Width, Real, Index> &bvh,
                                       cudaStream_t const stream = gwn_default_stream()) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
        auto &aux = detail::object_access::aux(bvh);
        gwnb_bvh4_f32 v = detail::to_gwnb(bvh.accessor(), aux, detail::object_access::capacity(bvh));
        std::uint64_t const before = v.revision;
        int const rc = gwnb_bvh4_refit_f32(&g, &v, detail::gwnb_stream(stream));
        aux = v.aux;
        detail::from_gwnb(v, bvh.accessor());
        if (rc == GWNB_OK || (before != 0 && v.revision == 0))
            bvh.set_stream(stream);
        return detail::gwnb_to_status(rc);
    }
}

template <int Order, int Width, gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] gwn_status gwn_refit_bvh_moment(gwn_bvh_object<Width, Real, Index> const &bvh,
                                              gwn_bvh_moment_object<Width, Order, Real, Index> &moment,
                                              cudaStream_t const stream = gwn_default_stream()) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        auto &bvh_mut = const_cast<gwn_bvh_object<Width, Real, Index> &>(bvh);
        auto &aux = detail::object_access::aux(bvh_mut);
        gwnb_bvh4_f32 v = detail::to_gwnb(bvh.accessor(), aux, detail::object_access::capacity(bvh_mut));
        gwnb_moment4_f32 staging{};
        int const rc = gwnb_moment4_refit_f32(&v, Order, &staging, detail::gwnb_stream(stream));
        aux = v.aux; // derived state may have been created for a hand-assembled accessor
        if (rc != GWNB_OK)
            return detail::gwnb_to_status(rc);
        gwn_bvh_moment_object<Width, Order, Real, Index> replacement;
        replacement.accessor().nodes = cuda::std::span<gwn_bvh_moment_node<Width, Order, Real>>(
            static_cast<gwn_bvh_moment_node<Width, Order, Real> *>(staging.nodes), staging.node_count);
        replacement.accessor().bvh_revision = staging.bvh_revision;
        detail::object_access::moment_aux(replacement) = staging.aux;
        replacement.set_stream(stream);
        swap(moment, replacement);
        return gwn_status::ok();
    }
}

} // namespace gwn
