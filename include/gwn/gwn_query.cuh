#pragma once

/// \file gwn_query.cuh
/// \brief Batch queries: exact, Taylor and antipodal winding numbers and gradients, unsigned
/// distance and ray first hit.
///
/// Template signatures follow smallgwn's include/gwn/gwn_query.cuh:41-96, :135-282, :308-445,
/// :497-654 and :688-756.
/// Batches validate their objects and spans, enqueue work on \p stream and return without
/// synchronizing. Deliberate difference: the traversal never traps. A query that would overflow
/// its stack writes NaN and raises a device error bit (read with gwnb_bvh4_sync_status_f32); the
/// overflow-callback parameter is accepted for source compatibility and is not invoked, because
/// device functors cannot cross the C ABI.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <limits>
#include <type_traits>

#include "gwn_boundary.cuh"
#include "gwn_bvh.cuh"
#include "gwn_geometry.cuh"

namespace gwn {

inline constexpr int k_gwn_default_query_batch_block_size = 256;
inline constexpr int k_gwn_default_traversal_stack_capacity = 64;

struct gwn_query_batch_config {
    int block_size = k_gwn_default_query_batch_block_size;
    int stack_capacity = k_gwn_default_traversal_stack_capacity;
};

template <gwn_query_batch_config Config>
concept gwn_query_batch_config_value = Config.block_size > 0 && Config.block_size <= 1024;

template <gwn_query_batch_config Config>
concept gwn_traversal_batch_config_value = gwn_query_batch_config_value<Config> && Config.stack_capacity > 0;

/// Accepted for source compatibility; see the file comment.
struct gwn_traversal_overflow_ignore {};

/// Completion state of a ray first-hit query (smallgwn include/gwn/gwn_query.cuh:63-68).
enum class gwn_ray_first_hit_status : std::uint8_t { k_miss = 0, k_hit = 1, k_overflow = 2 };

/// First-hit record (smallgwn include/gwn/gwn_query.cuh:70-96); the float / uint32_t instantiation
/// has the layout of gwnb_ray_hit_f32.
template <gwn_real_type Real, gwn_index_type Index = std::uint32_t> struct gwn_ray_first_hit_result {
    Real t{Real(-1)};
    Real u{Real(0)};
    Real v{Real(0)};
    Real geometric_normal_x{Real(0)};
    Real geometric_normal_y{Real(0)};
    Real geometric_normal_z{Real(0)};
    Index primitive_id{gwn_invalid_index<Index>()};
    gwn_ray_first_hit_status status{gwn_ray_first_hit_status::k_miss};

    [[nodiscard]] constexpr bool hit() const noexcept { return status == gwn_ray_first_hit_status::k_hit; }

private:
    std::uint8_t storage_padding_[sizeof(Index) == 4 ? 3 : 7]{};
};
static_assert(sizeof(gwn_ray_first_hit_result<float, std::uint32_t>) == sizeof(gwnb_ray_hit_f32));

/// Library-specific Taylor options (query ordering and near-field precision).
struct gwn_taylor_batch_options {
    bool sort_queries = true;
    int near_precision = GWNB_NEAR_PLAIN;
    // pairs whose numerator and denominator are both below threshold * |a||b||c| go to FP64; at
    // 1/16 that is ~0.03 pairs per query on near-surface sets, at no measurable cost
    float fp64_threshold = 1.0f / 16.0f;
    // GWNB_WALK_WARP, GWNB_WALK_THREAD or GWNB_WALK_TIMED (the faster walk for calls of this kind,
    // chosen from the timed first two); identical results
    int walk = GWNB_WALK_WARP;
};

namespace detail {

template <int Width, gwn_real_type Real, gwn_index_type Index>
[[nodiscard]] inline gwnb_bvh4_f32 query_view(gwn_bvh_object<Width, Real, Index> const &bvh) noexcept {
    auto &b = const_cast<gwn_bvh_object<Width, Real, Index> &>(bvh);
    return to_gwnb(bvh.accessor(), object_access::aux(b), object_access::capacity(b));
}

template <int Width, gwn_real_type Real, gwn_index_type Index>
inline void store_aux(gwn_bvh_object<Width, Real, Index> const &bvh, gwnb_bvh4_f32 const &v) noexcept {
    object_access::aux(const_cast<gwn_bvh_object<Width, Real, Index> &>(bvh)) = v.aux;
}

template <class T>
[[nodiscard]] inline gwn_status check_batch_spans(gwn_device_span<T const> x, gwn_device_span<T const> y,
                                                  gwn_device_span<T const> z, std::size_t out_size) noexcept {
    if (x.size() != y.size() || x.size() != z.size())
        return gwn_status::invalid_argument("Query SoA spans must have identical lengths.");
    if (x.size() != out_size)
        return gwn_status::invalid_argument("Output span size must match query count.");
    return gwn_status::ok();
}

} // namespace detail

template <gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t>
    requires gwn_query_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_winding_number_exact_batch(
    gwn_bvh_object<Width, Real, Index> const &bvh, gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const output,
    cudaStream_t const stream = gwn_default_stream()
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (!bvh.accessor().is_valid())
            return gwn_status::invalid_argument("BVH object contains no queryable data.");
        GWN_RETURN_ON_ERROR(detail::check_batch_spans(qx, qy, qz, output.size()));
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        int const rc = gwnb_winding_exact_batch_f32(&v, qx.data(), qy.data(), qz.data(), output.data(), output.size(),
                                                    Config.block_size, detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

template <int Order, gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t, typename OverflowCallback = gwn_traversal_overflow_ignore>
    requires gwn_traversal_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_winding_number_taylor_batch(
    gwn_bvh_object<Width, Real, Index> const &bvh, gwn_bvh_moment_object<Width, Order, Real, Index> const &moment,
    gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const output,
    Real const accuracy_scale = Real(2), cudaStream_t const stream = gwn_default_stream(),
    OverflowCallback const & = {}, gwn_taylor_batch_options const options = {}
) noexcept {
    static_assert(Order == 0 || Order == 1 || Order == 2, "Taylor order must be 0, 1, or 2.");
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        GWN_RETURN_ON_ERROR(detail::check_batch_spans(qx, qy, qz, output.size()));
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        gwnb_moment4_f32 m = moment.view();
        gwnb_taylor_options o{Config.block_size, Config.stack_capacity, options.sort_queries ? 1 : 0,
                              options.near_precision, options.fp64_threshold, options.walk};
        int const rc = gwnb_winding_taylor_batch_f32(&v, &m, qx.data(), qy.data(), qz.data(), output.data(),
                                                     output.size(), accuracy_scale, &o, detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

template <int Order, gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t, typename OverflowCallback = gwn_traversal_overflow_ignore>
    requires gwn_traversal_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_winding_gradient_taylor_batch(
    gwn_bvh_object<Width, Real, Index> const &bvh, gwn_bvh_moment_object<Width, Order, Real, Index> const &moment,
    gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const gx,
    gwn_device_span<Real> const gy, gwn_device_span<Real> const gz, Real const accuracy_scale = Real(2),
    cudaStream_t const stream = gwn_default_stream(), OverflowCallback const & = {}
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        GWN_RETURN_ON_ERROR(detail::check_batch_spans(qx, qy, qz, gx.size()));
        if (gy.size() != gx.size() || gz.size() != gx.size())
            return gwn_status::invalid_argument("Output span size must match query count.");
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        gwnb_moment4_f32 m = moment.view();
        gwnb_taylor_options o{Config.block_size, Config.stack_capacity, 1, GWNB_NEAR_PLAIN, 1.0f / 16.0f};
        int const rc = gwnb_winding_gradient_taylor_batch_f32(&v, &m, qx.data(), qy.data(), qz.data(), gx.data(),
                                                              gy.data(), gz.data(), gx.size(), accuracy_scale, &o,
                                                              detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

/// Unsigned point-to-mesh distances, at most \p culling_band (smallgwn gwn_query.cuh:135-183).
template <gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t, typename OverflowCallback = gwn_traversal_overflow_ignore>
    requires gwn_traversal_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_unsigned_distance_batch(
    gwn_bvh_object<Width, Real, Index> const &bvh, gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const output,
    Real const culling_band = std::numeric_limits<Real>::infinity(), cudaStream_t const stream = gwn_default_stream(),
    OverflowCallback const & = {}
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (!bvh.accessor().is_valid())
            return gwn_status::invalid_argument("BVH object contains no queryable data.");
        GWN_RETURN_ON_ERROR(detail::check_batch_spans(qx, qy, qz, output.size()));
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        gwnb_spatial_options const o{Config.block_size, Config.stack_capacity, 0, GWNB_WALK_WARP};
        int const rc = gwnb_unsigned_distance_batch_f32(&v, qx.data(), qy.data(), qz.data(), output.data(),
                                                        output.size(), culling_band, &o, detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

/// Nearest ray-triangle hits on [t_min, t_max] (smallgwn gwn_query.cuh:214-282). Among hits at
/// the same t the lower primitive id is reported.
template <gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t, typename OverflowCallback = gwn_traversal_overflow_ignore>
    requires gwn_traversal_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_ray_first_hit_batch(
    gwn_bvh_object<Width, Real, Index> const &bvh, gwn_device_span<std::type_identity_t<Real> const> const ox,
    gwn_device_span<std::type_identity_t<Real> const> const oy,
    gwn_device_span<std::type_identity_t<Real> const> const oz,
    gwn_device_span<std::type_identity_t<Real> const> const dx,
    gwn_device_span<std::type_identity_t<Real> const> const dy,
    gwn_device_span<std::type_identity_t<Real> const> const dz,
    gwn_device_span<gwn_ray_first_hit_result<Real, Index>> const output, Real const t_min = Real(0),
    Real const t_max = std::numeric_limits<Real>::infinity(), cudaStream_t const stream = gwn_default_stream(),
    OverflowCallback const & = {}
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (!bvh.accessor().is_valid())
            return gwn_status::invalid_argument("BVH object contains no queryable data.");
        std::size_t const n = ox.size();
        if (oy.size() != n || oz.size() != n || dx.size() != n || dy.size() != n || dz.size() != n ||
            output.size() != n)
            return gwn_status::invalid_argument("ray first-hit: mismatched span sizes");
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        gwnb_spatial_options const o{Config.block_size, Config.stack_capacity, 0, GWNB_WALK_WARP};
        int const rc = gwnb_ray_first_hit_batch_f32(&v, ox.data(), oy.data(), oz.data(), dx.data(), dy.data(),
                                                    dz.data(), reinterpret_cast<gwnb_ray_hit_f32 *>(output.data()), n,
                                                    t_min, t_max, &o, detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

/// Antipodal winding numbers (smallgwn gwn_query.cuh:497-556; Martens, Trettner and Bessmeltsev,
/// ACM TOG 45(4), 2026): +z, +x, +y coordinate-ray crossings plus the boundary term, NaN where
/// every axis is singular.
template <gwn_query_batch_config Config = gwn_query_batch_config{}, int Width, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t, typename OverflowCallback = gwn_traversal_overflow_ignore>
    requires gwn_traversal_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_winding_number_antipodal_batch(
    gwn_geometry_object<Real, Index> const &geometry, gwn_bvh_object<Width, Real, Index> const &bvh,
    gwn_boundary_chain_object<Index> const &boundary_chain,
    gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const output,
    cudaStream_t const stream = gwn_default_stream(), OverflowCallback const & = {}
) noexcept {
    if constexpr (Width != 4 || !detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (qx.size() != qy.size() || qx.size() != qz.size())
            return gwn_status::invalid_argument("Query SoA spans require identical lengths.");
        if (qx.size() != output.size())
            return gwn_status::invalid_argument("Output span size differs from query count.");
        gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
        gwnb_bvh4_f32 v = detail::query_view(bvh);
        gwnb_boundary_chain_u32 c = detail::to_gwnb(boundary_chain.accessor());
        gwnb_spatial_options const o{Config.block_size, Config.stack_capacity, 0, GWNB_WALK_WARP};
        int const rc = gwnb_winding_antipodal_batch_f32(&g, &v, &c, qx.data(), qy.data(), qz.data(), output.data(),
                                                        output.size(), &o, detail::gwnb_stream(stream));
        detail::store_aux(bvh, v);
        return detail::gwnb_to_status(rc);
    }
}

/// Gradient of the antipodal boundary term (smallgwn gwn_query.cuh:596-654).
template <gwn_query_batch_config Config = gwn_query_batch_config{}, gwn_real_type Real,
          gwn_index_type Index = std::uint32_t>
    requires gwn_query_batch_config_value<Config>
[[nodiscard]] gwn_status gwn_compute_winding_gradient_antipodal_batch(
    gwn_geometry_object<Real, Index> const &geometry, gwn_boundary_chain_object<Index> const &boundary_chain,
    gwn_device_span<std::type_identity_t<Real> const> const qx,
    gwn_device_span<std::type_identity_t<Real> const> const qy,
    gwn_device_span<std::type_identity_t<Real> const> const qz, gwn_device_span<Real> const gx,
    gwn_device_span<Real> const gy, gwn_device_span<Real> const gz, cudaStream_t const stream = gwn_default_stream()
) noexcept {
    if constexpr (!detail::k_supported<Real, Index>) {
        return detail::unsupported_instantiation();
    } else {
        if (qx.size() != qy.size() || qx.size() != qz.size())
            return gwn_status::invalid_argument("Query SoA spans require identical lengths.");
        if (qx.size() != gx.size() || qx.size() != gy.size() || qx.size() != gz.size())
            return gwn_status::invalid_argument("Output span sizes differ from query count.");
        gwnb_geometry_f32 g = detail::to_gwnb(geometry.accessor());
        gwnb_boundary_chain_u32 c = detail::to_gwnb(boundary_chain.accessor());
        int const rc = gwnb_winding_gradient_antipodal_batch_f32(&g, &c, qx.data(), qy.data(), qz.data(), gx.data(),
                                                                 gy.data(), gz.data(), gx.size(), Config.block_size,
                                                                 detail::gwnb_stream(stream));
        return detail::gwnb_to_status(rc);
    }
}

} // namespace gwn
